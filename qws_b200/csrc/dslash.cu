// Wilson-clover hopping kernels for the DD solver (FP64, FP32, and FP16
// storage with FP32 arithmetic).
//
// One templated kernel covers every operator the reference spreads over
// ddd_in_*, ddd_out_pre/pos_*, jinv_ddd_in_s_ and the SAP update loops:
//   SEL  which hops:  inner (stay inside the SAP block; ddd_in, open block
//        faces, ddd_in_d.cc:91-190), outer (cross a block face; the
//        reference's halo path ddd_out_*), or all (ddd_d_/ddd_s_).
//   EPI  what is done with acc = A^-1 * (sum of selected hops):
//        EPI_D    out = src - kappa*acc                (ddd_in / D)
//        EPI_ADD  out += coef*acc                      (ddd_out_pos, factor coef)
//        EPI_JINV out = aux + kappa*acc                (one Richardson step
//                 x <- b + kappa A^-1 H_blk x, algebraically the reference's
//                 x + (b - D_blk x), static_solver.cc:77-139)
//        EPI_SAPE out = out + (aux - (src - kappa*acc)) (s_e += in_e - D_blk a_e,
//                 qws.cc:815-818 with the ddd_in result kept in registers)
//   T    storage format (float, double, H16); arithmetic in Arith<T>::R.
// Faces are not packed: a face hop reads the neighbouring block's site of
// the source field directly from HBM (the whole lattice is resident).
#include <type_traits>

#include "kernels.h"
#include "lattice.cuh"

namespace qwsg {

// How a thread's values map to memory.  Scalar: one (site, RHS) entry per
// thread in the storage format's own layout.  Pair (FP16 multi-RHS fields):
// two RHS of one site per thread as F2 lanes, IOP layout.
template <typename T>
struct OneRhs {
  using V = typename Arith<T>::R;
  using S = typename Store<T>::type;
  __device__ __forceinline__ static int lanes_log(const Geom& G) { return G.lgnr; }
  __device__ __forceinline__ static int pad(const Geom& G) { return spad(G); }
  __device__ __forceinline__ static int entry(const Geom& G, int g, int lane) { return sentry(G, g, lane); }
  __device__ __forceinline__ static void load_raw(const S* p, int pd, int e, V v[24], V& s) {
    IO<T>::load_spinor_raw(p, pd, e, v, s);
  }
  __device__ __forceinline__ static void load_half_raw(const S* p, int pd, int e, int up, V v[24], V& s) {
    IO<T>::load_half_raw(p, pd, e, up, v, s);
  }
  __device__ __forceinline__ static void load(const S* p, int pd, int e, V v[24]) {
    IO<T>::load_spinor(p, pd, e, v);
  }
  __device__ __forceinline__ static void store(S* p, int pd, int e, const V v[24]) {
    IO<T>::store_spinor(p, pd, e, v);
  }
  // A^-1 v with the site's clover, or the entry's (PRK: per-RHS kappa)
  template <bool PRK>
  __device__ __forceinline__ static void clover(const HopArgs<T>& a, int g, int lane, V v[24]) {
    if constexpr (PRK)
      clover_apply<T, V>(a.Cr, spad(a.G), sentry(a.G, g, lane), v);
    else
      clover_apply<T, V>(a.C, a.G.pad, g, v);
  }
  template <bool PRK>
  __device__ __forceinline__ static V coef(const HopArgs<T>& a, int lane) {
    if constexpr (PRK) return copysign(a.kap[lane], a.coef);
    return a.coef;
  }
};
struct TwoRhs {
  using V = F2;
  using S = __half;
  __device__ __forceinline__ static int lanes_log(const Geom& G) { return G.lgnr - 1; }
  __device__ __forceinline__ static int pad(const Geom& G) { return spad(G) >> 1; }
  __device__ __forceinline__ static int entry(const Geom& G, int g, int lane) {
    return (g << (G.lgnr - 1)) + lane;
  }
  __device__ __forceinline__ static void load_raw(const S* p, int pd, int e, V v[24], V& s) {
    IOP::load_spinor_raw(p, pd, e, v, s);
  }
  __device__ __forceinline__ static void load_half_raw(const S* p, int pd, int e, int up, V v[24], V& s) {
    IOP::load_half_raw(p, pd, e, up, v, s);
  }
  __device__ __forceinline__ static void load(const S* p, int pd, int e, V v[24]) {
    IOP::load_spinor(p, pd, e, v);
  }
  __device__ __forceinline__ static void store(S* p, int pd, int e, const V v[24]) {
    IOP::store_spinor(p, pd, e, v);
  }
  // the site's clover for both lanes, or each lane's own (PRK: per-RHS kappa)
  template <bool PRK>
  __device__ __forceinline__ static void clover(const HopArgs<H16>& a, int g, int lane, V v[24]) {
    if constexpr (PRK) {
      const int sp = spad(a.G), e0 = sentry(a.G, g, 2 * lane);
      clover_apply_with<F2>(
          [&](int i, F2 c[36]) {
            float s0[36], s1[36];
            IO<H16>::load_clover_block(a.Cr, sp, e0, i, s0);
            IO<H16>::load_clover_block(a.Cr, sp, e0 + 1, i, s1);
#pragma unroll
            for (int k = 0; k < 36; k++) c[k] = F2{s0[k], s1[k]};
          },
          v);
    } else {
      clover_apply<H16, F2>(a.C, a.G.pad, g, v);
    }
  }
  template <bool PRK>
  __device__ __forceinline__ static V coef(const HopArgs<H16>& a, int lane) {
    if constexpr (PRK)
      return F2{copysignf(a.kap[2 * lane], a.coef), copysignf(a.kap[2 * lane + 1], a.coef)};
    return Lanes<F2>::bcast(a.coef);
  }
};

template <typename T, typename P, int SEL, int MU, int DIR, typename V = typename P::V>
__device__ __forceinline__ void do_hop(const HopArgs<T>& a, const Site& s, int g, int lane,
                                       V acc[24]) {
  using R = typename Arith<T>::R;
  const bool face = DIR > 0 ? (s.lc[MU] == a.G.B[MU] - 1) : (s.lc[MU] == 0);
  if (face) {
    if (!(SEL & HOP_OUTER)) return;
  } else {
    if (!(SEL & HOP_INNER)) return;
  }
  int gn;
  if (!face) {
    gn = g + rot_step(a.G, MU, s.lc[MU], DIR);
  } else {
    int ncol;
    gn = nbr_across(a.G, s, MU, DIR, &ncol);
    if (ncol == a.zero_col) return;  // that colour's source is defined as zero
  }
  V v[24], sc;
  const int pd = P::pad(a.G), en = P::entry(a.G, gn, lane);
  // the projection and the link product are linear: the source's scale
  // (FP16 storage) is applied once, in the reconstruction
  if (MU == 3)
    P::load_half_raw(a.src, pd, en, DIR > 0, v, sc);
  else
    P::load_raw(a.src, pd, en, v, sc);
  V h[12], r[12], ul[18];
  project<V, MU, DIR>(v, h);
  {
    R u[18];
    if constexpr (std::is_same<T, float>::value) {
      if (a.U12)
        load_link12(a.U12, a.G.pad, MU, DIR > 0 ? g : gn, u);
      else
        IO<T>::load_link(a.U, a.G.pad, MU, DIR > 0 ? g : gn, u);
    } else {
      IO<T>::load_link(a.U, a.G.pad, MU, DIR > 0 ? g : gn, u);
    }
#pragma unroll
    for (int e = 0; e < 18; e++) ul[e] = Lanes<V>::bcast(u[e]);
  }
  if (DIR > 0)
    link_mul<V, false>(ul, h, r);
  else
    link_mul<V, true>(ul, h, r);
  V f = sc;
  if (MU == 3) {
    f = Lanes<V>::bcast((R)2) * sc;
    if (face && (DIR > 0 ? s.bc[3] == a.G.NB[3] - 1 : s.bc[3] == 0))
      f = Lanes<V>::bcast((R)(2 * a.G.tbc)) * sc;
  }
  reconstruct<V, MU, DIR>(r, acc, f);
}

// The FP32 block and face kernels and the FP16 block kernels are held to
// 64 registers (4 CTAs of 256 or 8 of 128 threads per SM): more warps in
// flight hide more of the neighbour-load latency that bounds them (FP32
// Richardson step 7% faster, FP16 SAP 4-8%); the full-lattice FP32
// operator and the FP16 face kernel spill at that bound and keep theirs.
template <typename T, int SEL>
struct MinCtas {
  static constexpr int value =
      ((std::is_same<T, float>::value && SEL != HOP_ALL) || (std::is_same<T, H16>::value && SEL == HOP_INNER))
          ? 4
          : 1;
};

template <typename T, typename P, int SEL, int EPI, bool PRK>
__device__ __forceinline__ void hop_site_at(const HopArgs<T>& a, const int i) {
  using V = typename P::V;
  const int ll = P::lanes_log(a.G);
  if (i >= (a.nsites << ll)) return;
  // consecutive threads: the right-hand sides (or RHS pairs) of one site,
  // then the next site
  const int si = i >> ll, lane = i & ((1 << ll) - 1);
  const int g = a.list ? __ldg(a.list + si) : a.site0 + si;
  Site s;
  decode_site(a.G, g, s);
  if (a.dom >= 0 && (s.bc[0] & 1) != a.dom) return;
  if (SEL == HOP_OUTER) {
    bool face = false;
#pragma unroll
    for (int mu = 0; mu < 4; mu++) face |= (s.lc[mu] == 0) | (s.lc[mu] == a.G.B[mu] - 1);
    if (!face) return;
  }
  V acc[24];
#pragma unroll
  for (int j = 0; j < 24; j++) acc[j] = Lanes<V>::bcast((typename Arith<T>::R)0);
  do_hop<T, P, SEL, 0, +1>(a, s, g, lane, acc);
  do_hop<T, P, SEL, 0, -1>(a, s, g, lane, acc);
  do_hop<T, P, SEL, 1, +1>(a, s, g, lane, acc);
  do_hop<T, P, SEL, 1, -1>(a, s, g, lane, acc);
  do_hop<T, P, SEL, 2, +1>(a, s, g, lane, acc);
  do_hop<T, P, SEL, 2, -1>(a, s, g, lane, acc);
  do_hop<T, P, SEL, 3, +1>(a, s, g, lane, acc);
  do_hop<T, P, SEL, 3, -1>(a, s, g, lane, acc);
  P::template clover<PRK>(a, g, lane, acc);
  const int pd = P::pad(a.G), e = P::entry(a.G, g, lane);
  const V coef = P::template coef<PRK>(a, lane);
  V o[24];
  if (EPI == EPI_D) {
    P::load(a.src, pd, e, o);
#pragma unroll
    for (int j = 0; j < 24; j++) o[j] = madd(coef, acc[j], o[j]);
  } else if (EPI == EPI_ADD) {
    P::load(a.out, pd, e, o);
#pragma unroll
    for (int j = 0; j < 24; j++) o[j] = madd(coef, acc[j], o[j]);
  } else if (EPI == EPI_JINV) {
    P::load(a.aux, pd, e, o);
#pragma unroll
    for (int j = 0; j < 24; j++) o[j] = madd(coef, acc[j], o[j]);
  } else {  // EPI_SAPE: coef = -kappa
    V in[24], av[24];
    P::load(a.out, pd, e, o);
    P::load(a.aux, pd, e, in);
    P::load(a.src, pd, e, av);
#pragma unroll
    for (int j = 0; j < 24; j++) o[j] = o[j] + (in[j] - madd(coef, acc[j], av[j]));
  }
  P::store(a.out, pd, e, o);
}

template <typename T, typename P, int SEL, int EPI, bool PRK>
__device__ __forceinline__ void hop_site(const HopArgs<T>& a) {
  hop_site_at<T, P, SEL, EPI, PRK>(a, blockIdx.x * blockDim.x + threadIdx.x);
}

// the same body with and without the 64-register bound (an explicit
// minimum of one CTA per SM would let the compiler spend every register)
// PRK: per-RHS kappa (clover planes and kappa per RHS, multi-RHS handles only)
template <typename T, int SEL, int EPI, bool PRK>
__global__ void __launch_bounds__(256) k_hop(const HopArgs<T> a) {
  hop_site<T, OneRhs<T>, SEL, EPI, PRK>(a);
}
template <typename T, int SEL, int EPI, bool PRK>
__global__ void __launch_bounds__(256, 4) k_hop_r64(const HopArgs<T> a) {
  hop_site<T, OneRhs<T>, SEL, EPI, PRK>(a);
}
// The full-lattice operators at a register bound of their own: FP64 at 128
// registers (4 CTAs of 128 threads per SM instead of 3; 56 bytes spill) and
// FP32 at 72 with CTAs of 128 (7 CTAs instead of 6): 13 % and 3 % faster
// at 32^3x64; the FP16 face kernel at 72 too (7 instead of 6, ~5 % faster).
// Bit for bit the same results.  (The FP16 block kernels at 56 registers,
// 9 CTAs, ran 5 % slower than at 64.)
template <typename T, int SEL, int EPI, bool PRK>
__global__ void __launch_bounds__(256, 2) k_hop_r128(const HopArgs<T> a) {
  hop_site<T, OneRhs<T>, SEL, EPI, PRK>(a);
}
template <typename T, int SEL, int EPI, bool PRK>
__global__ void __launch_bounds__(128, 7) k_hop_r73(const HopArgs<T> a) {
  hop_site<T, OneRhs<T>, SEL, EPI, PRK>(a);
}
// FP16 fields with two or more RHS: two RHS per thread in packed FP32x2
// arithmetic (the link and clover of the site serve both lanes)
template <int SEL, int EPI, bool PRK>
__global__ void __launch_bounds__(256) k_hop_pair(const HopArgs<H16> a) {
  hop_site<H16, TwoRhs, SEL, EPI, PRK>(a);
}

// Several lattices in one launch (a group solve; one right-hand side each):
// block b runs threads [(b - starts[l]) * blockDim, ...) of member l's own
// launch, with l's arguments copied into shared memory first, so every
// member runs exactly the code and arithmetic of its own launch.
template <typename T, int SEL, int EPI>
__device__ __forceinline__ void hop_multi_body(const HopArgs<T>* __restrict__ args,
                                               const int* __restrict__ starts, int n) {
  __shared__ HopArgs<T> sa;
  const int l = group_member(starts, n, blockIdx.x);
  group_load_args(sa, args + l);
  hop_site_at<T, OneRhs<T>, SEL, EPI, false>(sa, (blockIdx.x - starts[l]) * blockDim.x +
                                                     threadIdx.x);
}
template <typename T, int SEL, int EPI>
__global__ void __launch_bounds__(256) k_hop_multi(const HopArgs<T>* __restrict__ args,
                                                   const int* __restrict__ starts, int n) {
  hop_multi_body<T, SEL, EPI>(args, starts, n);
}
template <typename T, int SEL, int EPI>
__global__ void __launch_bounds__(256, 4) k_hop_multi_r64(const HopArgs<T>* __restrict__ args,
                                                          const int* __restrict__ starts, int n) {
  hop_multi_body<T, SEL, EPI>(args, starts, n);
}

template <typename T, int SEL, int EPI, bool PRK>
static void launch_v(const HopArgs<T>& a, cudaStream_t st) {
  const int threads = a.G.hop_threads;
  if constexpr (std::is_same<T, H16>::value) {
    if (a.G.nr >= 2) {
      const int blocks = ((a.nsites << (a.G.lgnr - 1)) + threads - 1) / threads;
      k_hop_pair<SEL, EPI, PRK><<<blocks, threads, 0, st>>>(a);
      return;
    }
  }
  const int blocks = ((a.nsites << a.G.lgnr) + threads - 1) / threads;
  if constexpr (SEL == HOP_ALL && !PRK && std::is_same<T, double>::value) {
    k_hop_r128<T, SEL, EPI, PRK><<<blocks, threads, 0, st>>>(a);
    return;
  }
  if constexpr (!PRK && ((SEL == HOP_ALL && std::is_same<T, float>::value) ||
                         (SEL == HOP_OUTER && std::is_same<T, H16>::value))) {
    if (threads == 128) {  // (the bound assumes CTAs of at most 128 threads)
      k_hop_r73<T, SEL, EPI, PRK><<<blocks, threads, 0, st>>>(a);
      return;
    }
  }
  if constexpr (MinCtas<T, SEL>::value == 4)
    k_hop_r64<T, SEL, EPI, PRK><<<blocks, threads, 0, st>>>(a);
  else
    k_hop<T, SEL, EPI, PRK><<<blocks, threads, 0, st>>>(a);
}

template <typename T, int SEL, int EPI>
static void launch(const HopArgs<T>& a, cudaStream_t st) {
  if (a.nsites <= 0) return;
  count_launch();
  if (a.Cr && a.kap)
    launch_v<T, SEL, EPI, true>(a, st);
  else
    launch_v<T, SEL, EPI, false>(a, st);
}

// merge one hop launch of each group member: 128-thread blocks (a thread's
// work does not depend on the CTA size), each member's sites in its own
// blocks; the FP16 block kernels keep their 64-register bound (the FP32
// block kernels and the full-lattice operators would spill under the bounds
// of their one-lattice forms, where the arguments sit in kernel parameters)
template <typename T, int SEL, int EPI>
static void merge_hop(const GroupRec* const* recs, int n, GroupBatch& b) {
  constexpr int threads = 128;
  std::vector<HopArgs<T>> args(n);
  std::vector<int> starts(n + 1);
  int blocks = 0;
  for (int l = 0; l < n; l++) {
    args[l] = group_arg<HopArgs<T>>(recs[l]);
    starts[l] = blocks;
    blocks += args[l].nsites > 0 ? (args[l].nsites + threads - 1) / threads : 0;
  }
  starts[n] = blocks;
  if (blocks == 0) return;
  const size_t oa = b.put(args.data(), sizeof(HopArgs<T>) * n), os = b.put_starts(starts);
  b.launches.push_back([=](const unsigned char* dev, cudaStream_t st) {
    count_launch();
    const auto* A = reinterpret_cast<const HopArgs<T>*>(dev + oa);
    const auto* S = reinterpret_cast<const int*>(dev + os);
    if constexpr (std::is_same<T, H16>::value && MinCtas<T, SEL>::value == 4)
      k_hop_multi_r64<T, SEL, EPI><<<blocks, threads, 0, st>>>(A, S, n);
    else
      k_hop_multi<T, SEL, EPI><<<blocks, threads, 0, st>>>(A, S, n);
  });
}

template <typename T>
void launch_hop(int sel, int epi, const HopArgs<T>& a, cudaStream_t st) {
  if (g_group_rec) {  // a group solve: one right-hand side, one kappa per lattice
    if (a.G.nr != 1 || (a.Cr && a.kap)) group_unrecorded_launch();
#define QWSG_CASE(S, E)                           \
  if (sel == S && epi == E) {                     \
    group_record(&merge_hop<T, S, E>, a);         \
    return;                                       \
  }
    QWSG_CASE(HOP_ALL, EPI_D)
    QWSG_CASE(HOP_INNER, EPI_D)
    QWSG_CASE(HOP_OUTER, EPI_ADD)
    QWSG_CASE(HOP_INNER, EPI_JINV)
    QWSG_CASE(HOP_INNER, EPI_SAPE)
#undef QWSG_CASE
  }
#define QWSG_CASE(S, E)              \
  if (sel == S && epi == E) {        \
    launch<T, S, E>(a, st);          \
    return;                          \
  }
  QWSG_CASE(HOP_ALL, EPI_D)
  QWSG_CASE(HOP_INNER, EPI_D)
  QWSG_CASE(HOP_OUTER, EPI_ADD)
  QWSG_CASE(HOP_INNER, EPI_JINV)
  QWSG_CASE(HOP_INNER, EPI_SAPE)
#undef QWSG_CASE
}

template void launch_hop<float>(int, int, const HopArgs<float>&, cudaStream_t);
template void launch_hop<double>(int, int, const HopArgs<double>&, cudaStream_t);
template void launch_hop<H16>(int, int, const HopArgs<H16>&, cudaStream_t);

}  // namespace qwsg
