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

template <typename T, int SEL, int MU, int DIR, typename R = typename Arith<T>::R>
__device__ __forceinline__ void do_hop(const HopArgs<T>& a, const Site& s, int g, int rhs,
                                       R acc[24]) {
  const bool face = DIR > 0 ? (s.lc[MU] == a.G.B[MU] - 1) : (s.lc[MU] == 0);
  if (face) {
    if (!(SEL & HOP_OUTER)) return;
  } else {
    if (!(SEL & HOP_INNER)) return;
  }
  int gn;
  if (!face) {
    gn = g + DIR * a.G.str[MU];
  } else {
    int ncol;
    gn = nbr_across(a.G, s, MU, DIR, &ncol);
    if (ncol == a.zero_col) return;  // that colour's source is defined as zero
  }
  R v[24], sc;
  const int sp = spad(a.G), en = sentry(a.G, gn, rhs);
  // the projection and the link product are linear: the source's scale
  // (FP16 storage) is applied once, in the reconstruction
  if (MU == 3)
    IO<T>::load_half_raw(a.src, sp, en, DIR > 0, v, sc);
  else
    IO<T>::load_spinor_raw(a.src, sp, en, v, sc);
  R h[12], r[12], u[18];
  project<R, MU, DIR>(v, h);
  if constexpr (std::is_same<T, float>::value) {
    if (a.U12)
      load_link12(a.U12, a.G.pad, MU, DIR > 0 ? g : gn, u);
    else
      IO<T>::load_link(a.U, a.G.pad, MU, DIR > 0 ? g : gn, u);
  } else {
    IO<T>::load_link(a.U, a.G.pad, MU, DIR > 0 ? g : gn, u);
  }
  if (DIR > 0)
    link_mul<R, false>(u, h, r);
  else
    link_mul<R, true>(u, h, r);
  R f = sc;
  if (MU == 3) {
    f = 2 * sc;
    if (face && (DIR > 0 ? s.bc[3] == a.G.NB[3] - 1 : s.bc[3] == 0)) f = (R)(2 * a.G.tbc) * sc;
  }
  reconstruct<R, MU, DIR>(r, acc, f);
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

template <typename T, int SEL, int EPI>
__global__ void __launch_bounds__(256, (MinCtas<T, SEL>::value)) k_hop(const HopArgs<T> a) {
  using R = typename Arith<T>::R;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (a.nsites << a.G.lgnr)) return;
  // consecutive threads: the right-hand sides of one site, then the next site
  const int si = i >> a.G.lgnr, rhs = i & (a.G.nr - 1);
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
  R acc[24];
#pragma unroll
  for (int j = 0; j < 24; j++) acc[j] = 0;
  do_hop<T, SEL, 0, +1>(a, s, g, rhs, acc);
  do_hop<T, SEL, 0, -1>(a, s, g, rhs, acc);
  do_hop<T, SEL, 1, +1>(a, s, g, rhs, acc);
  do_hop<T, SEL, 1, -1>(a, s, g, rhs, acc);
  do_hop<T, SEL, 2, +1>(a, s, g, rhs, acc);
  do_hop<T, SEL, 2, -1>(a, s, g, rhs, acc);
  do_hop<T, SEL, 3, +1>(a, s, g, rhs, acc);
  do_hop<T, SEL, 3, -1>(a, s, g, rhs, acc);
  clover_apply<T>(a.C, a.G.pad, g, acc);
  const int sp = spad(a.G), e = sentry(a.G, g, rhs);
  R o[24];
  if (EPI == EPI_D) {
    IO<T>::load_spinor(a.src, sp, e, o);
#pragma unroll
    for (int j = 0; j < 24; j++) o[j] = o[j] + a.coef * acc[j];
  } else if (EPI == EPI_ADD) {
    IO<T>::load_spinor(a.out, sp, e, o);
#pragma unroll
    for (int j = 0; j < 24; j++) o[j] = o[j] + a.coef * acc[j];
  } else if (EPI == EPI_JINV) {
    IO<T>::load_spinor(a.aux, sp, e, o);
#pragma unroll
    for (int j = 0; j < 24; j++) o[j] = o[j] + a.coef * acc[j];
  } else {  // EPI_SAPE: coef = -kappa
    R in[24], av[24];
    IO<T>::load_spinor(a.out, sp, e, o);
    IO<T>::load_spinor(a.aux, sp, e, in);
    IO<T>::load_spinor(a.src, sp, e, av);
#pragma unroll
    for (int j = 0; j < 24; j++) o[j] = o[j] + (in[j] - (av[j] + a.coef * acc[j]));
  }
  IO<T>::store_spinor(a.out, sp, e, o);
}

template <typename T, int SEL, int EPI>
static void launch(const HopArgs<T>& a, cudaStream_t st) {
  if (a.nsites <= 0) return;
  const int threads = a.G.hop_threads;
  const int blocks = ((a.nsites << a.G.lgnr) + threads - 1) / threads;
  count_launch();
  k_hop<T, SEL, EPI><<<blocks, threads, 0, st>>>(a);
}

template <typename T>
void launch_hop(int sel, int epi, const HopArgs<T>& a, cudaStream_t st) {
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
