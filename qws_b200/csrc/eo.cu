// Even-odd (site parity) hopping kernels: the deo_* family of the reference
// (deo_in_d.cc:65-445, deo_out_d.cc:88-286, deo_dag_in.cc, deo_dag_out.cc and
// the FP32 deo_in_s.cc / deo_out_s.cc) on the library's DD-order planes.
//
// Sites of parity pe = (x+y+z+t) % 2 receive the hops from the other parity:
//   WHICH  1 = hops inside the rank box (deo_in_*), 2 = hops across its faces
//          (deo_out_pre/pos_*), 3 = both;
//   DAG    the adjoint hopping H^dagger (projectors 1 + gamma_mu forward,
//          1 - gamma_mu backward, deo_dag_*);
//   CLOV   multiply by the parity's A^-1 (dee_*);
//   MODE   0 out = acc (__store_sc), 1 out += coef acc (__store_add_sc),
//          2 out = in0 + coef acc (one_minus_*).
// A y/z/t hop that leaves the rank box reads the other parity's site at the
// same compressed index x/2 of the wrapped row, as the reference's face
// packers do (deo_out_d.cc:88-153); this is the geometric neighbour when the
// wrapped extent is even.
#include "kernels.h"
#include "lattice.cuh"

namespace qwsg {

template <typename T, int WHICH, int DAG, int MU, int DIR, typename R = typename Arith<T>::R>
__device__ __forceinline__ void eo_hop(const EoArgs<T>& a, const int x[4], int g, R acc[24]) {
  const int L = a.G.L[MU], box = a.box[MU];
  const bool inner = DIR > 0 ? (x[MU] % box) != box - 1 : (x[MU] % box) != 0;
  if (inner ? !(WHICH & 1) : !(WHICH & 2)) return;
  int xn[4] = {x[0], x[1], x[2], x[3]};
  xn[MU] = DIR > 0 ? (x[MU] + 1 == L ? 0 : x[MU] + 1) : (x[MU] == 0 ? L - 1 : x[MU] - 1);
  if (!inner && MU > 0) {
    const int po = 1 - ((x[0] + x[1] + x[2] + x[3]) & 1);
    xn[0] = 2 * (x[0] >> 1) + ((po + xn[1] + xn[2] + xn[3]) & 1);
  }
  const int gn = dd_index(a.G, xn);
  constexpr int PD = DAG ? -DIR : DIR;  // projector / reconstruction of this hop
  R v[24];
  if (MU == 3)
    IO<T>::load_half(a.src, a.G.pad, gn, PD > 0, v);
  else
    IO<T>::load_spinor(a.src, a.G.pad, gn, v);
  R h[12], r[12], u[18];
  project<R, MU, PD>(v, h);
  IO<T>::load_link(a.U, a.G.pad, MU, DIR > 0 ? g : gn, u);
  if (DIR > 0)
    link_mul<R, false>(u, h, r);
  else
    link_mul<R, true>(u, h, r);
  R f = 1;
  if (MU == 3) {
    f = 2;
    if (DIR > 0 ? x[3] == L - 1 : x[3] == 0) f = (R)(2 * a.G.tbc);
  }
  reconstruct<R, MU, PD>(r, acc, f);
}

template <typename T, int WHICH, int DAG, int CLOV, int MODE>
__global__ void __launch_bounds__(128) k_eo(const EoArgs<T> a) {
  using R = typename Arith<T>::R;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.G.Vh) return;
  const int nxh = a.G.L[0] >> 1;
  int x[4];
  const int xh = i % nxh;
  int k = i / nxh;
  x[1] = k % a.G.L[1];
  k /= a.G.L[1];
  x[2] = k % a.G.L[2];
  x[3] = k / a.G.L[2];
  x[0] = 2 * xh + ((a.pe + x[1] + x[2] + x[3]) & 1);
  const int g = dd_index(a.G, x);
  R acc[24];
#pragma unroll
  for (int j = 0; j < 24; j++) acc[j] = 0;
  eo_hop<T, WHICH, DAG, 0, +1>(a, x, g, acc);
  eo_hop<T, WHICH, DAG, 0, -1>(a, x, g, acc);
  eo_hop<T, WHICH, DAG, 1, +1>(a, x, g, acc);
  eo_hop<T, WHICH, DAG, 1, -1>(a, x, g, acc);
  eo_hop<T, WHICH, DAG, 2, +1>(a, x, g, acc);
  eo_hop<T, WHICH, DAG, 2, -1>(a, x, g, acc);
  eo_hop<T, WHICH, DAG, 3, +1>(a, x, g, acc);
  eo_hop<T, WHICH, DAG, 3, -1>(a, x, g, acc);
  if (CLOV) clover_apply<T>(a.C, a.G.pad, g, acc);
  R o[24];
  if (MODE == 0) {
#pragma unroll
    for (int j = 0; j < 24; j++) o[j] = acc[j];
  } else if (MODE == 1) {
    IO<T>::load_spinor(a.out, a.G.pad, g, o);
#pragma unroll
    for (int j = 0; j < 24; j++) o[j] = o[j] + acc[j] * a.coef;
  } else {
    IO<T>::load_spinor(a.in0, a.G.pad, g, o);
#pragma unroll
    for (int j = 0; j < 24; j++) o[j] = o[j] + acc[j] * a.coef;
  }
  IO<T>::store_spinor(a.out, a.G.pad, g, o);
}

// parity-pe clover multiplication (clvd_vm_/clv_s_, qws.cc:390-425)
template <typename T>
__global__ void k_clv(const EoArgs<T> a) {
  using R = typename Arith<T>::R;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.G.Vh) return;
  const int nxh = a.G.L[0] >> 1;
  int x[4];
  const int xh = i % nxh;
  int k = i / nxh;
  x[1] = k % a.G.L[1];
  k /= a.G.L[1];
  x[2] = k % a.G.L[2];
  x[3] = k / a.G.L[2];
  x[0] = 2 * xh + ((a.pe + x[1] + x[2] + x[3]) & 1);
  const int g = dd_index(a.G, x);
  R v[24];
  IO<T>::load_spinor(a.src, a.G.pad, g, v);
  clover_apply<T>(a.C, a.G.pad, g, v);
  IO<T>::store_spinor(a.out, a.G.pad, g, v);
}

template <typename T>
__global__ void k_parity_select(Geom G, typename Store<T>::type* dst,
                                const typename Store<T>::type* __restrict__ src, int pe) {
  using R = typename Arith<T>::R;
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  Site s;
  decode_site(G, g, s);
  int par = 0;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) par += s.bc[mu] * G.B[mu] + s.lc[mu];
  R v[24];
  if ((par & 1) == pe) {
    IO<T>::load_spinor(src, G.pad, g, v);
  } else {
#pragma unroll
    for (int j = 0; j < 24; j++) v[j] = 0;
  }
  IO<T>::store_spinor(dst, G.pad, g, v);
}

template <typename T>
void parity_select(const Geom& G, typename Store<T>::type* dst, const typename Store<T>::type* src,
                   int pe, cudaStream_t st) {
  count_launch();
  k_parity_select<T><<<(G.V + 127) / 128, 128, 0, st>>>(G, dst, src, pe);
}
template void parity_select<float>(const Geom&, float*, const float*, int, cudaStream_t);
template void parity_select<double>(const Geom&, double*, const double*, int, cudaStream_t);

template <typename T, int WHICH, int DAG, int CLOV, int MODE>
static void go(const EoArgs<T>& a, cudaStream_t st) {
  count_launch();
  k_eo<T, WHICH, DAG, CLOV, MODE><<<(a.G.Vh + 127) / 128, 128, 0, st>>>(a);
}

template <typename T>
void launch_eo(int which, int dag, int clov, int mode, const EoArgs<T>& a, cudaStream_t st) {
  // every combination the reference uses (12 FP64, 5 FP32 entry points)
#define QWSG_EO(W, D, C, M)                                    \
  if (which == W && dag == D && clov == C && mode == M) {      \
    go<T, W, D, C, M>(a, st);                                  \
    return;                                                    \
  }
  QWSG_EO(1, 0, 0, 0) QWSG_EO(1, 0, 1, 0) QWSG_EO(1, 1, 0, 0) QWSG_EO(1, 1, 1, 0)
  QWSG_EO(1, 0, 1, 2) QWSG_EO(1, 1, 0, 2)
  QWSG_EO(2, 0, 0, 1) QWSG_EO(2, 1, 0, 1) QWSG_EO(2, 0, 1, 1) QWSG_EO(2, 1, 1, 1)
  QWSG_EO(3, 0, 0, 0) QWSG_EO(3, 0, 1, 0) QWSG_EO(3, 1, 0, 0) QWSG_EO(3, 1, 1, 0)
  QWSG_EO(3, 0, 1, 2) QWSG_EO(3, 1, 0, 2) QWSG_EO(3, 0, 0, 1) QWSG_EO(3, 0, 1, 1)
#undef QWSG_EO
  throw_unsupported_eo();
}

template <typename T>
void launch_clv(const EoArgs<T>& a, cudaStream_t st) {
  count_launch();
  k_clv<T><<<(a.G.Vh + 127) / 128, 128, 0, st>>>(a);
}

template void launch_eo<float>(int, int, int, int, const EoArgs<float>&, cudaStream_t);
template void launch_eo<double>(int, int, int, int, const EoArgs<double>&, cudaStream_t);
template void launch_clv<float>(const EoArgs<float>&, cudaStream_t);
template void launch_clv<double>(const EoArgs<double>&, cudaStream_t);

}  // namespace qwsg
