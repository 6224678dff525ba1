// BQCD-format fields and spinors converted on the device.
//
// The reference's loaders (qws_bqcd.cc:66-642) reorder BQCD's arrays into
// QWS's host layout with host loops.  Here the raw BQCD array is copied to
// the device as it is and one kernel writes the library's planes: one
// thread per site (DD order) gathers its links / clover / spinor from the
// site's BQCD slot.
//
// BQCD numbering: site (x,y,z,t) of parity eo has index i (1-based within
// its parity, the host program's std_xyzt2i_/e_o_, qws_bqcd.cc:56-57); its
// slot is (i-1) + volh*eo, and
//   links   u[ri + 2*row + 6*col + 18*slot + 18*V*mu]   (column-major SU(3))
//   clover  c[perm[k] + 36*ud + 72*slot]                (two chiral blocks)
//   spinor  even/odd arrays, element 2*s + 8*c + ri + 24*(i-1)
// A caller-supplied site map gives each natural site's slot; without one,
// i - 1 = (lexicographic index) / 2, this library's default numbering.
#include "kernels.h"
#include "lattice.cuh"

namespace qwsg {

namespace {

// BQCD's 36 reals of one chiral block -> QWS packing (qws_bqcd.cc:301-377):
// QWS element k of a block is BQCD element kPerm[k]
__constant__ int kPerm[36] = {0,  1,  20, 21, 32, 33, 2,  3,  4,  5,  6,  7,
                              8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 19,
                              22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 34, 35};

__device__ __forceinline__ long slot_of(const Geom& G, const int* __restrict__ map, int g) {
  Site s;
  decode_site(G, g, s);
  int x[4];
#pragma unroll
  for (int mu = 0; mu < 4; mu++) x[mu] = s.bc[mu] * G.B[mu] + s.lc[mu];
  const long n = x[0] + (long)G.L[0] * (x[1] + (long)G.L[1] * (x[2] + (long)G.L[2] * x[3]));
  if (map) return __ldg(map + n);
  return n / 2 + (long)(G.V / 2) * ((x[0] + x[1] + x[2] + x[3]) & 1);
}

template <typename R>
__global__ void k_bqcd2pl_gauge(Geom G, R* dst, const double* __restrict__ u,
                                const int* __restrict__ map) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  const long slot = slot_of(G, map, g);
  for (int mu = 0; mu < 4; mu++) {
    const double* p = u + 18 * (slot + (long)mu * G.V);
    R v[18];
#pragma unroll
    for (int row = 0; row < 3; row++)
#pragma unroll
      for (int col = 0; col < 3; col++) {
        v[6 * row + 2 * col] = (R)p[2 * row + 6 * col];
        v[6 * row + 2 * col + 1] = (R)p[2 * row + 6 * col + 1];
      }
    store_link<R>(dst, G.pad, mu, g, v);
  }
}

template <typename R>
__global__ void k_bqcd2pl_clover(Geom G, R* dst, const double* __restrict__ c,
                                 const int* __restrict__ map) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  const double* p = c + 72 * slot_of(G, map, g);
  R a[72];
#pragma unroll
  for (int ud = 0; ud < 2; ud++)
#pragma unroll
    for (int k = 0; k < 36; k++) a[36 * ud + k] = (R)p[36 * ud + kPerm[k]];
  store_clover<R>(dst, G.pad, g, a);
}

// spinors: `both` = the even array followed by the odd one (V*24 reals)
template <typename R>
__global__ void k_bqcd2pl_spinor(Geom G, R* dst, const double* __restrict__ both,
                                 const int* __restrict__ map, int rhs) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  const double* p = both + 24 * slot_of(G, map, g);
  R v[24];
#pragma unroll
  for (int j = 0; j < 24; j++) v[j] = (R)p[j];
  IO<R>::store_spinor(dst, spad(G), sentry(G, g, rhs), v);
}

template <typename R>
__global__ void k_pl2bqcd_spinor(Geom G, double* both, const R* __restrict__ src,
                                 const int* __restrict__ map, int rhs) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  double* p = both + 24 * slot_of(G, map, g);
  R v[24];
  IO<R>::load_spinor(src, spad(G), sentry(G, g, rhs), v);
#pragma unroll
  for (int j = 0; j < 24; j++) p[j] = (double)v[j];
}

inline int nblk(int n) { return (n + 127) / 128; }

}  // namespace

template <typename R>
void bqcd_to_planes_gauge(const Geom& G, R* dst, const double* u, const int* map,
                          cudaStream_t st) {
  count_launch();
  k_bqcd2pl_gauge<R><<<nblk(G.V), 128, 0, st>>>(G, dst, u, map);
}
template <typename R>
void bqcd_to_planes_clover(const Geom& G, R* dst, const double* c, const int* map,
                           cudaStream_t st) {
  count_launch();
  k_bqcd2pl_clover<R><<<nblk(G.V), 128, 0, st>>>(G, dst, c, map);
}
template <typename R>
void bqcd_to_planes_spinor(const Geom& G, R* dst, const double* both, const int* map, int rhs,
                           cudaStream_t st) {
  count_launch();
  k_bqcd2pl_spinor<R><<<nblk(G.V), 128, 0, st>>>(G, dst, both, map, rhs);
}
template <typename R>
void planes_to_bqcd_spinor(const Geom& G, double* both, const R* src, const int* map, int rhs,
                           cudaStream_t st) {
  count_launch();
  k_pl2bqcd_spinor<R><<<nblk(G.V), 128, 0, st>>>(G, both, src, map, rhs);
}

#define QWSG_INST(R)                                                                           \
  template void bqcd_to_planes_gauge<R>(const Geom&, R*, const double*, const int*,            \
                                        cudaStream_t);                                         \
  template void bqcd_to_planes_clover<R>(const Geom&, R*, const double*, const int*,           \
                                         cudaStream_t);                                        \
  template void bqcd_to_planes_spinor<R>(const Geom&, R*, const double*, const int*, int,      \
                                         cudaStream_t);                                        \
  template void planes_to_bqcd_spinor<R>(const Geom&, double*, const R*, const int*, int,      \
                                         cudaStream_t);
QWSG_INST(float)
QWSG_INST(double)
#undef QWSG_INST

}  // namespace qwsg
