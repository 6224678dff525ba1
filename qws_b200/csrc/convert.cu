// Layout converters between host formats and the device planes.
//
// QWS host layout (qws.h:111-192; main.cc:426-429; reordering.cc:59-105):
// the (single-rank) lattice is split into two x-halves ("domains") of
// nxh = Lx/2 sites; inside a domain sites are vectors of `vlen` consecutive x
// sites (SIMD lanes):
//   elem  = dom*vol + xv + nxv*(y + Ly*(z + Lz*t)),  nxv = nxh/vlen
//   spinor real r (0..23, order [colour][spin][re,im]) at (elem*24 + r)*vlen + lane
//   link   (dom*4 + mu)*vol + ...; U[row][col] stored column-major c[col][row]:
//          ((elem*18) + (col*3 + row)*2 + ri)*vlen + lane
//   clover real j (0..71) at (elem*72 + j)*vlen + lane
// Natural layout: site n = x + Lx*(y + Ly*(z + Lz*t)); spinor [n][24],
// gauge [mu][n][row][col][2], clover [n][72].
// Every converter runs one thread per device site and is a pure gather/scatter.
#include "kernels.h"

namespace qwsg {

namespace {

struct QwsIdx {
  long elem_sp;  // spinor / clover element
  long elem_g0;  // link element for mu = 0 (add mu*vol)
  long vol;
  int lane;
};

__device__ __forceinline__ void global_coords(const Geom& G, int g, int x[4]) {
  Site s;
  decode_site(G, g, s);
#pragma unroll
  for (int mu = 0; mu < 4; mu++) x[mu] = s.bc[mu] * G.B[mu] + s.lc[mu];
}

__device__ __forceinline__ QwsIdx qws_index(const Geom& G, const int x[4], int vlen) {
  int nxh = G.L[0] / 2, nxv = nxh / vlen;
  int dom = x[0] / nxh, xh = x[0] - dom * nxh;
  long vol = (long)nxv * G.L[1] * G.L[2] * G.L[3];
  long in_dom = xh / vlen + (long)nxv * (x[1] + (long)G.L[1] * (x[2] + (long)G.L[2] * x[3]));
  QwsIdx q;
  q.elem_sp = dom * vol + in_dom;
  q.elem_g0 = dom * 4 * vol + in_dom;
  q.vol = vol;
  q.lane = xh % vlen;
  return q;
}

// Even-odd reading of the same host arrays (qws_bqcd.cc:66-85; deo_in_d.cc:65-86):
// the site (x,y,z,t) of parity p = (x+y+z+t)%2 sits in the x-half slot p at
// compressed x index x/2.  Maps x[0] to that slot's x so qws_index applies.
__device__ __forceinline__ void eo_slot(const Geom& G, int x[4]) {
  const int p = (x[0] + x[1] + x[2] + x[3]) & 1;
  x[0] = p * (G.L[0] / 2) + x[0] / 2;
}

__device__ __forceinline__ long nat_index(const Geom& G, const int x[4]) {
  return x[0] + (long)G.L[0] * (x[1] + (long)G.L[1] * (x[2] + (long)G.L[2] * x[3]));
}

template <typename R>
__device__ __forceinline__ void store_sp(R* p, int pad, int g, const R v[24]) {
  IO<R>::store_spinor(p, pad, g, v);
}

template <typename R>
__global__ void k_qws2pl_sp(Geom G, R* dst, const R* __restrict__ q, int vlen, int site0, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int g = site0 + i, x[4];
  global_coords(G, g, x);
  QwsIdx Q = qws_index(G, x, vlen);
  R v[24];
#pragma unroll
  for (int r = 0; r < 24; r++) v[r] = q[(Q.elem_sp * 24 + r) * vlen + Q.lane];
  store_sp(dst, G.pad, g, v);
}

template <typename R>
__global__ void k_pl2qws_sp(Geom G, R* q, const R* __restrict__ src, int vlen, int site0, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int g = site0 + i, x[4];
  global_coords(G, g, x);
  QwsIdx Q = qws_index(G, x, vlen);
  R v[24];
  IO<R>::load_spinor(src, G.pad, g, v);
#pragma unroll
  for (int r = 0; r < 24; r++) q[(Q.elem_sp * 24 + r) * vlen + Q.lane] = v[r];
}

// Half array of one parity p in the even-odd layout (vol elements, the
// compressed index x/2) -> full planes, zero on the other parity.
template <typename R>
__global__ void k_qwseo2pl_sp(Geom G, R* dst, const R* __restrict__ q, int vlen, int p) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  int x[4];
  global_coords(G, g, x);
  R v[24];
  if (((x[0] + x[1] + x[2] + x[3]) & 1) == p) {
    x[0] /= 2;  // slot 0 of a half array
    QwsIdx Q = qws_index(G, x, vlen);
#pragma unroll
    for (int r = 0; r < 24; r++) v[r] = q[(Q.elem_sp * 24 + r) * vlen + Q.lane];
  } else {
#pragma unroll
    for (int r = 0; r < 24; r++) v[r] = 0;
  }
  store_sp(dst, G.pad, g, v);
}

template <typename R>
__global__ void k_pl2qwseo_sp(Geom G, R* q, const R* __restrict__ src, int vlen, int p) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  int x[4];
  global_coords(G, g, x);
  if (((x[0] + x[1] + x[2] + x[3]) & 1) != p) return;
  x[0] /= 2;
  QwsIdx Q = qws_index(G, x, vlen);
  R v[24];
  IO<R>::load_spinor(src, G.pad, g, v);
#pragma unroll
  for (int r = 0; r < 24; r++) q[(Q.elem_sp * 24 + r) * vlen + Q.lane] = v[r];
}

template <typename R>
__global__ void k_qws2pl_gauge(Geom G, R* dst, const R* __restrict__ q, int vlen, int eo) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  int x[4];
  global_coords(G, g, x);
  if (eo) eo_slot(G, x);
  QwsIdx Q = qws_index(G, x, vlen);
  for (int mu = 0; mu < 4; mu++) {
    long elem = Q.elem_g0 + mu * Q.vol;
    R u[18];
#pragma unroll
    for (int row = 0; row < 3; row++)
#pragma unroll
      for (int col = 0; col < 3; col++)
#pragma unroll
        for (int ri = 0; ri < 2; ri++)
          u[2 * (3 * row + col) + ri] = q[(elem * 18 + (col * 3 + row) * 2 + ri) * vlen + Q.lane];
    store_link<R>(dst, G.pad, mu, g, u);
  }
}

template <typename R>
__global__ void k_qws2pl_clover(Geom G, R* dst, const R* __restrict__ q, int vlen, int eo) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  int x[4];
  global_coords(G, g, x);
  if (eo) eo_slot(G, x);
  QwsIdx Q = qws_index(G, x, vlen);
  R a[72];
#pragma unroll
  for (int j = 0; j < 72; j++) a[j] = q[(Q.elem_sp * 72 + j) * vlen + Q.lane];
  store_clover<R>(dst, G.pad, g, a);
}

template <typename R>
__global__ void k_nat2pl_sp(Geom G, R* dst, const R* __restrict__ nat, int rhs) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  int x[4];
  global_coords(G, g, x);
  long n = nat_index(G, x);
  R v[24];
#pragma unroll
  for (int r = 0; r < 24; r++) v[r] = nat[n * 24 + r];
  store_sp(dst, spad(G), sentry(G, g, rhs), v);
}

template <typename R>
__global__ void k_pl2nat_sp(Geom G, R* nat, const R* __restrict__ src, int rhs) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  int x[4];
  global_coords(G, g, x);
  long n = nat_index(G, x);
  R v[24];
  IO<R>::load_spinor(src, spad(G), sentry(G, g, rhs), v);
#pragma unroll
  for (int r = 0; r < 24; r++) nat[n * 24 + r] = v[r];
}

template <typename Rin, typename R>
__global__ void k_nat2pl_gauge(Geom G, R* dst, const Rin* __restrict__ nat) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  int x[4];
  global_coords(G, g, x);
  long n = nat_index(G, x);
  for (int mu = 0; mu < 4; mu++) {
    R u[18];
#pragma unroll
    for (int e = 0; e < 18; e++) u[e] = (R)nat[((long)mu * G.V + n) * 18 + e];
    store_link<R>(dst, G.pad, mu, g, u);
  }
}

template <typename Rin, typename R>
__global__ void k_nat2pl_clover(Geom G, R* dst, const Rin* __restrict__ nat) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  int x[4];
  global_coords(G, g, x);
  long n = nat_index(G, x);
  R a[72];
#pragma unroll
  for (int j = 0; j < 72; j++) a[j] = (R)nat[n * 72 + j];
  store_clover<R>(dst, G.pad, g, a);
}

inline int nb(long n) { return (int)((n + 127) / 128); }

// spinor precision conversions: one thread per (site, rhs) entry
enum { CONV_S2H = 0, CONV_H2S = 1, CONV_H2H = 2 };
template <int K>
__device__ __forceinline__ void conv_entry(const Geom& G, void* dst, const void* src, int e) {
  if (e >= (G.V << G.lgnr)) return;
  const int sp = spad(G);
  if (K == CONV_S2H) {
    float v[24];
    IO<float>::load_spinor(static_cast<const float*>(src), sp, e, v);
    IO<H16>::store_spinor(static_cast<__half*>(dst), sp, e, v);
  } else if (K == CONV_H2S) {
    float v[24];
    IO<H16>::load_spinor(static_cast<const __half*>(src), sp, e, v);
    IO<float>::store_spinor(static_cast<float*>(dst), sp, e, v);
  } else {
    // the IO<H16> spinor layout: three 16-byte planes, then the scale plane
    const size_t p = sp;
    const uint4* s = static_cast<const uint4*>(src);
    uint4* d = static_cast<uint4*>(dst);
#pragma unroll
    for (int j = 0; j < 3; j++) d[j * p + e] = s[j * p + e];
    reinterpret_cast<float*>(d + 3 * p)[e] = reinterpret_cast<const float*>(s + 3 * p)[e];
  }
}
__global__ void k_s2h(Geom G, __half* dst, const float* __restrict__ src) {
  conv_entry<CONV_S2H>(G, dst, src, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void k_h2s(Geom G, float* dst, const __half* __restrict__ src) {
  conv_entry<CONV_H2S>(G, dst, src, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void k_h2h(Geom G, __half* dst, const __half* __restrict__ src) {
  conv_entry<CONV_H2H>(G, dst, src, blockIdx.x * blockDim.x + threadIdx.x);
}

// the same conversions for several lattices in one launch (group solves;
// one RHS each)
struct ConvArgs {
  Geom G;
  void* dst;
  const void* src;
};
template <int K>
__global__ void k_conv_multi(const ConvArgs* __restrict__ args, const int* __restrict__ starts,
                             int n) {
  __shared__ ConvArgs sa;
  const int l = group_member(starts, n, blockIdx.x);
  group_load_args(sa, args + l);
  conv_entry<K>(sa.G, sa.dst, sa.src, (blockIdx.x - starts[l]) * blockDim.x + threadIdx.x);
}
template <int K>
void merge_conv(const GroupRec* const* recs, int n, GroupBatch& b) {
  std::vector<ConvArgs> args(n);
  std::vector<int> starts(n + 1);
  int blocks = 0;
  for (int l = 0; l < n; l++) {
    args[l] = group_arg<ConvArgs>(recs[l]);
    starts[l] = blocks;
    blocks += (args[l].G.V + 127) / 128;
  }
  starts[n] = blocks;
  const size_t oa = b.put(args.data(), sizeof(ConvArgs) * n), os = b.put_starts(starts);
  b.launches.push_back([=](const unsigned char* dev, cudaStream_t st) {
    count_launch();
    k_conv_multi<K><<<blocks, 128, 0, st>>>(reinterpret_cast<const ConvArgs*>(dev + oa),
                                            reinterpret_cast<const int*>(dev + os), n);
  });
}
template <int K>
bool record_conv(const Geom& G, void* dst, const void* src) {
  if (!g_group_rec) return false;
  if (G.nr != 1) group_unrecorded_launch();
  return group_record(&merge_conv<K>, ConvArgs{G, dst, src});
}

// the same three conversions for FP16 fields of two or more RHS (IOP
// layout): one thread per (site, RHS pair)
__global__ void k_s2h_pair(Geom G, __half* dst, const float* __restrict__ src) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (G.V << (G.lgnr - 1))) return;
  const int sp = spad(G);
  float a[24], b[24];
  IO<float>::load_spinor(src, sp, 2 * e, a);
  IO<float>::load_spinor(src, sp, 2 * e + 1, b);
  F2 v[24];
#pragma unroll
  for (int j = 0; j < 24; j++) v[j] = F2{a[j], b[j]};
  IOP::store_spinor(dst, sp >> 1, e, v);
}
__global__ void k_h2s_pair(Geom G, float* dst, const __half* __restrict__ src) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (G.V << (G.lgnr - 1))) return;
  const int sp = spad(G);
  F2 v[24];
  IOP::load_spinor(src, sp >> 1, e, v);
  float a[24], b[24];
#pragma unroll
  for (int j = 0; j < 24; j++) {
    a[j] = v[j].x;
    b[j] = v[j].y;
  }
  IO<float>::store_spinor(dst, sp, 2 * e, a);
  IO<float>::store_spinor(dst, sp, 2 * e + 1, b);
}
__global__ void k_h2h_pair(Geom G, __half* dst, const __half* __restrict__ src) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (G.V << (G.lgnr - 1))) return;
  const size_t pp = spad(G) >> 1;
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4* d = reinterpret_cast<uint4*>(dst);
#pragma unroll
  for (int j = 0; j < 6; j++) d[j * pp + e] = s[j * pp + e];
  reinterpret_cast<float2*>(d + 6 * pp)[e] = reinterpret_cast<const float2*>(s + 6 * pp)[e];
}

// FP16 copy of per-RHS clover planes (entry (g << lgnr) + r, stride spad)
__global__ void k_clover_s2h_entries(Geom G, __half* Ch, const float* __restrict__ Cs) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (G.V << G.lgnr)) return;
  const int sp = spad(G);
  float a[72];
  IO<float>::load_clover_block(Cs, sp, e, 0, a);
  IO<float>::load_clover_block(Cs, sp, e, 1, a + 36);
  IO<H16>::store_clover(Ch, sp, e, a);
}

__global__ void k_fields_s2h(Geom G, __half* Uh, const float* __restrict__ Us, __half* Ch,
                             const float* __restrict__ Cs) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  for (int mu = 0; mu < 4; mu++) {
    float u[18];
    IO<float>::load_link(Us, G.pad, mu, g, u);
    IO<H16>::store_link(Uh, G.pad, mu, g, u);
  }
  const float4* c = reinterpret_cast<const float4*>(Cs);
  float a[72];
#pragma unroll
  for (int j = 0; j < 18; j++) {
    const float4 t = c[(size_t)j * G.pad + g];
    a[4 * j] = t.x;
    a[4 * j + 1] = t.y;
    a[4 * j + 2] = t.z;
    a[4 * j + 3] = t.w;
  }
  IO<H16>::store_clover(Ch, G.pad, g, a);
}

// largest deviation from SU(3) of the FP32 link of one (site, direction)
__global__ void k_su3_dev(Geom G, const float* __restrict__ Us, unsigned* dev) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  float worst = 0;
  if (g < G.V) {
    for (int mu = 0; mu < 4; mu++) {
      float u[18];
      IO<float>::load_link(Us, G.pad, mu, g, u);
      double d = 0;
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {  // (U U^+)_ab - delta_ab
          double re = 0, im = 0;
          for (int k = 0; k < 3; k++) {
            const double xr = u[2 * (3 * a + k)], xi = u[2 * (3 * a + k) + 1];
            const double yr = u[2 * (3 * b + k)], yi = -u[2 * (3 * b + k) + 1];
            re += xr * yr - xi * yi;
            im += xr * yi + xi * yr;
          }
          d = fmax(d, fabs(re - (a == b)) + fabs(im));
        }
      // det U by the first row's cofactors
      double dr = 0, di = 0;
      for (int b = 0; b < 3; b++) {
        const int b1 = (b + 1) % 3, b2 = (b + 2) % 3;
        const double pr = (double)u[6 + 2 * b1] * u[12 + 2 * b2] - (double)u[7 + 2 * b1] * u[13 + 2 * b2] -
                          ((double)u[6 + 2 * b2] * u[12 + 2 * b1] - (double)u[7 + 2 * b2] * u[13 + 2 * b1]);
        const double pi = (double)u[6 + 2 * b1] * u[13 + 2 * b2] + (double)u[7 + 2 * b1] * u[12 + 2 * b2] -
                          ((double)u[6 + 2 * b2] * u[13 + 2 * b1] + (double)u[7 + 2 * b2] * u[12 + 2 * b1]);
        dr += u[2 * b] * pr - u[2 * b + 1] * pi;
        di += u[2 * b] * pi + u[2 * b + 1] * pr;
      }
      d = fmax(d, fabs(dr - 1) + fabs(di));
      worst = fmaxf(worst, isfinite(d) ? (float)d : 3.0e38f);
    }
  }
  // non-negative floats order like their bit patterns
  for (int o = 16; o > 0; o >>= 1) worst = fmaxf(worst, __shfl_xor_sync(0xffffffffu, worst, o));
  if ((threadIdx.x & 31) == 0) atomicMax(dev, __float_as_uint(worst));
}

__global__ void k_compress12(Geom G, float* __restrict__ U12, const float* __restrict__ Us) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  float4* q = reinterpret_cast<float4*>(U12);
  for (int mu = 0; mu < 4; mu++) {
    float u[18];
    IO<float>::load_link(Us, G.pad, mu, g, u);
#pragma unroll
    for (int k = 0; k < 3; k++)
      q[(size_t)(3 * mu + k) * G.pad + g] = make_float4(u[4 * k], u[4 * k + 1], u[4 * k + 2], u[4 * k + 3]);
  }
}

}  // namespace

void links_su3_deviation(const Geom& G, const float* Us, unsigned* dev, cudaStream_t st) {
  count_launch();
  k_su3_dev<<<nb(G.V), 128, 0, st>>>(G, Us, dev);
}
void links_compress12(const Geom& G, float* U12, const float* Us, cudaStream_t st) {
  count_launch();
  k_compress12<<<nb(G.V), 128, 0, st>>>(G, U12, Us);
}

// FP16 spinors of one RHS use IO<H16>, of two or more the IOP layout of the
// paired hop kernels
void spinor_s2h(const Geom& G, __half* dst, const float* src, cudaStream_t st) {
  if (record_conv<CONV_S2H>(G, dst, src)) return;
  count_launch();
  if (G.nr >= 2)
    k_s2h_pair<<<nb(G.V << (G.lgnr - 1)), 128, 0, st>>>(G, dst, src);
  else
    k_s2h<<<nb(G.V), 128, 0, st>>>(G, dst, src);
}
void spinor_h2s(const Geom& G, float* dst, const __half* src, cudaStream_t st) {
  if (record_conv<CONV_H2S>(G, dst, src)) return;
  count_launch();
  if (G.nr >= 2)
    k_h2s_pair<<<nb(G.V << (G.lgnr - 1)), 128, 0, st>>>(G, dst, src);
  else
    k_h2s<<<nb(G.V), 128, 0, st>>>(G, dst, src);
}
void spinor_h2h(const Geom& G, __half* dst, const __half* src, cudaStream_t st) {
  if (record_conv<CONV_H2H>(G, dst, src)) return;
  count_launch();
  if (G.nr >= 2)
    k_h2h_pair<<<nb(G.V << (G.lgnr - 1)), 128, 0, st>>>(G, dst, src);
  else
    k_h2h<<<nb(G.V), 128, 0, st>>>(G, dst, src);
}
void clover_s2h_entries(const Geom& G, __half* Ch, const float* Cs, cudaStream_t st) {
  count_launch();
  k_clover_s2h_entries<<<nb(G.V << G.lgnr), 128, 0, st>>>(G, Ch, Cs);
}
void fields_s2h(const Geom& G, __half* Uh, const float* Us, __half* Ch, const float* Cs,
                cudaStream_t st) {
  count_launch();
  k_fields_s2h<<<nb(G.V), 128, 0, st>>>(G, Uh, Us, Ch, Cs);
}

template <typename R>
void qws_to_planes_spinor(const Geom& G, R* dst, const R* qws, int vlen, int site0, int n,
                          cudaStream_t st) {
  if (n > 0) {
    count_launch();
    k_qws2pl_sp<R><<<nb(n), 128, 0, st>>>(G, dst, qws, vlen, site0, n);
  }
}
template <typename R>
void planes_to_qws_spinor(const Geom& G, R* qws, const R* src, int vlen, int site0, int n,
                          cudaStream_t st) {
  if (n > 0) {
    count_launch();
    k_pl2qws_sp<R><<<nb(n), 128, 0, st>>>(G, qws, src, vlen, site0, n);
  }
}
template <typename R>
void qws_eo_to_planes_spinor(const Geom& G, R* dst, const R* qws_half, int vlen, int p,
                             cudaStream_t st) {
  count_launch();
  k_qwseo2pl_sp<R><<<nb(G.V), 128, 0, st>>>(G, dst, qws_half, vlen, p);
}
template <typename R>
void planes_to_qws_eo_spinor(const Geom& G, R* qws_half, const R* src, int vlen, int p,
                             cudaStream_t st) {
  count_launch();
  k_pl2qwseo_sp<R><<<nb(G.V), 128, 0, st>>>(G, qws_half, src, vlen, p);
}
template <typename R>
void qws_to_planes_gauge(const Geom& G, R* dst, const R* qws, int vlen, cudaStream_t st, bool eo) {
  count_launch();
  k_qws2pl_gauge<R><<<nb(G.V), 128, 0, st>>>(G, dst, qws, vlen, eo ? 1 : 0);
}
template <typename R>
void qws_to_planes_clover(const Geom& G, R* dst, const R* qws, int vlen, cudaStream_t st, bool eo) {
  count_launch();
  k_qws2pl_clover<R><<<nb(G.V), 128, 0, st>>>(G, dst, qws, vlen, eo ? 1 : 0);
}
template <typename R>
void nat_to_planes_spinor(const Geom& G, R* dst, const R* nat, cudaStream_t st, int rhs) {
  count_launch();
  k_nat2pl_sp<R><<<nb(G.V), 128, 0, st>>>(G, dst, nat, rhs);
}
template <typename R>
void planes_to_nat_spinor(const Geom& G, R* nat, const R* src, cudaStream_t st, int rhs) {
  count_launch();
  k_pl2nat_sp<R><<<nb(G.V), 128, 0, st>>>(G, nat, src, rhs);
}
template <typename Rin, typename R>
void nat_to_planes_gauge(const Geom& G, R* dst, const Rin* nat, cudaStream_t st) {
  count_launch();
  k_nat2pl_gauge<Rin, R><<<nb(G.V), 128, 0, st>>>(G, dst, nat);
}
template <typename Rin, typename R>
void nat_to_planes_clover(const Geom& G, R* dst, const Rin* nat, cudaStream_t st) {
  count_launch();
  k_nat2pl_clover<Rin, R><<<nb(G.V), 128, 0, st>>>(G, dst, nat);
}

#define QWSG_INST(R)                                                                             \
  template void qws_to_planes_spinor<R>(const Geom&, R*, const R*, int, int, int, cudaStream_t); \
  template void planes_to_qws_spinor<R>(const Geom&, R*, const R*, int, int, int, cudaStream_t); \
  template void qws_eo_to_planes_spinor<R>(const Geom&, R*, const R*, int, int, cudaStream_t);   \
  template void planes_to_qws_eo_spinor<R>(const Geom&, R*, const R*, int, int, cudaStream_t);   \
  template void qws_to_planes_gauge<R>(const Geom&, R*, const R*, int, cudaStream_t, bool);      \
  template void qws_to_planes_clover<R>(const Geom&, R*, const R*, int, cudaStream_t, bool);     \
  template void nat_to_planes_spinor<R>(const Geom&, R*, const R*, cudaStream_t, int);           \
  template void planes_to_nat_spinor<R>(const Geom&, R*, const R*, cudaStream_t, int);
QWSG_INST(float)
QWSG_INST(double)
#undef QWSG_INST
template void nat_to_planes_gauge<double, double>(const Geom&, double*, const double*, cudaStream_t);
template void nat_to_planes_gauge<double, float>(const Geom&, float*, const double*, cudaStream_t);
template void nat_to_planes_gauge<float, float>(const Geom&, float*, const float*, cudaStream_t);
template void nat_to_planes_clover<double, double>(const Geom&, double*, const double*,
                                                   cudaStream_t);
template void nat_to_planes_clover<double, float>(const Geom&, float*, const double*, cudaStream_t);
template void nat_to_planes_clover<float, float>(const Geom&, float*, const float*, cudaStream_t);

}  // namespace qwsg
