// Device-side lattice geometry and field storage for the B200 DD solver.
//
// Site order in HBM ("DD order"): the lattice is cut into SAP blocks of
// B[0]xB[1]xB[2]xB[3] sites on a block grid NB[4] (NB[0] even).  Blocks are
// coloured (ibx+iby+ibz+ibt) % 2 -- the reference's domain_e/domain_o
// assignment (qws.cc:224-225, 275-276) when NB = (2*npe0, npe1, npe2, npe3).
// Sites are stored colour-major, then block-major, then lexicographic inside
// the block:
//     g = colour*Vh + (block_linear >> 1)*Vb + local
// so every SAP half-sweep (one colour) touches one contiguous half of every
// field, and a block's sites are contiguous.
//
// Fields are structure-of-arrays "planes" of 16-byte (FP32 float4 / FP64
// double2) or 8-byte (FP32 float2 links) vectors with plane stride `pad`
// (>= V, multiple of 128), so a warp's load of one plane is one contiguous,
// fully coalesced 512-byte (or 256-byte) transaction:
//   spinor  : 24 reals/site, per-site order [colour][spin][re,im] (QWS's own,
//             qws.h:134-139); FP32 6 float4 planes, FP64 12 double2 planes.
//   gauge   : per direction mu, U_mu(x)[row][col] complex; 9 complex planes
//             per mu (float2 / double2), plane index mu*9 + 3*row + col.
//   clover  : the reference's packed 2x36 chiral blocks (clover_def.h:88-284);
//             FP32 18 float4 planes, FP64 36 double2 planes.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <type_traits>

namespace qwsg {

// n / d for 0 <= n < 2^31 by a multiply-high (Granlund-Montgomery): with
// s = ceil(log2 d) and m = floor(2^(32+s) / d) + 1 - 2^32 (fits 32 bits),
// floor(n / d) = (umulhi(n, m) + n) >> s exactly for every n < 2^32; the sum
// cannot overflow for n < 2^31.  Replaces the integer divisions of the site
// decoding, which ran in every hop thread.
struct FastDiv {
  unsigned m;
  int s;
};
inline FastDiv make_fastdiv(int d) {
  int s = 0;
  while ((1u << s) < (unsigned)d) s++;
  const unsigned long long m = ((1ull << (32 + s)) / (unsigned long long)d) + 1 - (1ull << 32);
  return {(unsigned)m, s};
}
__host__ __device__ __forceinline__ int fdiv(int n, FastDiv f) {
#ifdef __CUDA_ARCH__
  const unsigned hi = __umulhi((unsigned)n, f.m);
#else
  const unsigned hi = (unsigned)(((unsigned long long)(unsigned)n * f.m) >> 32);
#endif
  return (int)((hi + (unsigned)n) >> f.s);
}

struct Geom {
  int L[4];    // global extents
  int B[4];    // block extents
  int NB[4];   // block grid
  int Vb;      // sites per block
  int V;       // sites
  int Vh;      // sites per colour
  int nbh0;    // NB[0] / 2
  int tbc;     // +1 periodic / -1 antiperiodic in t (fbc_f[3], qws.cc:298-310)
  int pad;     // plane stride in elements
  int str[4];  // in-block strides of x, y, z, t (block_local)
  int rot;     // the fastest in-block direction (str 1), stored rotated by one
  // right-hand sides per spinor field (a power of two, 1..32).  Spinor
  // fields interleave them RHS-minor: RHS r of site g is entry
  // (g << lgnr) + r of planes with stride pad << lgnr, so the threads of one
  // site's RHS sit side by side in a warp and share every link and clover
  // load.  Gauge and clover fields are per site (stride pad).
  int nr;
  int lgnr;
  // threads per CTA of the hop kernels (a launch shape: 64, 128 or 256;
  // host-side only, chosen per lattice)
  int hop_threads;
  // multipliers for the divisions of the site decoding
  FastDiv fB[4], fVb, fnbh0, fNB1, fNB2, fstr[4];
};

// The members of G that follow from its extents L, block extents B and block
// grid NB (set and checked by the caller): site counts, plane stride, the
// in-block order (block_local) and the multipliers of the site decoding.
//
// In-block order: the faces of the fastest direction are the only strided
// ones, so it should have the largest extent; the slowest direction's stride
// Vb/B_slowest is how far apart in a launch a site and its farthest neighbour
// are read, which must stay within a few MB for the neighbour to be in L2
// (16384 sites, ~13 MB of FP32 operator traffic).  Take the largest-extent
// direction as fastest whose remaining largest extent, made slowest,
// satisfies that; else the largest slowest and the second largest fastest.
// Ties: t, z, y, x.
inline void geom_layout(Geom& G) {
  G.V = G.L[0] * G.L[1] * G.L[2] * G.L[3];
  G.Vh = G.V / 2;
  G.Vb = G.B[0] * G.B[1] * G.B[2] * G.B[3];
  G.nbh0 = G.NB[0] / 2;
  G.pad = (G.V + 127) / 128 * 128;
  int d[4] = {3, 2, 1, 0};
  std::stable_sort(d, d + 4, [&](int a, int b) { return G.B[a] > G.B[b]; });
  int order[4] = {d[1], d[2], d[3], d[0]};  // fastest .. slowest
  for (int f = 0; f < 4; f++) {
    const int slow = d[f == 0 ? 1 : 0];
    if (G.Vb / G.B[slow] <= 16384) {
      int k = 0;
      order[k++] = d[f];
      for (int j = 0; j < 4; j++)
        if (j != f && d[j] != slow) order[k++] = d[j];
      order[3] = slow;
      break;
    }
  }
  int stride = 1;
  for (int k = 0; k < 4; k++) {
    G.str[order[k]] = stride;
    stride *= G.B[order[k]];
  }
  G.rot = order[0];
  for (int mu = 0; mu < 4; mu++) G.fstr[mu] = make_fastdiv(G.str[mu]);
  for (int mu = 0; mu < 4; mu++) G.fB[mu] = make_fastdiv(G.B[mu]);
  G.fVb = make_fastdiv(G.Vb);
  G.fnbh0 = make_fastdiv(G.nbh0);
  G.fNB1 = make_fastdiv(G.NB[1]);
  G.fNB2 = make_fastdiv(G.NB[2]);
}

// plane stride of spinor fields and the entry of (site, rhs)
__host__ __device__ __forceinline__ int spad(const Geom& G) { return G.pad << G.lgnr; }
__host__ __device__ __forceinline__ int sentry(const Geom& G, int g, int r) {
  return (g << G.lgnr) + r;
}

struct Site {
  int col;     // block colour
  int lc[4];   // coordinates inside the block
  int bc[4];   // block coordinates
};

// Inside a block, sites are lexicographic in an order of the four
// directions chosen per block shape (G.str, set by geom_layout):
// the largest extent is slowest, so the far neighbours of a site are the
// nearest they can be and stay in L2 between the launches' reads; the
// second largest is fastest, so every block face but that direction's is a
// run of whole rows and the face kernels read whole sectors.
//
// Along the fastest direction a row is stored rotated by one -- in-block
// coordinates B-1, 0, 1, ..., B-2 -- so that the row's two face sites (0 and
// B-1) are adjacent: the face kernels, which visit only face sites, then read
// them as one 32-byte sector instead of two sectors that each hold one site.
// Interior hops along that direction keep stride 1 except the step between
// B-2 and B-1 (see rot_step).
__host__ __device__ __forceinline__ int rot_pos(const Geom& G, int mu, int l) {
  return mu == G.rot ? (l + 1 == G.B[mu] ? 0 : l + 1) : l;
}
__host__ __device__ __forceinline__ int rot_coord(const Geom& G, int mu, int p) {
  return mu == G.rot ? (p == 0 ? G.B[mu] - 1 : p - 1) : p;
}
__host__ __device__ __forceinline__ int block_local(const Geom& G, const int lc[4]) {
  return rot_pos(G, 0, lc[0]) * G.str[0] + rot_pos(G, 1, lc[1]) * G.str[1] +
         rot_pos(G, 2, lc[2]) * G.str[2] + rot_pos(G, 3, lc[3]) * G.str[3];
}
// whether DD-order site g lies on a face of its block (an in-block
// coordinate 0 or B-1): the sites the face kernels visit
__host__ __device__ __forceinline__ bool on_block_face(const Geom& G, int g) {
  const int col = g >= G.Vh;
  const int t = (g - col * G.Vh) % G.Vb;
  bool face = false;
  for (int mu = 0; mu < 4; mu++) {
    const int l = rot_coord(G, mu, (t / G.str[mu]) % G.B[mu]);
    face |= (l == 0) || (l == G.B[mu] - 1);
  }
  return face;
}
// offset of the interior hop from in-block coordinate l to l + dir along mu
__host__ __device__ __forceinline__ int rot_step(const Geom& G, int mu, int l, int dir) {
  int d = dir * G.str[mu];
  if (mu == G.rot) {
    if (dir > 0 && l == G.B[mu] - 2) d -= G.B[mu];  // B-2 -> B-1: back to the row's start
    if (dir < 0 && l == G.B[mu] - 1) d += G.B[mu];  // B-1 -> B-2: to the row's end
  }
  return d;
}

__host__ __device__ __forceinline__ void decode_site(const Geom& G, int g, Site& s) {
  s.col = g >= G.Vh;
  int rem = g - s.col * G.Vh;
  int k = fdiv(rem, G.fVb);
  int t = rem - k * G.Vb;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    const int q = fdiv(t, G.fstr[mu]);
    s.lc[mu] = rot_coord(G, mu, q - fdiv(q, G.fB[mu]) * G.B[mu]);
  }
  int q = fdiv(k, G.fnbh0);
  int r = k - q * G.nbh0;
  int q1 = fdiv(q, G.fNB1);
  s.bc[1] = q - q1 * G.NB[1];
  int q2 = fdiv(q1, G.fNB2);
  s.bc[2] = q1 - q2 * G.NB[2];
  s.bc[3] = q2;
  s.bc[0] = 2 * r + ((s.col + s.bc[1] + s.bc[2] + s.bc[3]) & 1);
}

// DD-order index of the site with global coordinates x
__host__ __device__ __forceinline__ int dd_index(const Geom& G, const int x[4]) {
  int bc[4], lc[4];
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    bc[mu] = fdiv(x[mu], G.fB[mu]);
    lc[mu] = x[mu] - bc[mu] * G.B[mu];
  }
  int col = (bc[0] + bc[1] + bc[2] + bc[3]) & 1;
  int blin = bc[0] + G.NB[0] * (bc[1] + G.NB[1] * (bc[2] + G.NB[2] * bc[3]));
  return col * G.Vh + (blin >> 1) * G.Vb + block_local(G, lc);
}

// global coordinates of the site with DD-order index g
__device__ __forceinline__ void site_coords(const Geom& G, int g, int x[4]) {
  Site s;
  decode_site(G, g, s);
#pragma unroll
  for (int mu = 0; mu < 4; mu++) x[mu] = s.bc[mu] * G.B[mu] + s.lc[mu];
}

// index of the neighbour across the block face in direction mu (dir = +1/-1)
__host__ __device__ __forceinline__ int nbr_across(const Geom& G, const Site& s, int mu, int dir,
                                                   int* ncol) {
  int bc0 = s.bc[0], bc1 = s.bc[1], bc2 = s.bc[2], bc3 = s.bc[3];
  int l0 = s.lc[0], l1 = s.lc[1], l2 = s.lc[2], l3 = s.lc[3];
  int* bcp = mu == 0 ? &bc0 : mu == 1 ? &bc1 : mu == 2 ? &bc2 : &bc3;
  int* lcp = mu == 0 ? &l0 : mu == 1 ? &l1 : mu == 2 ? &l2 : &l3;
  if (dir > 0) {
    *lcp = 0;
    *bcp = (*bcp + 1 == G.NB[mu]) ? 0 : *bcp + 1;
  } else {
    *lcp = G.B[mu] - 1;
    *bcp = (*bcp == 0) ? G.NB[mu] - 1 : *bcp - 1;
  }
  int col = (bc0 + bc1 + bc2 + bc3) & 1;
  int blin = bc0 + G.NB[0] * (bc1 + G.NB[1] * (bc2 + G.NB[2] * bc3));
  const int lc[4] = {l0, l1, l2, l3};
  *ncol = col;
  return col * G.Vh + (blin >> 1) * G.Vb + block_local(G, lc);
}

// ---------------------------------------------------------------------------
// Values the stencil computes with: a scalar (float, double) or F2, two FP32
// lanes (two right-hand sides of one site) in one 64-bit register pair,
// computed with sm_100's packed FP32x2 instructions (add/sub/mul/fma .f32x2:
// two IEEE single-precision results per instruction, each rounded as the
// scalar instruction rounds it).  The stencil pieces below use madd(a, b, c)
// = a*b + c with one rounding and a fixed order of operations, so a lane of
// F2 computes bit for bit what the scalar float code computes.
// ---------------------------------------------------------------------------
struct F2 {
  float x, y;
};

__device__ __forceinline__ unsigned long long f2_bits(F2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ F2 f2_from_bits(unsigned long long r) {
  F2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ F2 operator+(F2 a, F2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return f2_from_bits(d);
}
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return f2_from_bits(d);
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return f2_from_bits(d);
}
__device__ __forceinline__ F2 operator-(F2 a) { return F2{-a.x, -a.y}; }
__device__ __forceinline__ F2& operator+=(F2& a, F2 b) { return a = a + b; }
__device__ __forceinline__ F2& operator-=(F2& a, F2 b) { return a = a - b; }

__device__ __forceinline__ float madd(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double madd(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ F2 madd(F2 a, F2 b, F2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)), "l"(f2_bits(c)));
  return f2_from_bits(d);
}

// a site quantity (link or clover entry) for every lane of V
template <typename V>
struct Lanes {
  template <typename R>
  __device__ __forceinline__ static V bcast(R a) { return (V)a; }
};
template <>
struct Lanes<F2> {
  __device__ __forceinline__ static F2 bcast(float a) { return F2{a, a}; }
};

// ---------------------------------------------------------------------------
// plane I/O.  A storage tag T selects the in-memory format; arithmetic is in
// Arith<T>::R.  float / double store what they compute; H16 stores FP16 and
// computes in FP32:
//   spinor  three 16-byte planes of 8 halves holding v / n (grouped so that
//           a t-hop's half spinor is one 16- and one 8-byte load, see
//           IO<H16>), followed by one float plane of per-site scales
//           n = max |v_i| over the 24 reals (a per-site norm);
//   gauge   per direction two 16-byte planes and one 4-byte plane (the 9
//           complex entries, which are <= 1 for SU(3));
//   clover  nine 16-byte planes (the 72 reals; block 0 = reals 0-35).
// ---------------------------------------------------------------------------
struct H16 {};

template <typename T>
struct Arith {
  using R = T;
};
template <>
struct Arith<H16> {
  using R = float;
};
template <typename T>
struct Store {
  using type = T;
};
template <>
struct Store<H16> {
  using type = __half;
};

template <typename R>
struct IO;

template <>
struct IO<float> {
  __device__ __forceinline__ static void load_spinor(const float* __restrict__ p, int pad, int g,
                                                     float v[24]) {
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      float4 t = __ldg(q + (size_t)j * pad + g);
      v[4 * j + 0] = t.x;
      v[4 * j + 1] = t.y;
      v[4 * j + 2] = t.z;
      v[4 * j + 3] = t.w;
    }
  }
  // the *_raw loads return the stored values and the site's scale (1 here)
  __device__ __forceinline__ static void load_spinor_raw(const float* __restrict__ p, int pad,
                                                         int g, float v[24], float& s) {
    load_spinor(p, pad, g, v);
    s = 1.0f;
  }
  __device__ __forceinline__ static void load_half_raw(const float* __restrict__ p, int pad, int g,
                                                       int upper, float v[24], float& s) {
    load_half(p, pad, g, upper, v);
    s = 1.0f;
  }
  // spins {s0, s0+1} only (t-direction projections need half the spinor)
  __device__ __forceinline__ static void load_half(const float* __restrict__ p, int pad, int g,
                                                   int upper, float v[24]) {
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      int j = 2 * c + (upper ? 1 : 0);
      float4 t = __ldg(q + (size_t)j * pad + g);
      v[4 * j + 0] = t.x;
      v[4 * j + 1] = t.y;
      v[4 * j + 2] = t.z;
      v[4 * j + 3] = t.w;
    }
  }
  __device__ __forceinline__ static void store_spinor(float* __restrict__ p, int pad, int g,
                                                      const float v[24]) {
    float4* q = reinterpret_cast<float4*>(p);
#pragma unroll
    for (int j = 0; j < 6; j++)
      q[(size_t)j * pad + g] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
  }
  __device__ __forceinline__ static void load_link(const float* __restrict__ U, int pad, int mu,
                                                   int g, float u[18]) {
    const float2* q = reinterpret_cast<const float2*>(U);
#pragma unroll
    for (int e = 0; e < 9; e++) {
      float2 t = __ldg(q + (size_t)(mu * 9 + e) * pad + g);
      u[2 * e] = t.x;
      u[2 * e + 1] = t.y;
    }
  }
  __device__ __forceinline__ static void load_clover_block(const float* __restrict__ C, int pad,
                                                           int g, int blk, float a[36]) {
    const float4* q = reinterpret_cast<const float4*>(C);
#pragma unroll
    for (int j = 0; j < 9; j++) {
      float4 t = __ldg(q + (size_t)(9 * blk + j) * pad + g);
      a[4 * j + 0] = t.x;
      a[4 * j + 1] = t.y;
      a[4 * j + 2] = t.z;
      a[4 * j + 3] = t.w;
    }
  }
};

template <>
struct IO<double> {
  __device__ __forceinline__ static void load_spinor(const double* __restrict__ p, int pad, int g,
                                                     double v[24]) {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int j = 0; j < 12; j++) {
      double2 t = __ldg(q + (size_t)j * pad + g);
      v[2 * j] = t.x;
      v[2 * j + 1] = t.y;
    }
  }
  __device__ __forceinline__ static void load_spinor_raw(const double* __restrict__ p, int pad,
                                                         int g, double v[24], double& s) {
    load_spinor(p, pad, g, v);
    s = 1.0;
  }
  __device__ __forceinline__ static void load_half_raw(const double* __restrict__ p, int pad,
                                                       int g, int upper, double v[24], double& s) {
    load_half(p, pad, g, upper, v);
    s = 1.0;
  }
  __device__ __forceinline__ static void load_half(const double* __restrict__ p, int pad, int g,
                                                   int upper, double v[24]) {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int s = 0; s < 2; s++) {
        int j = 4 * c + 2 * (upper ? 1 : 0) + s;
        double2 t = __ldg(q + (size_t)j * pad + g);
        v[2 * j] = t.x;
        v[2 * j + 1] = t.y;
      }
  }
  __device__ __forceinline__ static void store_spinor(double* __restrict__ p, int pad, int g,
                                                      const double v[24]) {
    double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
    for (int j = 0; j < 12; j++) q[(size_t)j * pad + g] = make_double2(v[2 * j], v[2 * j + 1]);
  }
  __device__ __forceinline__ static void load_link(const double* __restrict__ U, int pad, int mu,
                                                   int g, double u[18]) {
    const double2* q = reinterpret_cast<const double2*>(U);
#pragma unroll
    for (int e = 0; e < 9; e++) {
      double2 t = __ldg(q + (size_t)(mu * 9 + e) * pad + g);
      u[2 * e] = t.x;
      u[2 * e + 1] = t.y;
    }
  }
  __device__ __forceinline__ static void load_clover_block(const double* __restrict__ C, int pad,
                                                           int g, int blk, double a[36]) {
    const double2* q = reinterpret_cast<const double2*>(C);
#pragma unroll
    for (int j = 0; j < 18; j++) {
      double2 t = __ldg(q + (size_t)(18 * blk + j) * pad + g);
      a[2 * j] = t.x;
      a[2 * j + 1] = t.y;
    }
  }
};

template <>
struct IO<H16> {
  // Spinor fields: three 16-byte planes and a float plane of per-site scales.
  //   P0 = spins 0-1 of colours 0-1   (reals 0-3, 8-11 of [c][s][ri])
  //   P1 = spins 2-3 of colours 0-1   (reals 4-7, 12-15)
  //   P2 = colour 2, spins 0-1 then 2-3 (reals 16-23)
  // A full spinor is three 16-byte loads; the half spinor a t-hop projects
  // (spins 0-1 or 2-3) is one 16-byte and one 8-byte load.
  __device__ __forceinline__ static const float* scale_plane(const __half* p, int pad) {
    return reinterpret_cast<const float*>(reinterpret_cast<const uint4*>(p) + (size_t)3 * pad);
  }
  __device__ __forceinline__ static float scale(const __half* p, int pad, int g) {
    return __ldg(scale_plane(p, pad) + g);
  }
  __device__ __forceinline__ static void unpack4(unsigned x, unsigned y, float s, float* o) {
    __half2 a, b;
    memcpy(&a, &x, 4);
    memcpy(&b, &y, 4);
    float2 fa = __half22float2(a), fb = __half22float2(b);
    o[0] = fa.x * s;
    o[1] = fa.y * s;
    o[2] = fb.x * s;
    o[3] = fb.y * s;
  }
  __device__ __forceinline__ static void unpack4(uint2 t, float s, float* o) {
    unpack4(t.x, t.y, s, o);
  }
  __device__ __forceinline__ static uint2 pack4(const float* v, float inv) {
    __half2 a = __floats2half2_rn(v[0] * inv, v[1] * inv);
    __half2 b = __floats2half2_rn(v[2] * inv, v[3] * inv);
    uint2 t;
    memcpy(&t.x, &a, 4);
    memcpy(&t.y, &b, 4);
    return t;
  }
  // the stored (normalised) values; the site's scale in s
  __device__ __forceinline__ static void load_spinor_raw(const __half* __restrict__ p, int pad,
                                                         int g, float v[24], float& s) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
    s = scale(p, pad, g);
    const uint4 a = __ldg(q + g), b = __ldg(q + (size_t)pad + g), c = __ldg(q + (size_t)2 * pad + g);
    unpack4(a.x, a.y, 1.0f, v + 0);
    unpack4(a.z, a.w, 1.0f, v + 8);
    unpack4(b.x, b.y, 1.0f, v + 4);
    unpack4(b.z, b.w, 1.0f, v + 12);
    unpack4(c.x, c.y, 1.0f, v + 16);
    unpack4(c.z, c.w, 1.0f, v + 20);
  }
  __device__ __forceinline__ static void load_spinor(const __half* __restrict__ p, int pad, int g,
                                                     float v[24]) {
    float s;
    load_spinor_raw(p, pad, g, v, s);
#pragma unroll
    for (int j = 0; j < 24; j++) v[j] *= s;
  }
  // upper = 0: spins 0-1 (reals 0-3, 8-11, 16-19); 1: spins 2-3 (+4)
  __device__ __forceinline__ static void load_half_raw(const __half* __restrict__ p, int pad,
                                                       int g, int upper, float v[24], float& s) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
    s = scale(p, pad, g);
    const int o = upper ? 4 : 0;
    const uint4 a = __ldg(q + (size_t)(upper ? pad : 0) + g);
    const uint2 c = __ldg(reinterpret_cast<const uint2*>(q + (size_t)2 * pad) + 2 * (size_t)g + (upper ? 1 : 0));
    unpack4(a.x, a.y, 1.0f, v + o);
    unpack4(a.z, a.w, 1.0f, v + 8 + o);
    unpack4(c, 1.0f, v + 16 + o);
  }
  __device__ __forceinline__ static void load_half(const __half* __restrict__ p, int pad, int g,
                                                   int upper, float v[24]) {
    float s;
    load_half_raw(p, pad, g, upper, v, s);
    const int o = upper ? 4 : 0;
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int k = 0; k < 4; k++) v[8 * c + o + k] *= s;
  }
  __device__ __forceinline__ static void store_spinor(__half* __restrict__ p, int pad, int g,
                                                      const float v[24]) {
    float n = 0;
#pragma unroll
    for (int j = 0; j < 24; j++) n = fmaxf(n, fabsf(v[j]));
    // A site whose largest component is below 1e-30 is stored as zero: 1/n
    // overflows FP32 for denormal n (0 * inf would give NaN), and such
    // entries sit far below what FP16 storage resolves next to the O(1)
    // entries of the normalised fields the SAP works on (a point source's
    // solution decays below FP32's normal range across a large lattice).
    const bool keep = n >= 1e-30f;
    const float inv = keep ? 1.0f / n : 0.0f;
    uint4* q = reinterpret_cast<uint4*>(p);
    const uint2 a0 = pack4(v + 0, inv), a1 = pack4(v + 8, inv);
    const uint2 b0 = pack4(v + 4, inv), b1 = pack4(v + 12, inv);
    const uint2 c0 = pack4(v + 16, inv), c1 = pack4(v + 20, inv);
    q[g] = make_uint4(a0.x, a0.y, a1.x, a1.y);
    q[(size_t)pad + g] = make_uint4(b0.x, b0.y, b1.x, b1.y);
    q[(size_t)2 * pad + g] = make_uint4(c0.x, c0.y, c1.x, c1.y);
    reinterpret_cast<float*>(q + (size_t)3 * pad)[g] = keep ? n : 0.0f;
  }
  // Links: per direction 36 bytes a site, as two 16-byte planes (complex
  // elements 0-3 and 4-7 of the row-major matrix) and one 4-byte plane
  // (element 8): three loads per link.
  __device__ __forceinline__ static void load_link(const __half* __restrict__ U, int pad, int mu,
                                                   int g, float u[18]) {
    const char* base = reinterpret_cast<const char*>(U) + (size_t)mu * 36 * pad;
    const uint4 a = __ldg(reinterpret_cast<const uint4*>(base) + g);
    const uint4 b = __ldg(reinterpret_cast<const uint4*>(base + (size_t)16 * pad) + g);
    const unsigned c = __ldg(reinterpret_cast<const unsigned*>(base + (size_t)32 * pad) + g);
    const unsigned w[9] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c};
#pragma unroll
    for (int e = 0; e < 9; e++) {
      __half2 h;
      memcpy(&h, &w[e], 4);
      const float2 f = __half22float2(h);
      u[2 * e] = f.x;
      u[2 * e + 1] = f.y;
    }
  }
  __device__ __forceinline__ static void store_link(__half* U, int pad, int mu, int g,
                                                    const float u[18]) {
    char* base = reinterpret_cast<char*>(U) + (size_t)mu * 36 * pad;
    unsigned w[9];
#pragma unroll
    for (int e = 0; e < 9; e++) {
      const __half2 h = __floats2half2_rn(u[2 * e], u[2 * e + 1]);
      memcpy(&w[e], &h, 4);
    }
    reinterpret_cast<uint4*>(base)[g] = make_uint4(w[0], w[1], w[2], w[3]);
    reinterpret_cast<uint4*>(base + (size_t)16 * pad)[g] = make_uint4(w[4], w[5], w[6], w[7]);
    reinterpret_cast<unsigned*>(base + (size_t)32 * pad)[g] = w[8];
  }
  // Clover: the 72 reals (two chiral blocks of 36) as nine 16-byte planes;
  // block 0 is planes 0-3 and the first half of plane 4, block 1 the second
  // half of plane 4 and planes 5-8.
  __device__ __forceinline__ static void load_clover_block(const __half* __restrict__ C, int pad,
                                                           int g, int blk, float a[36]) {
    const uint4* q = reinterpret_cast<const uint4*>(C);
    const uint2 mid = __ldg(reinterpret_cast<const uint2*>(q + (size_t)4 * pad) + 2 * (size_t)g + blk);
    const int first = blk ? 5 : 0, o = blk ? 4 : 0;
    if (blk) unpack4(mid, 1.0f, a);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const uint4 t = __ldg(q + (size_t)(first + j) * pad + g);
      unpack4(t.x, t.y, 1.0f, a + o + 8 * j);
      unpack4(t.z, t.w, 1.0f, a + o + 8 * j + 4);
    }
    if (!blk) unpack4(mid, 1.0f, a + 32);
  }
  __device__ __forceinline__ static void store_clover(__half* C, int pad, int g, const float a[72]) {
    uint4* q = reinterpret_cast<uint4*>(C);
#pragma unroll
    for (int j = 0; j < 9; j++) {
      const uint2 x = pack4(a + 8 * j, 1.0f), y = pack4(a + 8 * j + 4, 1.0f);
      q[(size_t)j * pad + g] = make_uint4(x.x, x.y, y.x, y.y);
    }
  }
};

// FP16 spinors of a multi-RHS field computed two right-hand sides per
// thread (F2 lanes): the entry of (site g, RHS pair p) is (g << (lgnr-1)) + p
// with plane stride pad << (lgnr-1); six 16-byte planes whose 32-bit words
// hold one component of both RHS as a half2 (plane k, word j: component
// 4k + j), then a float2 plane of the two RHS' scales.  The same bytes per
// (site, RHS) as IO<H16>, and the same half values: only the order differs.
struct IOP {
  __device__ __forceinline__ static F2 f2_of(unsigned w) {
    __half2 h;
    memcpy(&h, &w, 4);
    const float2 f = __half22float2(h);
    return F2{f.x, f.y};
  }
  __device__ __forceinline__ static unsigned word_of(F2 v) {
    const __half2 h = __floats2half2_rn(v.x, v.y);
    unsigned w;
    memcpy(&w, &h, 4);
    return w;
  }
  __device__ __forceinline__ static F2 scale(const __half* p, int ppad, int e) {
    const float2 s =
        __ldg(reinterpret_cast<const float2*>(reinterpret_cast<const uint4*>(p) + (size_t)6 * ppad) + e);
    return F2{s.x, s.y};
  }
  __device__ __forceinline__ static void load_spinor_raw(const __half* __restrict__ p, int ppad,
                                                         int e, F2 v[24], F2& s) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
    s = scale(p, ppad, e);
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const uint4 t = __ldg(q + (size_t)k * ppad + e);
      v[4 * k] = f2_of(t.x);
      v[4 * k + 1] = f2_of(t.y);
      v[4 * k + 2] = f2_of(t.z);
      v[4 * k + 3] = f2_of(t.w);
    }
  }
  // spins 0-1 (upper = 0) or 2-3 of every colour: planes 2c + upper
  __device__ __forceinline__ static void load_half_raw(const __half* __restrict__ p, int ppad,
                                                       int e, int upper, F2 v[24], F2& s) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
    s = scale(p, ppad, e);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const int k = 2 * c + (upper ? 1 : 0);
      const uint4 t = __ldg(q + (size_t)k * ppad + e);
      v[4 * k] = f2_of(t.x);
      v[4 * k + 1] = f2_of(t.y);
      v[4 * k + 2] = f2_of(t.z);
      v[4 * k + 3] = f2_of(t.w);
    }
  }
  __device__ __forceinline__ static void load_spinor(const __half* __restrict__ p, int ppad, int e,
                                                     F2 v[24]) {
    F2 s;
    load_spinor_raw(p, ppad, e, v, s);
#pragma unroll
    for (int j = 0; j < 24; j++) v[j] = v[j] * s;
  }
  // per lane exactly IO<H16>::store_spinor
  __device__ __forceinline__ static void store_spinor(__half* __restrict__ p, int ppad, int e,
                                                      const F2 v[24]) {
    float n0 = 0, n1 = 0;
#pragma unroll
    for (int j = 0; j < 24; j++) {
      n0 = fmaxf(n0, fabsf(v[j].x));
      n1 = fmaxf(n1, fabsf(v[j].y));
    }
    const bool k0 = n0 >= 1e-30f, k1 = n1 >= 1e-30f;
    const F2 inv{k0 ? 1.0f / n0 : 0.0f, k1 ? 1.0f / n1 : 0.0f};
    uint4* q = reinterpret_cast<uint4*>(p);
#pragma unroll
    for (int k = 0; k < 6; k++)
      q[(size_t)k * ppad + e] = make_uint4(word_of(v[4 * k] * inv), word_of(v[4 * k + 1] * inv),
                                           word_of(v[4 * k + 2] * inv), word_of(v[4 * k + 3] * inv));
    reinterpret_cast<float2*>(q + (size_t)6 * ppad)[e] = make_float2(k0 ? n0 : 0.0f, k1 ? n1 : 0.0f);
  }
};

// bytes each format moves per site (algorithmic traffic accounting)
template <typename T>
struct Bytes {
  static constexpr int spinor = 24 * sizeof(T);
  static constexpr int links = 72 * sizeof(T);  // 4 directions
  static constexpr int clover = 72 * sizeof(T);
};
template <>
struct Bytes<H16> {
  static constexpr int spinor = 48 + 4;
  static constexpr int links = 72 * 2;
  static constexpr int clover = 72 * 2;
};

// ---------------------------------------------------------------------------
// Wilson hop pieces.  v[24] = spinor [c][s][ri]; h = 2-spinor per colour.
// Spin projections and reconstructions follow the reference's Dirac-basis
// conventions (wilson_d.h: __s_xf/__s_xb/__s_yf/..., ddd_in_d.cc:97-178):
//   x+  h = (v0 - i v3, v1 - i v2)   recon (h0, h1,  i h1,  i h0)
//   x-  h = (v0 + i v3, v1 + i v2)   recon (h0, h1, -i h1, -i h0)
//   y+  h = (v0 - v3,   v1 + v2)     recon (h0, h1,  h1,   -h0)
//   y-  h = (v0 + v3,   v1 - v2)     recon (h0, h1, -h1,    h0)
//   z+  h = (v0 - i v2, v1 + i v3)   recon (h0, h1,  i h0, -i h1)
//   z-  h = (v0 + i v2, v1 - i v3)   recon (h0, h1, -i h0,  i h1)
//   t+  h = (v2, v3) * 2             recon (0, 0, h0, h1)
//   t-  h = (v0, v1) * 2             recon (h0, h1, 0, 0)
// ---------------------------------------------------------------------------
#define RE(c, s) v[8 * (c) + 2 * (s)]
#define IM(c, s) v[8 * (c) + 2 * (s) + 1]

template <typename R, int MU, int DIR>
__device__ __forceinline__ void project(const R v[24], R h[12]) {
  // h[4*c + 2*k + ri]
#pragma unroll
  for (int c = 0; c < 3; c++) {
    R* o = h + 4 * c;
    if (MU == 0 && DIR > 0) {
      o[0] = RE(c, 0) + IM(c, 3); o[1] = IM(c, 0) - RE(c, 3);
      o[2] = RE(c, 1) + IM(c, 2); o[3] = IM(c, 1) - RE(c, 2);
    } else if (MU == 0) {
      o[0] = RE(c, 0) - IM(c, 3); o[1] = IM(c, 0) + RE(c, 3);
      o[2] = RE(c, 1) - IM(c, 2); o[3] = IM(c, 1) + RE(c, 2);
    } else if (MU == 1 && DIR > 0) {
      o[0] = RE(c, 0) - RE(c, 3); o[1] = IM(c, 0) - IM(c, 3);
      o[2] = RE(c, 1) + RE(c, 2); o[3] = IM(c, 1) + IM(c, 2);
    } else if (MU == 1) {
      o[0] = RE(c, 0) + RE(c, 3); o[1] = IM(c, 0) + IM(c, 3);
      o[2] = RE(c, 1) - RE(c, 2); o[3] = IM(c, 1) - IM(c, 2);
    } else if (MU == 2 && DIR > 0) {
      o[0] = RE(c, 0) + IM(c, 2); o[1] = IM(c, 0) - RE(c, 2);
      o[2] = RE(c, 1) - IM(c, 3); o[3] = IM(c, 1) + RE(c, 3);
    } else if (MU == 2) {
      o[0] = RE(c, 0) - IM(c, 2); o[1] = IM(c, 0) + RE(c, 2);
      o[2] = RE(c, 1) + IM(c, 3); o[3] = IM(c, 1) - RE(c, 3);
    } else if (MU == 3 && DIR > 0) {
      o[0] = RE(c, 2); o[1] = IM(c, 2); o[2] = RE(c, 3); o[3] = IM(c, 3);
    } else {
      o[0] = RE(c, 0); o[1] = IM(c, 0); o[2] = RE(c, 1); o[3] = IM(c, 1);
    }
  }
}
#undef RE
#undef IM

// r = U h (forward) or U^dagger h (backward); U row-major complex [3][3].
// Products in a fixed order (one rounding each), the minus signs taken from
// the negated h components.
// (-a) b + c: a scalar takes the minus as an operand modifier of its fused
// multiply-add; F2 lanes use a negated copy of b made once (same value:
// negation is exact)
template <typename R>
struct Neg {
  static constexpr bool copies = false;
};
template <>
struct Neg<F2> {
  static constexpr bool copies = true;
};

template <typename R, bool DAG>
__device__ __forceinline__ void link_mul(const R u[18], const R h[12], R r[12]) {
  if constexpr (std::is_same<R, double>::value) {
    // FP64: sums left to the compiler's contraction (fewer registers)
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int k = 0; k < 2; k++) {
        R re = 0, im = 0;
#pragma unroll
        for (int b = 0; b < 3; b++) {
          const int e = DAG ? 3 * b + a : 3 * a + b;
          const R ur = u[2 * e], ui = DAG ? -u[2 * e + 1] : u[2 * e + 1];
          const R hr = h[4 * b + 2 * k], hi = h[4 * b + 2 * k + 1];
          re += ur * hr - ui * hi;
          im += ur * hi + ui * hr;
        }
        r[4 * a + 2 * k] = re;
        r[4 * a + 2 * k + 1] = im;
      }
    return;
  }
  R nh[6];  // F2 only: -h_i (forward) or -h_r (backward)
  if (Neg<R>::copies) {
#pragma unroll
    for (int j = 0; j < 6; j++) nh[j] = -h[2 * j + (DAG ? 0 : 1)];
  }
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int k = 0; k < 2; k++) {
      R re, im;
#pragma unroll
      for (int b = 0; b < 3; b++) {
        const int e = DAG ? 3 * b + a : 3 * a + b;
        const R ur = u[2 * e], ui = u[2 * e + 1];
        const R hr = h[4 * b + 2 * k], hi = h[4 * b + 2 * k + 1];
        if (b == 0) {
          re = ur * hr;
          im = ur * hi;
        } else {
          re = madd(ur, hr, re);
          im = madd(ur, hi, im);
        }
        if (DAG) {  // conj(u): re += ui hi, im -= ui hr
          re = madd(ui, hi, re);
          im = Neg<R>::copies ? madd(ui, nh[2 * b + k], im) : madd(-ui, hr, im);
        } else {    // re -= ui hi, im += ui hr
          re = Neg<R>::copies ? madd(ui, nh[2 * b + k], re) : madd(-ui, hi, re);
          im = madd(ui, hr, im);
        }
      }
      r[4 * a + 2 * k] = re;
      r[4 * a + 2 * k + 1] = im;
    }
}

#define AR(c, s) acc[8 * (c) + 2 * (s)]
#define AI(c, s) acc[8 * (c) + 2 * (s) + 1]
// acc += recon(f r); f: the hop's factor times the source's scale (FP16
// storage; 1 otherwise).  Additions as madd(+-f, r, acc).
template <typename R, int MU, int DIR>
__device__ __forceinline__ void reconstruct(const R r[12], R acc[24], R f) {
  if constexpr (std::is_same<R, double>::value) {
    // FP64 (f = 1 but for the t hops): plain sums
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const R r0 = f * r[4 * c], i0 = f * r[4 * c + 1], r1 = f * r[4 * c + 2], i1 = f * r[4 * c + 3];
      if (MU == 3) {
        if (DIR > 0) {
          AR(c, 2) += r0; AI(c, 2) += i0; AR(c, 3) += r1; AI(c, 3) += i1;
        } else {
          AR(c, 0) += r0; AI(c, 0) += i0; AR(c, 1) += r1; AI(c, 1) += i1;
        }
        continue;
      }
      AR(c, 0) += r0; AI(c, 0) += i0; AR(c, 1) += r1; AI(c, 1) += i1;
      if (MU == 0 && DIR > 0) {
        AR(c, 2) -= i1; AI(c, 2) += r1; AR(c, 3) -= i0; AI(c, 3) += r0;
      } else if (MU == 0) {
        AR(c, 2) += i1; AI(c, 2) -= r1; AR(c, 3) += i0; AI(c, 3) -= r0;
      } else if (MU == 1 && DIR > 0) {
        AR(c, 2) += r1; AI(c, 2) += i1; AR(c, 3) -= r0; AI(c, 3) -= i0;
      } else if (MU == 1) {
        AR(c, 2) -= r1; AI(c, 2) -= i1; AR(c, 3) += r0; AI(c, 3) += i0;
      } else if (MU == 2 && DIR > 0) {
        AR(c, 2) -= i0; AI(c, 2) += r0; AR(c, 3) += i1; AI(c, 3) -= r1;
      } else {
        AR(c, 2) += i0; AI(c, 2) -= r0; AR(c, 3) -= i1; AI(c, 3) += r1;
      }
    }
    return;
  }
  const R nf = -f;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const R r0 = r[4 * c], i0 = r[4 * c + 1], r1 = r[4 * c + 2], i1 = r[4 * c + 3];
    if (MU == 3) {
      if (DIR > 0) {
        AR(c, 2) = madd(f, r0, AR(c, 2)); AI(c, 2) = madd(f, i0, AI(c, 2));
        AR(c, 3) = madd(f, r1, AR(c, 3)); AI(c, 3) = madd(f, i1, AI(c, 3));
      } else {
        AR(c, 0) = madd(f, r0, AR(c, 0)); AI(c, 0) = madd(f, i0, AI(c, 0));
        AR(c, 1) = madd(f, r1, AR(c, 1)); AI(c, 1) = madd(f, i1, AI(c, 1));
      }
      continue;
    }
    AR(c, 0) = madd(f, r0, AR(c, 0)); AI(c, 0) = madd(f, i0, AI(c, 0));
    AR(c, 1) = madd(f, r1, AR(c, 1)); AI(c, 1) = madd(f, i1, AI(c, 1));
    if (MU == 0 && DIR > 0) {
      AR(c, 2) = madd(nf, i1, AR(c, 2)); AI(c, 2) = madd(f, r1, AI(c, 2));
      AR(c, 3) = madd(nf, i0, AR(c, 3)); AI(c, 3) = madd(f, r0, AI(c, 3));
    } else if (MU == 0) {
      AR(c, 2) = madd(f, i1, AR(c, 2)); AI(c, 2) = madd(nf, r1, AI(c, 2));
      AR(c, 3) = madd(f, i0, AR(c, 3)); AI(c, 3) = madd(nf, r0, AI(c, 3));
    } else if (MU == 1 && DIR > 0) {
      AR(c, 2) = madd(f, r1, AR(c, 2)); AI(c, 2) = madd(f, i1, AI(c, 2));
      AR(c, 3) = madd(nf, r0, AR(c, 3)); AI(c, 3) = madd(nf, i0, AI(c, 3));
    } else if (MU == 1) {
      AR(c, 2) = madd(nf, r1, AR(c, 2)); AI(c, 2) = madd(nf, i1, AI(c, 2));
      AR(c, 3) = madd(f, r0, AR(c, 3)); AI(c, 3) = madd(f, i0, AI(c, 3));
    } else if (MU == 2 && DIR > 0) {
      AR(c, 2) = madd(nf, i0, AR(c, 2)); AI(c, 2) = madd(f, r0, AI(c, 2));
      AR(c, 3) = madd(f, i1, AR(c, 3)); AI(c, 3) = madd(nf, r1, AI(c, 3));
    } else {
      AR(c, 2) = madd(f, i0, AR(c, 2)); AI(c, 2) = madd(nf, r0, AI(c, 2));
      AR(c, 3) = madd(nf, i1, AR(c, 3)); AI(c, 3) = madd(f, r1, AI(c, 3));
    }
  }
}
#undef AR
#undef AI

// v <- A^-1 v with the packed chiral clover (clover_def.h:88-284):
// x0 = (s0+s2, s1+s3), x1 = (s0-s2, s1-s3) per colour (no 1/2), y_i = A_i x_i,
// s0 = y0+y1, s2 = y0-y1 (colours 0..2), s1/s3 likewise from entries 3..5.
// V: the value type (the field's arithmetic type, or F2 for two lanes that
// share the site's clover).
// load_block(i, a) fills block i's 36 values for every lane of V.
template <typename V, typename Load>
__device__ __forceinline__ void clover_apply_with(Load&& load_block, V v[24]) {
  V xr[2][6], xi[2][6];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const V s0r = v[8 * c], s0i = v[8 * c + 1], s1r = v[8 * c + 2], s1i = v[8 * c + 3];
    const V s2r = v[8 * c + 4], s2i = v[8 * c + 5], s3r = v[8 * c + 6], s3i = v[8 * c + 7];
    xr[0][c] = s0r + s2r; xi[0][c] = s0i + s2i;
    xr[0][3 + c] = s1r + s3r; xi[0][3 + c] = s1i + s3i;
    xr[1][c] = s0r - s2r; xi[1][c] = s0i - s2i;
    xr[1][3 + c] = s1r - s3r; xi[1][3 + c] = s1i - s3i;
  }
  V yr[2][6], yi[2][6];
#pragma unroll
  for (int i = 0; i < 2; i++) {
    V a[36];
    load_block(i, a);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      yr[i][j] = a[j] * xr[i][j];
      yi[i][j] = a[j] * xi[i][j];
    }
    int n = 0;
#pragma unroll
    for (int j = 0; j < 6; j++)
#pragma unroll
      for (int k = j + 1; k < 6; k++, n++) {
        if constexpr (std::is_same<V, double>::value) {
          // FP64: left to the compiler's contraction (the explicit chain
          // below costs FP64 kernels ~80 registers)
          const double mr = a[6 + 2 * n], mi = a[7 + 2 * n];
          yr[i][j] += mr * xr[i][k] - mi * xi[i][k];
          yi[i][j] += mr * xi[i][k] + mi * xr[i][k];
          yr[i][k] += mr * xr[i][j] + mi * xi[i][j];
          yi[i][k] += mr * xi[i][j] - mi * xr[i][j];
          continue;
        }
        // y_j += M_jk x_k ; y_k += conj(M_jk) x_j; the minus signs on m_i
        // (negation is exact, so every form computes the same value)
        const V mr = a[6 + 2 * n], mi = a[7 + 2 * n];
        const V nmi = -a[7 + 2 * n];
        yr[i][j] = madd(mr, xr[i][k], yr[i][j]);
        yr[i][j] = madd(nmi, xi[i][k], yr[i][j]);
        yi[i][j] = madd(mr, xi[i][k], yi[i][j]);
        yi[i][j] = madd(mi, xr[i][k], yi[i][j]);
        yr[i][k] = madd(mr, xr[i][j], yr[i][k]);
        yr[i][k] = madd(mi, xi[i][j], yr[i][k]);
        yi[i][k] = madd(mr, xi[i][j], yi[i][k]);
        yi[i][k] = madd(nmi, xr[i][j], yi[i][k]);
      }
  }
#pragma unroll
  for (int c = 0; c < 3; c++) {
    v[8 * c + 0] = yr[0][c] + yr[1][c];
    v[8 * c + 1] = yi[0][c] + yi[1][c];
    v[8 * c + 4] = yr[0][c] - yr[1][c];
    v[8 * c + 5] = yi[0][c] - yi[1][c];
    v[8 * c + 2] = yr[0][3 + c] + yr[1][3 + c];
    v[8 * c + 3] = yi[0][3 + c] + yi[1][3 + c];
    v[8 * c + 6] = yr[0][3 + c] - yr[1][3 + c];
    v[8 * c + 7] = yi[0][3 + c] - yi[1][3 + c];
  }
}

// the clover of site g (or entry g of per-RHS clover planes) from field T's
// planes, the same for every lane of V
template <typename T, typename V = typename Arith<T>::R>
__device__ __forceinline__ void clover_apply(const typename Store<T>::type* __restrict__ C, int pad,
                                             int g, V v[24]) {
  using R = typename Arith<T>::R;
  clover_apply_with<V>(
      [&](int i, V a[36]) {
        R s[36];
        IO<T>::load_clover_block(C, pad, g, i, s);
#pragma unroll
        for (int k = 0; k < 36; k++) a[k] = Lanes<V>::bcast(s[k]);
      },
      v);
}

// FP32 links in 12-real form: the first two rows of U_mu (6 complex) as three
// float4 planes per direction; the third row of an SU(3) matrix is the
// complex conjugate of the cross product of the first two,
//   u_2b = conj(u_0,b+1 u_1,b+2 - u_0,b+2 u_1,b+1)   (indices mod 3).
__device__ __forceinline__ void load_link12(const float* __restrict__ U12, int pad, int mu, int g,
                                            float u[18]) {
  const float4* q = reinterpret_cast<const float4*>(U12);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const float4 t = __ldg(q + (size_t)(3 * mu + k) * pad + g);
    u[4 * k] = t.x;
    u[4 * k + 1] = t.y;
    u[4 * k + 2] = t.z;
    u[4 * k + 3] = t.w;
  }
#pragma unroll
  for (int b = 0; b < 3; b++) {
    const int b1 = (b + 1) % 3, b2 = (b + 2) % 3;
    const float ar = u[2 * b1], ai = u[2 * b1 + 1], br = u[6 + 2 * b2], bi = u[6 + 2 * b2 + 1];
    const float cr = u[2 * b2], ci = u[2 * b2 + 1], dr = u[6 + 2 * b1], di = u[6 + 2 * b1 + 1];
    const float re = (ar * br - ai * bi) - (cr * dr - ci * di);
    const float im = (ar * bi + ai * br) - (cr * di + ci * dr);
    u[12 + 2 * b] = re;
    u[12 + 2 * b + 1] = -im;
  }
}

// writers of one site's link (9 complex, row-major U_mu) and clover (72
// reals, QWS packing) into the device planes
template <typename R>
__device__ __forceinline__ void store_link(R* p, int pad, int mu, int g, const R u[18]);
template <>
__device__ __forceinline__ void store_link<float>(float* p, int pad, int mu, int g,
                                                  const float u[18]) {
  float2* q = reinterpret_cast<float2*>(p);
#pragma unroll
  for (int e = 0; e < 9; e++) q[(size_t)(mu * 9 + e) * pad + g] = make_float2(u[2 * e], u[2 * e + 1]);
}
template <>
__device__ __forceinline__ void store_link<double>(double* p, int pad, int mu, int g,
                                                   const double u[18]) {
  double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
  for (int e = 0; e < 9; e++)
    q[(size_t)(mu * 9 + e) * pad + g] = make_double2(u[2 * e], u[2 * e + 1]);
}

template <typename R>
__device__ __forceinline__ void store_clover(R* p, int pad, int g, const R a[72]);
template <>
__device__ __forceinline__ void store_clover<float>(float* p, int pad, int g, const float a[72]) {
  float4* q = reinterpret_cast<float4*>(p);
#pragma unroll
  for (int j = 0; j < 18; j++)
    q[(size_t)j * pad + g] = make_float4(a[4 * j], a[4 * j + 1], a[4 * j + 2], a[4 * j + 3]);
}
template <>
__device__ __forceinline__ void store_clover<double>(double* p, int pad, int g, const double a[72]) {
  double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
  for (int j = 0; j < 36; j++) q[(size_t)j * pad + g] = make_double2(a[2 * j], a[2 * j + 1]);
}

}  // namespace qwsg
