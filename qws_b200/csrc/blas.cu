// BLAS-1 kernels on spinor planes for the BiCGStab loops, with the dot
// products and norms fused into the update kernels that produce their inputs
// (bicgstab_precdd_s.cc:223-543, bicgstab_dd_mix.cc:140-368).
//
// Reductions: every thread accumulates in FP64, warps reduce with shuffles,
// each block writes one partial; the last block to finish (threadfence +
// counter) sums the partials in a fixed order with double-double (two-sum)
// arithmetic, so results are deterministic run to run and compensated.
#include "kernels.h"

namespace qwsg {

namespace {

constexpr int kThreads = 256;

template <typename R>
struct V4 {
  R x, y, z, w;
};

template <typename R>
__device__ __forceinline__ V4<R> ld4(const R* __restrict__ p, int pad, int g, int j);
template <>
__device__ __forceinline__ V4<float> ld4<float>(const float* __restrict__ p, int pad, int g, int j) {
  float4 t = reinterpret_cast<const float4*>(p)[(size_t)j * pad + g];
  return {t.x, t.y, t.z, t.w};
}
template <>
__device__ __forceinline__ V4<double> ld4<double>(const double* __restrict__ p, int pad, int g,
                                                  int j) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = q[(size_t)(2 * j) * pad + g], b = q[(size_t)(2 * j + 1) * pad + g];
  return {a.x, a.y, b.x, b.y};
}
template <typename R>
__device__ __forceinline__ void st4(R* p, int pad, int g, int j, V4<R> v);
template <>
__device__ __forceinline__ void st4<float>(float* p, int pad, int g, int j, V4<float> v) {
  reinterpret_cast<float4*>(p)[(size_t)j * pad + g] = make_float4(v.x, v.y, v.z, v.w);
}
template <>
__device__ __forceinline__ void st4<double>(double* p, int pad, int g, int j, V4<double> v) {
  double2* q = reinterpret_cast<double2*>(p);
  q[(size_t)(2 * j) * pad + g] = make_double2(v.x, v.y);
  q[(size_t)(2 * j + 1) * pad + g] = make_double2(v.z, v.w);
}

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  double bp = s - a;
  e = (a - (s - bp)) + (b - bp);
}

__device__ __forceinline__ void dd_add(double& hi, double& lo, double bhi, double blo) {
  double s, e;
  two_sum(hi, bhi, s, e);
  e += lo + blo;
  hi = s + e;
  lo = e - (hi - s);
}

// Per-RHS reductions.  The grid stride is a multiple of nr, so every thread
// only ever sees RHS r = (thread index) & (nr-1), and lanes l, l+nr, ... of a
// warp share one RHS: shuffles at offsets 16 .. nr leave the warp's sums in
// lanes 0..nr-1.  Block partials go to partial[(block*32 + r)*4 + k]; the last
// block to finish sums every (r, k) over the blocks in block order in
// double-double and writes res[r*4 + k].
template <int NR>
__device__ void finish_reduction(const double (&v)[8], int nr, const RedBuf& rb, double* res,
                                 int blk, int nblk) {
  __shared__ double sh[kThreads / 32][32][NR > 0 ? NR : 1];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NR; k++) {
    double x = v[k];
    for (int o = 16; o >= nr; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane < nr) sh[warp][lane][k] = x;
  }
  __syncthreads();
  if (threadIdx.x < nr) {
#pragma unroll
    for (int k = 0; k < NR; k++) {
      double x = 0;
      for (int w = 0; w < kThreads / 32; w++) x += sh[w][threadIdx.x][k];
      rb.partial[((size_t)blk * 32 + threadIdx.x) * 4 + k] = x;
    }
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned done = atomicAdd(rb.counter, 1u);
    last = (done == (unsigned)nblk - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int pr = warp; pr < nr * NR; pr += kThreads / 32) {
    const int r = pr / NR, k = pr - r * NR;
    double hi = 0, lo = 0;
    for (int b = lane; b < nblk; b += 32) {
      double x = *((volatile double*)&rb.partial[((size_t)b * 32 + r) * 4 + k]);
      dd_add(hi, lo, x, 0.0);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double h2 = __shfl_down_sync(0xffffffffu, hi, o);
      double l2 = __shfl_down_sync(0xffffffffu, lo, o);
      dd_add(hi, lo, h2, l2);
    }
    if (lane == 0) res[r * 4 + k] = hi + lo;
  }
  __syncthreads();
  if (threadIdx.x == 0) *rb.counter = 0;
}

// a per-RHS scalar: cf[r*4 + k] when a table is given, else the value
template <typename R>
__device__ __forceinline__ R coef(const double* cf, int r, int k, R v) {
  return cf ? (R)cf[r * 4 + k] : v;
}

// ---- per-site operations ---------------------------------------------------
// every (site, rhs) entry; op(G, entry, rhs, acc)
// block blk of nblk (grid stride nblk * kThreads)
template <int NR, typename Op>
__device__ __forceinline__ void sites_body(const Geom& G, const Op& op, const RedBuf& rb,
                                           double* res, int blk, int nblk) {
  double acc[8];
#pragma unroll
  for (int k = 0; k < 8; k++) acc[k] = 0;
  const int n = G.V << G.lgnr;
  for (int e = blk * kThreads + threadIdx.x; e < n; e += nblk * kThreads)
    op(G, e, e & (G.nr - 1), acc);
  if constexpr (NR > 0) finish_reduction<NR>(acc, G.nr, rb, res, blk, nblk);
}
template <typename R, int NR, typename Op>
__global__ void __launch_bounds__(kThreads) k_sites(Geom G, Op op, RedBuf rb, double* res) {
  sites_body<NR>(G, op, rb, res, blockIdx.x, gridDim.x);
}

// one launch over several lattices (group solves): each member runs the
// blocks of its own launch -- the same grid stride, partials and final sum,
// so its results are those of its own launch
template <typename Op>
struct SitesArgs {
  Geom G;
  Op op;
  RedBuf rb;
  double* res;
};
template <typename R, int NR, typename Op>
__global__ void __launch_bounds__(kThreads)
    k_sites_multi(const SitesArgs<Op>* __restrict__ args, const int* __restrict__ starts, int n) {
  __shared__ SitesArgs<Op> sa;
  const int l = group_member(starts, n, blockIdx.x);
  group_load_args(sa, args + l);
  sites_body<NR>(sa.G, sa.op, sa.rb, sa.res, blockIdx.x - starts[l], starts[l + 1] - starts[l]);
}

template <typename R>
struct OpNorm2 {
  const R* x;
  __device__ void operator()(const Geom& G, int g, int rhs, double* acc) const {
    const int sp = spad(G);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      V4<R> a = ld4(x, sp, g, j);
      acc[0] += (double)a.x * a.x + (double)a.y * a.y + (double)a.z * a.z + (double)a.w * a.w;
    }
  }
};

template <typename R>
struct OpCdot {
  const R *x, *y;
  __device__ void operator()(const Geom& G, int g, int rhs, double* acc) const {
    const int sp = spad(G);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      V4<R> a = ld4(x, sp, g, j), b = ld4(y, sp, g, j);
      acc[0] += (double)a.x * b.x + (double)a.y * b.y + (double)a.z * b.z + (double)a.w * b.w;
      acc[1] += (double)a.x * b.y - (double)a.y * b.x + (double)a.z * b.w - (double)a.w * b.z;
    }
  }
};

template <typename R>
struct OpNormCdot {  // |y|^2, <y, x>
  const R *y, *x;
  __device__ void operator()(const Geom& G, int g, int rhs, double* acc) const {
    const int sp = spad(G);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      V4<R> a = ld4(y, sp, g, j), b = ld4(x, sp, g, j);
      acc[0] += (double)a.x * a.x + (double)a.y * a.y + (double)a.z * a.z + (double)a.w * a.w;
      acc[1] += (double)a.x * b.x + (double)a.y * b.y + (double)a.z * b.z + (double)a.w * b.w;
      acc[2] += (double)a.x * b.y - (double)a.y * b.x + (double)a.z * b.w - (double)a.w * b.z;
    }
  }
};

// x += a p ; r -= a q ; |r|^2 (+ <r0, r> when r0 != nullptr)
template <typename R>
struct OpBicgUpdate {
  R *x, *r;
  const R *p, *q, *r0;
  R ar_, ai_;
  const double* cf;  // per-RHS (ar, ai) when set
  __device__ void operator()(const Geom& G, int g, int rhs, double* acc) const {
    const int sp = spad(G);
    const R ar = coef(cf, rhs, 0, ar_), ai = coef(cf, rhs, 1, ai_);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      V4<R> X = ld4<R>(x, sp, g, j), Rr = ld4<R>(r, sp, g, j);
      V4<R> P = ld4(p, sp, g, j), Q = ld4(q, sp, g, j);
      X.x = X.x + ar * P.x - ai * P.y;
      X.y = X.y + ar * P.y + ai * P.x;
      X.z = X.z + ar * P.z - ai * P.w;
      X.w = X.w + ar * P.w + ai * P.z;
      Rr.x = Rr.x - ar * Q.x + ai * Q.y;
      Rr.y = Rr.y - ar * Q.y - ai * Q.x;
      Rr.z = Rr.z - ar * Q.z + ai * Q.w;
      Rr.w = Rr.w - ar * Q.w - ai * Q.z;
      st4<R>(x, sp, g, j, X);
      st4<R>(r, sp, g, j, Rr);
      acc[0] += (double)Rr.x * Rr.x + (double)Rr.y * Rr.y + (double)Rr.z * Rr.z +
                (double)Rr.w * Rr.w;
      if (r0) {
        V4<R> A = ld4(r0, sp, g, j);
        acc[1] += (double)A.x * Rr.x + (double)A.y * Rr.y + (double)A.z * Rr.z + (double)A.w * Rr.w;
        acc[2] += (double)A.x * Rr.y - (double)A.y * Rr.x + (double)A.z * Rr.w - (double)A.w * Rr.z;
      }
    }
  }
};

// p = r + b (p - w q)   (bicgstab_precdd_s.cc:528-543)
template <typename R>
struct OpBicgP {
  R* p;
  const R *r, *q;
  R br_, bi_, wr_, wi_;
  const double* cf;  // per-RHS (br, bi, wr, wi) when set
  __device__ void operator()(const Geom& G, int g, int rhs, double*) const {
    const int sp = spad(G);
    const R br = coef(cf, rhs, 0, br_), bi = coef(cf, rhs, 1, bi_);
    const R wr = coef(cf, rhs, 2, wr_), wi = coef(cf, rhs, 3, wi_);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      V4<R> P = ld4<R>(p, sp, g, j), Rr = ld4(r, sp, g, j), Q = ld4(q, sp, g, j);
      R c0 = P.x - wr * Q.x + wi * Q.y, c1 = P.y - wr * Q.y - wi * Q.x;
      R c2 = P.z - wr * Q.z + wi * Q.w, c3 = P.w - wr * Q.w - wi * Q.z;
      P.x = br * c0 - bi * c1 + Rr.x;
      P.y = br * c1 + bi * c0 + Rr.y;
      P.z = br * c2 - bi * c3 + Rr.z;
      P.w = br * c3 + bi * c2 + Rr.w;
      st4<R>(p, sp, g, j, P);
    }
  }
};

// r = b - q ; p = r ; r0 = r ; |b|^2 ; |r|^2  (bicgstab_dd_mix.cc:140-152)
template <typename R>
struct OpBicgInit {
  const R *b, *q;
  R *r, *p, *r0;
  __device__ void operator()(const Geom& G, int g, int rhs, double* acc) const {
    const int sp = spad(G);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      V4<R> B = ld4(b, sp, g, j), Q;
      if (q)
        Q = ld4(q, sp, g, j);
      else
        Q = {0, 0, 0, 0};
      V4<R> Rr = {B.x - Q.x, B.y - Q.y, B.z - Q.z, B.w - Q.w};
      st4<R>(r, sp, g, j, Rr);
      st4<R>(p, sp, g, j, Rr);
      st4<R>(r0, sp, g, j, Rr);
      acc[0] += (double)B.x * B.x + (double)B.y * B.y + (double)B.z * B.z + (double)B.w * B.w;
      acc[1] += (double)Rr.x * Rr.x + (double)Rr.y * Rr.y + (double)Rr.z * Rr.z +
                (double)Rr.w * Rr.w;
    }
  }
};

// r += a q ; |r|^2
template <typename R>
struct OpAxpyNorm {
  R* r;
  const R* q;
  R a;
  __device__ void operator()(const Geom& G, int g, int, double* acc) const {
    const int sp = spad(G);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      V4<R> Rr = ld4<R>(r, sp, g, j), Q = ld4(q, sp, g, j);
      Rr.x += a * Q.x;
      Rr.y += a * Q.y;
      Rr.z += a * Q.z;
      Rr.w += a * Q.w;
      st4<R>(r, sp, g, j, Rr);
      acc[0] += (double)Rr.x * Rr.x + (double)Rr.y * Rr.y + (double)Rr.z * Rr.z +
                (double)Rr.w * Rr.w;
    }
  }
};

// the shift updates of one multi-shift CG iteration, all shifts in one pass
// over the sites: r and p are read once per site, each shift's x_k and pp_k
// once (single RHS: g is the site)
struct OpMshift {
  double *x, *pp, *p;
  const double* r;
  const double* cf;
  size_t stride;
  int n;
  double beta;
  bool update;
  __device__ void operator()(const Geom& G, int g, int, double*) const {
    const int sp = spad(G);
    for (int j = 0; j < 6; j++) {
      const V4<double> Rr = ld4<double>(r, sp, g, j);
      for (int k = 0; k < n; k++) {
        if (__ldg(cf + 4 * k + 3) == 0.0) continue;  // converged shift
        const double c = __ldg(cf + 4 * k), z = __ldg(cf + 4 * k + 1), d = __ldg(cf + 4 * k + 2);
        double* xk = x + k * stride;
        double* pk = pp + k * stride;
        V4<double> X = ld4<double>(xk, sp, g, j), P = ld4<double>(pk, sp, g, j);
        X.x -= c * P.x;
        X.y -= c * P.y;
        X.z -= c * P.z;
        X.w -= c * P.w;
        st4<double>(xk, sp, g, j, X);
        if (update)
          st4<double>(pk, sp, g, j,
                      {z * Rr.x + d * P.x, z * Rr.y + d * P.y, z * Rr.z + d * P.z,
                       z * Rr.w + d * P.w});
      }
      if (update) {
        V4<double> P = ld4<double>(p, sp, g, j);
        st4<double>(p, sp, g, j,
                    {Rr.x + beta * P.x, Rr.y + beta * P.y, Rr.z + beta * P.z, Rr.w + beta * P.w});
      }
    }
  }
};

struct OpD2S {
  float* y;
  const double* x;
  double s_;
  const double* cf;  // per-RHS scale when set
  __device__ void operator()(const Geom& G, int g, int rhs, double*) const {
    const int sp = spad(G);
    const double s = coef(cf, rhs, 0, s_);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      V4<double> a = ld4(x, sp, g, j);
      st4<float>(y, sp, g, j,
                 {(float)(a.x * s), (float)(a.y * s), (float)(a.z * s), (float)(a.w * s)});
    }
  }
};

struct OpS2D {
  double* y;
  const float* x;
  double s_;
  const double* cf;  // per-RHS scale when set
  __device__ void operator()(const Geom& G, int g, int rhs, double*) const {
    const int sp = spad(G);
    const double s = coef(cf, rhs, 0, s_);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      V4<float> a = ld4(x, sp, g, j);
      st4<double>(y, sp, g, j,
                  {(double)a.x * s, (double)a.y * s, (double)a.z * s, (double)a.w * s});
    }
  }
};

// complex float arithmetic of the inner loop's scalars, each product and
// sum rounded on its own (no contraction), as the host loop computes them;
// the quotient is formed in FP64 and rounded once
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                     __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 cdivf(float2 a, float2 b) {
  const double den = (double)b.x * b.x + (double)b.y * b.y;
  return make_float2((float)(((double)a.x * b.x + (double)a.y * b.y) / den),
                     (float)(((double)a.y * b.x - (double)a.x * b.y) / den));
}
__device__ __forceinline__ float cabsf2(float2 a) { return hypotf(a.x, a.y); }

__device__ void inner_scalars_body(InnerScalars* s, const double* __restrict__ res, int phase,
                                   double tol) {
  const bool done = s->done != 0;
  switch (phase) {
    case 0: {
      const float bn = (float)res[0];
      s->bnorm = bn;
      s->rnorm = bn;
      s->rho0r = bn;
      s->rho0i = 0;
      s->done = bn == 0;
      s->iters = 0;
      s->bad = 0;
      s->iter = 0;
      for (int k = 0; k < 12; k++) s->cf[k] = 0;
      break;
    }
    case 1: {  // alpha = rho0 / <r0, q>, zero when |<r0, q>| <= 1e-15
      float2 a = make_float2(0, 0);
      if (!done) {
        const float2 ct = make_float2((float)res[0], (float)res[1]);
        a = cdivf(make_float2(s->rho0r, s->rho0i), ct);
        if (cabsf2(ct) <= 1e-15f) a = make_float2(0, 0);
      }
      s->ar = a.x;
      s->ai = a.y;
      s->cf[0] = a.x;
      s->cf[1] = a.y;
      break;
    }
    case 2:
    case 4: {
      float2 beta = make_float2(0, 0), w = make_float2(0, 0);
      if (!done) {
        const float rn = (float)res[0];
        s->rnorm = rn;
        if (!isfinite(rn)) {
          s->bad = 1;
          s->done = 1;
        } else if ((double)sqrtf(rn / s->bnorm) < tol) {
          s->done = 1;
          s->iters = s->iter + 1;
        } else if (phase == 4) {  // beta = alpha rho / (rho0 omega); rho0 = rho
          const float2 rho = make_float2((float)res[1], (float)res[2]);
          w = make_float2(s->wr, s->wi);
          beta = cdivf(cmulf(make_float2(s->ar, s->ai), rho),
                       cmulf(make_float2(s->rho0r, s->rho0i), w));
          s->rho0r = rho.x;
          s->rho0i = rho.y;
          if (cabsf2(w) == 0 || cabsf2(rho) == 0) beta = make_float2(0, 0);
        }
      }
      if (phase == 4) {
        s->cf[8] = beta.x;
        s->cf[9] = beta.y;
        s->cf[10] = w.x;
        s->cf[11] = w.y;
        s->iter++;
      }
      break;
    }
    case 3: {  // omega = <t, r> / |t|^2, zero when |t|^2 <= 1e-30
      float2 w = make_float2(0, 0);
      if (!done) {
        const float r0 = (float)res[0], r1 = (float)res[1], r2 = (float)res[2];
        w = make_float2(r1 / r0, r2 / r0);
        if (r0 <= 1e-30f) w = make_float2(0, 0);
      }
      s->wr = w.x;
      s->wi = w.y;
      s->cf[4] = w.x;
      s->cf[5] = w.y;
      break;
    }
  }
}

__global__ void k_inner_scalars(InnerScalars* s, const double* __restrict__ res, int phase,
                                double tol) {
  inner_scalars_body(s, res, phase, tol);
}
struct InnerScalarsArgs {
  InnerScalars* s;
  const double* res;
  double tol;
  int phase;
  int pad_;
};
__global__ void k_inner_scalars_multi(const InnerScalarsArgs* __restrict__ a, int n) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l < n) inner_scalars_body(a[l].s, a[l].res, a[l].phase, a[l].tol);
}

int grid_for(const Geom& G, const RedBuf* rb) {
  int b = ((G.V << G.lgnr) + kThreads - 1) / kThreads;
  int cap = rb ? rb->nblk : 148 * 8;
  return b < cap ? b : cap;
}

// merge one per-site launch of each group member (each with the block
// count of its own launch)
template <typename R, int NR, typename Op>
void merge_sites(const GroupRec* const* recs, int n, GroupBatch& b) {
  std::vector<SitesArgs<Op>> args(n);
  std::vector<int> starts(n + 1);
  int blocks = 0;
  for (int l = 0; l < n; l++) {
    args[l] = group_arg<SitesArgs<Op>>(recs[l]);
    starts[l] = blocks;
    blocks += grid_for(args[l].G, args[l].rb.partial ? &args[l].rb : nullptr);
  }
  starts[n] = blocks;
  const size_t oa = b.put(args.data(), sizeof(SitesArgs<Op>) * n), os = b.put_starts(starts);
  b.launches.push_back([=](const unsigned char* dev, cudaStream_t st) {
    count_launch();
    k_sites_multi<R, NR, Op><<<blocks, kThreads, 0, st>>>(
        reinterpret_cast<const SitesArgs<Op>*>(dev + oa), reinterpret_cast<const int*>(dev + os),
        n);
  });
}

template <typename R, int NR, typename Op>
void run(const Geom& G, Op op, RedBuf* rb, double* res, cudaStream_t st) {
  RedBuf dummy{nullptr, nullptr, 0};
  if (g_group_rec) {
    if (G.nr != 1) group_unrecorded_launch();
    group_record(&merge_sites<R, NR, Op>, SitesArgs<Op>{G, op, rb ? *rb : dummy, res});
    return;
  }
  count_launch();
  k_sites<R, NR, Op><<<grid_for(G, rb), kThreads, 0, st>>>(G, op, rb ? *rb : dummy, res);
}

// entries [e0, e0 + n) (all RHS of the sites [site0, site0 + n/nr))
template <typename R>
__global__ void k_copy(Geom G, R* y, const R* x, int e0, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int e = e0 + i, sp = spad(G);
#pragma unroll
  for (int j = 0; j < 6; j++) st4<R>(y, sp, e, j, ld4<R>(x, sp, e, j));
}
template <typename R>
__global__ void k_zero(Geom G, R* y, int e0, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int e = e0 + i, sp = spad(G);
#pragma unroll
  for (int j = 0; j < 6; j++) st4<R>(y, sp, e, j, {0, 0, 0, 0});
}

// copy (x set) or zero (x null) of entries [e0, e0 + n) for several lattices
template <typename R>
struct CopyArgs {
  Geom G;
  R* y;
  const R* x;
  int e0, n;
};
template <typename R>
__global__ void k_copy_multi(const CopyArgs<R>* __restrict__ args, const int* __restrict__ starts,
                             int n) {
  __shared__ CopyArgs<R> sa;
  const int l = group_member(starts, n, blockIdx.x);
  group_load_args(sa, args + l);
  const int i = (blockIdx.x - starts[l]) * blockDim.x + threadIdx.x;
  if (i >= sa.n) return;
  const int e = sa.e0 + i, sp = spad(sa.G);
  if (sa.x) {
#pragma unroll
    for (int j = 0; j < 6; j++) st4<R>(sa.y, sp, e, j, ld4<R>(sa.x, sp, e, j));
  } else {
#pragma unroll
    for (int j = 0; j < 6; j++) st4<R>(sa.y, sp, e, j, {0, 0, 0, 0});
  }
}
template <typename R>
void merge_copy(const GroupRec* const* recs, int n, GroupBatch& b) {
  std::vector<CopyArgs<R>> args(n);
  std::vector<int> starts(n + 1);
  int blocks = 0;
  for (int l = 0; l < n; l++) {
    args[l] = group_arg<CopyArgs<R>>(recs[l]);
    starts[l] = blocks;
    blocks += (args[l].n + 255) / 256;
  }
  starts[n] = blocks;
  if (blocks == 0) return;
  const size_t oa = b.put(args.data(), sizeof(CopyArgs<R>) * n), os = b.put_starts(starts);
  b.launches.push_back([=](const unsigned char* dev, cudaStream_t st) {
    count_launch();
    k_copy_multi<R><<<blocks, 256, 0, st>>>(reinterpret_cast<const CopyArgs<R>*>(dev + oa),
                                            reinterpret_cast<const int*>(dev + os), n);
  });
}
void merge_inner_scalars(const GroupRec* const* recs, int n, GroupBatch& b) {
  std::vector<InnerScalarsArgs> args(n);
  for (int l = 0; l < n; l++) args[l] = group_arg<InnerScalarsArgs>(recs[l]);
  const size_t oa = b.put(args.data(), sizeof(InnerScalarsArgs) * n);
  b.launches.push_back([=](const unsigned char* dev, cudaStream_t st) {
    count_launch();
    k_inner_scalars_multi<<<(n + 31) / 32, 32, 0, st>>>(
        reinterpret_cast<const InnerScalarsArgs*>(dev + oa), n);
  });
}

}  // namespace

template <typename R>
void blas_copy(const Geom& G, R* y, const R* x, int site0, int n, cudaStream_t st) {
  const int ne = n << G.lgnr;
  if (group_record(&merge_copy<R>, CopyArgs<R>{G, y, x, site0 << G.lgnr, ne})) return;
  if (ne > 0) {
    count_launch();
    k_copy<R><<<(ne + 255) / 256, 256, 0, st>>>(G, y, x, site0 << G.lgnr, ne);
  }
}
template <typename R>
void blas_zero(const Geom& G, R* y, int site0, int n, cudaStream_t st) {
  const int ne = n << G.lgnr;
  if (group_record(&merge_copy<R>, CopyArgs<R>{G, y, nullptr, site0 << G.lgnr, ne})) return;
  if (ne > 0) {
    count_launch();
    k_zero<R><<<(ne + 255) / 256, 256, 0, st>>>(G, y, site0 << G.lgnr, ne);
  }
}
template <typename R>
void blas_norm2(const Geom& G, const R* x, double* res, RedBuf& rb, cudaStream_t st) {
  run<R, 1>(G, OpNorm2<R>{x}, &rb, res, st);
}
template <typename R>
void blas_cdot(const Geom& G, const R* x, const R* y, double* res, RedBuf& rb, cudaStream_t st) {
  run<R, 2>(G, OpCdot<R>{x, y}, &rb, res, st);
}
template <typename R>
void blas_norm_cdot(const Geom& G, const R* y, const R* x, double* res, RedBuf& rb,
                    cudaStream_t st) {
  run<R, 3>(G, OpNormCdot<R>{y, x}, &rb, res, st);
}
template <typename R>
void blas_bicg_update(const Geom& G, R* x, R* r, const R* p, const R* q, double ar, double ai,
                      const R* r0, double* res, RedBuf& rb, cudaStream_t st, const double* cf) {
  OpBicgUpdate<R> op{x, r, p, q, r0, (R)ar, (R)ai, cf};
  if (r0)
    run<R, 3>(G, op, &rb, res, st);
  else
    run<R, 1>(G, op, &rb, res, st);
}
template <typename R>
void blas_bicg_p(const Geom& G, R* p, const R* r, const R* q, double br, double bi, double wr,
                 double wi, cudaStream_t st, const double* cf) {
  run<R, 0>(G, OpBicgP<R>{p, r, q, (R)br, (R)bi, (R)wr, (R)wi, cf}, nullptr, nullptr, st);
}
template <typename R>
void blas_bicg_init(const Geom& G, const R* b, const R* q, R* r, R* p, R* r0, double* res,
                    RedBuf& rb, cudaStream_t st) {
  run<R, 2>(G, OpBicgInit<R>{b, q, r, p, r0}, &rb, res, st);
}
template <typename R>
void blas_axpy_norm(const Geom& G, R* r, const R* q, double a, double* res, RedBuf& rb,
                    cudaStream_t st) {
  run<R, 1>(G, OpAxpyNorm<R>{r, q, (R)a}, &rb, res, st);
}
void blas_mshift(const Geom& G, double* x, double* pp, int n, const double* r, double* p,
                 double beta, const double* cf, bool update, cudaStream_t st) {
  OpMshift op{x, pp, p, r, cf, (size_t)24 * spad(G), n, beta, update};
  run<double, 0>(G, op, nullptr, nullptr, st);
}
void blas_d2s(const Geom& G, float* y, const double* x, double s, cudaStream_t st,
              const double* cf) {
  run<float, 0>(G, OpD2S{y, x, s, cf}, nullptr, nullptr, st);
}
void blas_s2d(const Geom& G, double* y, const float* x, double s, cudaStream_t st,
              const double* cf) {
  run<float, 0>(G, OpS2D{y, x, s, cf}, nullptr, nullptr, st);
}

void inner_scalars(InnerScalars* s, const double* res, int phase, double tol, cudaStream_t st) {
  if (group_record(&merge_inner_scalars, InnerScalarsArgs{s, res, tol, phase, 0})) return;
  count_launch();
  k_inner_scalars<<<1, 1, 0, st>>>(s, res, phase, tol);
}

#define QWSG_INST(R)                                                                         \
  template void blas_copy<R>(const Geom&, R*, const R*, int, int, cudaStream_t);             \
  template void blas_zero<R>(const Geom&, R*, int, int, cudaStream_t);                       \
  template void blas_norm2<R>(const Geom&, const R*, double*, RedBuf&, cudaStream_t);        \
  template void blas_cdot<R>(const Geom&, const R*, const R*, double*, RedBuf&, cudaStream_t); \
  template void blas_norm_cdot<R>(const Geom&, const R*, const R*, double*, RedBuf&,         \
                                  cudaStream_t);                                             \
  template void blas_bicg_update<R>(const Geom&, R*, R*, const R*, const R*, double, double, \
                                    const R*, double*, RedBuf&, cudaStream_t, const double*); \
  template void blas_bicg_p<R>(const Geom&, R*, const R*, const R*, double, double, double,  \
                               double, cudaStream_t, const double*);                         \
  template void blas_bicg_init<R>(const Geom&, const R*, const R*, R*, R*, R*, double*,      \
                                  RedBuf&, cudaStream_t);                                    \
  template void blas_axpy_norm<R>(const Geom&, R*, const R*, double, double*, RedBuf&,        \
                                  cudaStream_t);
QWSG_INST(float)
QWSG_INST(double)
#undef QWSG_INST

}  // namespace qwsg
