// Seeded synthetic gauge field generated on the device, straight into the
// resident DD-order planes (FP64 and FP32).  Same construction and random
// streams as the host generator (fields.cu: SplitMix64 keyed by (seed,
// natural site, mu), Box-Muller, Gram-Schmidt + determinant phase, APE-style
// smoothing U' = Proj[(1-alpha) U + alpha/6 * staples]); the transcendental
// functions are CUDA's, so the fields agree with the host's to rounding.
// No counterpart in the reference, which loads gauge fields from BQCD.
#include <cmath>

#include "ctx.h"

namespace qwsg {
namespace {

struct Cx {
  double r, i;
};
__device__ __forceinline__ Cx cmul(Cx a, Cx b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
__device__ __forceinline__ Cx cadd(Cx a, Cx b) { return {a.r + b.r, a.i + b.i}; }
__device__ __forceinline__ Cx csub(Cx a, Cx b) { return {a.r - b.r, a.i - b.i}; }
__device__ __forceinline__ Cx conj(Cx a) { return {a.r, -a.i}; }

struct Mat {
  Cx a[3][3];
};

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

struct Rng {
  unsigned long long state;
  __device__ Rng(unsigned long long seed, unsigned long long a, unsigned long long b)
      : state(splitmix64(seed ^ splitmix64(a * 0x100000001b3ull + b * 0x9e3779b97f4a7c15ull))) {}
  __device__ double uniform() {  // (0, 1]
    state += 0x9e3779b97f4a7c15ull;
    unsigned long long z = splitmix64(state);
    return ((z >> 11) + 1) * (1.0 / 9007199254740992.0);
  }
  __device__ Cx gauss() {  // unit-variance complex Gaussian
    double r = sqrt(-log(uniform()));
    double t = 2 * M_PI * uniform();
    return {r * cos(t), r * sin(t)};
  }
};

// Gram-Schmidt on the rows, then the determinant phase divided out
__device__ void project_su3(Mat& m) {
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < i; j++) {
      Cx p = {0, 0};
      for (int k = 0; k < 3; k++) p = cadd(p, cmul(conj(m.a[j][k]), m.a[i][k]));
      for (int k = 0; k < 3; k++) m.a[i][k] = csub(m.a[i][k], cmul(p, m.a[j][k]));
    }
    double n = 0;
    for (int k = 0; k < 3; k++) n += m.a[i][k].r * m.a[i][k].r + m.a[i][k].i * m.a[i][k].i;
    n = 1.0 / sqrt(n);
    for (int k = 0; k < 3; k++) m.a[i][k] = {m.a[i][k].r * n, m.a[i][k].i * n};
  }
  const auto& a = m.a;
  Cx d = csub(cmul(a[0][0], csub(cmul(a[1][1], a[2][2]), cmul(a[1][2], a[2][1]))),
              cmul(a[0][1], csub(cmul(a[1][0], a[2][2]), cmul(a[1][2], a[2][0]))));
  d = cadd(d, cmul(a[0][2], csub(cmul(a[1][0], a[2][1]), cmul(a[1][1], a[2][0]))));
  const double ph = -atan2(d.i, d.r) / 3.0;
  const Cx f = {cos(ph), sin(ph)};
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++) m.a[i][k] = cmul(m.a[i][k], f);
}

__device__ void load(const double* U, int pad, int mu, int g, Mat& m) {
  const double2* q = reinterpret_cast<const double2*>(U);
  for (int e = 0; e < 9; e++) {
    double2 t = q[(size_t)(mu * 9 + e) * pad + g];
    m.a[e / 3][e % 3] = {t.x, t.y};
  }
}
__device__ void store(double* U, int pad, int mu, int g, const Mat& m) {
  double2* q = reinterpret_cast<double2*>(U);
  for (int e = 0; e < 9; e++)
    q[(size_t)(mu * 9 + e) * pad + g] = make_double2(m.a[e / 3][e % 3].r, m.a[e / 3][e % 3].i);
}

template <bool DA, bool DB>
__device__ void mul(const Mat& a, const Mat& b, Mat& c) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      Cx s = {0, 0};
      for (int k = 0; k < 3; k++) {
        Cx x = DA ? conj(a.a[k][i]) : a.a[i][k];
        Cx y = DB ? conj(b.a[j][k]) : b.a[k][j];
        s = cadd(s, cmul(x, y));
      }
      c.a[i][j] = s;
    }
}

__device__ int shifted(const Geom& G, const int x[4], int mu, int d, int nu, int e) {
  int y[4] = {x[0], x[1], x[2], x[3]};
  y[mu] = (y[mu] + d + G.L[mu]) % G.L[mu];
  if (e) y[nu] = (y[nu] + e + G.L[nu]) % G.L[nu];
  return dd_index(G, y);
}

__device__ long natural(const Geom& G, const int x[4]) {
  return x[0] + (long)G.L[0] * (x[1] + (long)G.L[1] * (x[2] + (long)G.L[2] * x[3]));
}

// one thread per (site, mu): thread i handles site i / 4, direction i % 4
__global__ void k_random_su3(Geom G, double* U, unsigned long long seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 4 * G.V) return;
  const int g = i >> 2, mu = i & 3;
  int x[4];
  site_coords(G, g, x);
  Rng r(seed, (unsigned long long)natural(G, x), (unsigned long long)mu);
  Mat m;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) m.a[a][b] = r.gauss();
  project_su3(m);
  store(U, G.pad, mu, g, m);
}

// W_mu(x) = Proj[(1-alpha) U_mu(x) + alpha/6 sum_nu staples], staples in the
// host generator's order
__global__ void k_ape(Geom G, const double* __restrict__ U, double* W, double alpha) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 4 * G.V) return;
  const int g = i >> 2, mu = i & 3;
  int x[4];
  site_coords(G, g, x);
  Mat S;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) S.a[a][b] = {0, 0};
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    const int sp_mu = shifted(G, x, mu, 1, nu, 0), sp_nu = shifted(G, x, nu, 1, mu, 0);
    const int sm_nu = shifted(G, x, nu, -1, mu, 0), sm_nu_p_mu = shifted(G, x, nu, -1, mu, 1);
    Mat A, B, C, P, Q;
    // U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag
    load(U, G.pad, nu, g, A);
    load(U, G.pad, mu, sp_nu, B);
    load(U, G.pad, nu, sp_mu, C);
    mul<false, false>(A, B, P);
    mul<false, true>(P, C, Q);
    // U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu)
    load(U, G.pad, nu, sm_nu, A);
    load(U, G.pad, mu, sm_nu, B);
    load(U, G.pad, nu, sm_nu_p_mu, C);
    mul<true, false>(A, B, P);
    mul<false, false>(P, C, A);
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) S.a[a][b] = cadd(S.a[a][b], cadd(Q.a[a][b], A.a[a][b]));
  }
  Mat o;
  load(U, G.pad, mu, g, o);
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++)
      o.a[a][b] = {(1 - alpha) * o.a[a][b].r + (alpha / 6.0) * S.a[a][b].r,
                   (1 - alpha) * o.a[a][b].i + (alpha / 6.0) * S.a[a][b].i};
  project_su3(o);
  store(W, G.pad, mu, g, o);
}

// per-block partial sums of Re tr(plaquette)/3 over the six planes
__global__ void k_plaquette(Geom G, const double* __restrict__ U, double* partial) {
  __shared__ double sh[128];
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0;
  if (g < G.V) {
    int x[4];
    site_coords(G, g, x);
    for (int mu = 0; mu < 4; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        Mat A, B, C, D, P, Q, R;
        load(U, G.pad, mu, g, A);
        load(U, G.pad, nu, shifted(G, x, mu, 1, nu, 0), B);
        load(U, G.pad, mu, shifted(G, x, nu, 1, mu, 0), C);
        load(U, G.pad, nu, g, D);
        mul<false, false>(A, B, P);
        mul<true, true>(C, D, Q);
        mul<false, false>(P, Q, R);
        v += (R.a[0][0].r + R.a[1][1].r + R.a[2][2].r) / 3.0;
      }
  }
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = 64; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__global__ void k_d2f_planes(const double* __restrict__ a, float* b, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

}  // namespace

// gauge field on the device; returns the plaquette
double gen_gauge_device(Ctx& c, unsigned long long seed, int n_smear, double alpha) {
  if (c.parent) throw Error(1, "generate the gauge field on the parent lattice");
  c.ensure_fields_d();
  c.ensure_fields_s();
  const Geom& G = c.G;
  const size_t n = (size_t)72 * G.pad;
  // the smearing steps ping-pong between the link planes and the FP64
  // clover planes (the same size; the clover term of the new field is
  // built, or loaded, afterwards), so a field of any size needs no scratch
  const int nb = (4 * G.V + 127) / 128;
  double* cur = c.Ud;
  double* nxt = c.Cd;
  count_launch();
  k_random_su3<<<nb, 128, 0, c.st>>>(G, cur, seed);
  for (int it = 0; it < n_smear; it++) {
    count_launch();
    k_ape<<<nb, 128, 0, c.st>>>(G, cur, nxt, alpha);
    double* t = cur;
    cur = nxt;
    nxt = t;
  }
  if (cur != c.Ud)
    QWSG_CUDA(cudaMemcpyAsync(c.Ud, cur, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.st));
  count_launch();
  k_d2f_planes<<<(unsigned)((n + 255) / 256), 256, 0, c.st>>>(c.Ud, c.Us, n);
  const int pb = (G.V + 127) / 128;
  double* part = nullptr;  // stream-ordered: no device-wide synchronisation
  QWSG_CUDA(cudaMallocAsync(&part, sizeof(double) * pb, c.st));
  count_launch();
  k_plaquette<<<pb, 128, 0, c.st>>>(G, c.Ud, part);
  c.check_launch("gen_gauge_device");
  std::vector<double> h(pb);
  QWSG_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double) * pb, cudaMemcpyDeviceToHost, c.st));
  QWSG_CUDA(cudaFreeAsync(part, c.st));
  QWSG_CUDA(cudaStreamSynchronize(c.st));
  c.fields_h_valid = false;
  double tot = 0;
  for (double v : h) tot += v;
  return tot / (6.0 * G.V);
}

}  // namespace qwsg
