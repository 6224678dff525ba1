// On-device clover term: the clover-leaf field strength of the resident FP64
// gauge field and the packed inverse chiral blocks the DD kernels read.
//
// No counterpart in the reference: QWS loads a clover term that BQCD built
// and inverted (qws_bqcd.cc:284-382).  The conventions are those of the host
// generator (fields.cu), so the two agree to rounding:
//   F_{mu nu} = (Q - Q^dag) / (8i), traceless, Q the four-leaf sum;
//   T = 1 - csw*kappa * sum_{mu<nu} sigma_{mu nu} F_{mu nu};
//   stored: the two 6x6 chiral blocks M_i = (P T P^T / 2)_i^-1 / 2 in the
//   reference's packing (clover_def.h:88-284, diagonal then pairs j<k).
// In the chiral basis sigma_{mu nu} is block diagonal, so each block is built
// directly: (P T P^T / 2)_i = 1 - csw*kappa * sum S_{mu nu,i} (x) F_{mu nu},
// S the 2x2 spin tables of clover_chiral_tables().  One thread per site;
// Gauss-Jordan inversion with partial pivoting, as on the host.
#include <cmath>

#include <type_traits>

#include "ctx.h"

namespace qwsg {

double clover_chiral_tables(double S[6][2][2][2][2]);

namespace {

struct Cx {
  double r, i;
};
__device__ __forceinline__ Cx cmul(Cx a, Cx b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
__device__ __forceinline__ Cx cadd(Cx a, Cx b) { return {a.r + b.r, a.i + b.i}; }
__device__ __forceinline__ Cx csub(Cx a, Cx b) { return {a.r - b.r, a.i - b.i}; }
__device__ __forceinline__ Cx conj(Cx a) { return {a.r, -a.i}; }
__device__ __forceinline__ double cabs2(Cx a) { return a.r * a.r + a.i * a.i; }

struct Mat {
  Cx a[3][3];
};

__constant__ double c_S[6][2][2][2][2];

__device__ void load_link(const double* U, int pad, int mu, int g, Mat& m) {
  const double2* q = reinterpret_cast<const double2*>(U);
#pragma unroll
  for (int e = 0; e < 9; e++) {
    double2 t = q[(size_t)(mu * 9 + e) * pad + g];
    m.a[e / 3][e % 3] = {t.x, t.y};
  }
}

// c = op(a) op(b), op = identity or Hermitian conjugate
template <bool DA, bool DB>
__device__ void mul(const Mat& a, const Mat& b, Mat& c) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      Cx s = {0, 0};
#pragma unroll
      for (int k = 0; k < 3; k++) {
        Cx x = DA ? conj(a.a[k][i]) : a.a[i][k];
        Cx y = DB ? conj(b.a[j][k]) : b.a[k][j];
        s = cadd(s, cmul(x, y));
      }
      c.a[i][j] = s;
    }
}

__device__ void accumulate(Mat& Q, const Mat& q) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) Q.a[i][j] = cadd(Q.a[i][j], q.a[i][j]);
}

__device__ int shifted(const Geom& G, const int x[4], int mu, int d, int nu, int e) {
  int y[4] = {x[0], x[1], x[2], x[3]};
  y[mu] = (y[mu] + d + G.L[mu]) % G.L[mu];
  if (e) y[nu] = (y[nu] + e + G.L[nu]) % G.L[nu];
  return dd_index(G, y);
}

// the four-leaf sum Q_{mu nu}(x), products in the host generator's order
__device__ void leaf_sum(const Geom& G, const double* U, const int x[4], int g, int mu, int nu,
                         Mat& Q) {
  const int xpm = shifted(G, x, mu, 1, nu, 0), xpn = shifted(G, x, nu, 1, mu, 0);
  const int xmm = shifted(G, x, mu, -1, nu, 0), xmn = shifted(G, x, nu, -1, mu, 0);
  const int xmm_pn = shifted(G, x, mu, -1, nu, 1), xmm_mn = shifted(G, x, mu, -1, nu, -1);
  const int xmn_pm = shifted(G, x, nu, -1, mu, 1);
  Mat A, B, C, D, P1, P2, q;
  // q1 = (U_mu(x) U_nu(x+mu)) (U_mu(x+nu)^dag U_nu(x)^dag)
  load_link(U, G.pad, mu, g, A);
  load_link(U, G.pad, nu, xpm, B);
  load_link(U, G.pad, mu, xpn, C);
  load_link(U, G.pad, nu, g, D);
  mul<false, false>(A, B, P1);
  mul<true, true>(C, D, P2);
  mul<false, false>(P1, P2, Q);
  // q2 = (U_nu(x) U_mu(x-mu+nu)^dag) (U_nu(x-mu)^dag U_mu(x-mu))
  load_link(U, G.pad, mu, xmm_pn, B);
  load_link(U, G.pad, nu, xmm, C);
  load_link(U, G.pad, mu, xmm, A);
  mul<false, true>(D, B, P1);
  mul<true, false>(C, A, P2);
  mul<false, false>(P1, P2, q);
  accumulate(Q, q);
  // q3 = (U_mu(x-mu)^dag U_nu(x-mu-nu)^dag) (U_mu(x-mu-nu) U_nu(x-nu))
  load_link(U, G.pad, nu, xmm_mn, B);
  load_link(U, G.pad, mu, xmm_mn, C);
  load_link(U, G.pad, nu, xmn, D);
  mul<true, true>(A, B, P1);
  mul<false, false>(C, D, P2);
  mul<false, false>(P1, P2, q);
  accumulate(Q, q);
  // q4 = (U_nu(x-nu)^dag U_mu(x-nu)) (U_nu(x-nu+mu) U_mu(x)^dag)
  load_link(U, G.pad, mu, xmn, A);
  load_link(U, G.pad, nu, xmn_pm, B);
  load_link(U, G.pad, mu, g, C);
  mul<true, false>(D, A, P1);
  mul<false, true>(B, C, P2);
  mul<false, false>(P1, P2, q);
  accumulate(Q, q);
}

// in-place inverse of a 6x6 complex matrix (Gauss-Jordan, partial pivoting on
// the modulus); returns false for a singular block
__device__ bool invert6(Cx a[6][6]) {
  Cx inv[6][6];
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) inv[i][j] = {i == j ? 1.0 : 0.0, 0.0};
  for (int c = 0; c < 6; c++) {
    int p = c;
    for (int r = c + 1; r < 6; r++)
      if (cabs2(a[r][c]) > cabs2(a[p][c])) p = r;
    if (cabs2(a[p][c]) == 0) return false;
    if (p != c)
      for (int k = 0; k < 6; k++) {
        Cx t = a[p][k];
        a[p][k] = a[c][k];
        a[c][k] = t;
        t = inv[p][k];
        inv[p][k] = inv[c][k];
        inv[c][k] = t;
      }
    const double n = cabs2(a[c][c]);
    const Cx d = {a[c][c].r / n, -a[c][c].i / n};
    for (int k = 0; k < 6; k++) {
      a[c][k] = cmul(a[c][k], d);
      inv[c][k] = cmul(inv[c][k], d);
    }
    for (int r = 0; r < 6; r++) {
      if (r == c) continue;
      const Cx f = a[r][c];
      if (f.r == 0 && f.i == 0) continue;
      for (int k = 0; k < 6; k++) {
        a[r][k] = csub(a[r][k], cmul(f, a[c][k]));
        inv[r][k] = csub(inv[r][k], cmul(f, inv[c][k]));
      }
    }
  }
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) a[i][j] = inv[i][j];
  return true;
}

// writes the FP64 and FP32 planes at entry (g << oshift) + orhs, plane
// stride ostride (a lattice's own clover: 0, 0, pad; one RHS of a handle
// with per-RHS kappa: lgnr, rhs, spad)
__global__ void k_build_clover(Geom G, const double* __restrict__ U, double* Cd, float* Cs,
                               double ck, unsigned* bad, int oshift, int orhs, int ostride) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.V) return;
  int x[4];
  site_coords(G, g, x);
  Cx T[2][6][6];
  for (int b = 0; b < 2; b++)
    for (int i = 0; i < 6; i++)
      for (int j = 0; j < 6; j++) T[b][i][j] = {i == j ? 1.0 : 0.0, 0.0};
  int p = 0;
  for (int mu = 0; mu < 4; mu++)
    for (int nu = mu + 1; nu < 4; nu++, p++) {
      Mat Q, F;
      leaf_sum(G, U, x, g, mu, nu, Q);
      // F = (Q - Q^dag) / (8 i), traceless
      Cx tr = {0, 0};
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          const Cx d = csub(Q.a[i][j], conj(Q.a[j][i]));
          F.a[i][j] = {d.i / 8.0, -d.r / 8.0};
        }
      for (int i = 0; i < 3; i++) tr = cadd(tr, F.a[i][i]);
      for (int i = 0; i < 3; i++) F.a[i][i] = csub(F.a[i][i], {tr.r / 3.0, tr.i / 3.0});
      for (int b = 0; b < 2; b++)
        for (int h = 0; h < 2; h++)
          for (int h2 = 0; h2 < 2; h2++) {
            const Cx s = {c_S[p][b][h][h2][0] * ck, c_S[p][b][h][h2][1] * ck};
            if (s.r == 0 && s.i == 0) continue;
            for (int c = 0; c < 3; c++)
              for (int c2 = 0; c2 < 3; c2++)
                T[b][3 * h + c][3 * h2 + c2] =
                    csub(T[b][3 * h + c][3 * h2 + c2], cmul(s, F.a[c][c2]));
          }
    }
  double out[72];
  for (int b = 0; b < 2; b++) {
    if (!invert6(T[b])) {
      atomicAdd(bad, 1u);
      for (int j = 0; j < 36; j++) out[36 * b + j] = 0;
      continue;
    }
    double* o = out + 36 * b;
    for (int j = 0; j < 6; j++) o[j] = 0.5 * T[b][j][j].r;
    int n = 0;
    for (int j = 0; j < 6; j++)
      for (int k = j + 1; k < 6; k++, n++) {
        o[6 + 2 * n] = 0.5 * T[b][j][k].r;
        o[7 + 2 * n] = 0.5 * T[b][j][k].i;
      }
  }
  double2* qd = reinterpret_cast<double2*>(Cd);
  float4* qs = reinterpret_cast<float4*>(Cs);
  const size_t e = ((size_t)g << oshift) + orhs;
  for (int j = 0; j < 36; j++) qd[(size_t)j * ostride + e] = make_double2(out[2 * j], out[2 * j + 1]);
  for (int j = 0; j < 18; j++)
    qs[(size_t)j * ostride + e] = make_float4((float)out[4 * j], (float)out[4 * j + 1],
                                              (float)out[4 * j + 2], (float)out[4 * j + 3]);
}

}  // namespace

static const double (*chiral_tables())[2][2][2][2] {
  struct Tables {
    double S[6][2][2][2][2];
    double off;
    Tables() { off = clover_chiral_tables(S); }
  };
  static const Tables tab;  // built once, thread-safe
  if (tab.off > 1e-14) throw Error(3, "sigma_{mu nu} is not block diagonal in the chiral basis");
  return tab.S;
}

// one clover build on c's stream into (Cd, Cs) at (oshift, orhs, ostride)
static void build_into(Ctx& c, const double* Ud, double* Cd, float* Cs, double ck, int oshift,
                       int orhs, int ostride) {
  QWSG_CUDA(cudaMemcpyToSymbolAsync(c_S, chiral_tables(), sizeof(double) * 6 * 16, 0,
                                    cudaMemcpyHostToDevice, c.st));
  unsigned* bad = c.rb.counter + 1;  // a spare counter slot
  QWSG_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned), c.st));
  count_launch();
  k_build_clover<<<(c.G.V + 127) / 128, 128, 0, c.st>>>(c.G, Ud, Cd, Cs, ck, bad, oshift, orhs,
                                                         ostride);
  c.check_launch("build_clover");
  unsigned h_bad = 0;
  QWSG_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, c.st));
  QWSG_CUDA(cudaStreamSynchronize(c.st));
  if (h_bad) throw Error(2, "clover term singular on " + std::to_string(h_bad) + " blocks");
}

// clover term of the resident FP64 gauge field for this context's kappa:
// writes the FP64 and FP32 clover planes (the FP16 copies follow on demand)
void build_clover(Ctx& c, double csw) {
  if (!c.Ud) throw Error(4, "gauge field not loaded");
  if (c.parent) throw Error(1, "build the clover term on the parent lattice");
  c.ensure_fields_d();
  c.ensure_fields_s();
  c.fields_h_valid = false;
  build_into(c, c.Ud, c.Cd, c.Cs, csw * c.kappa, 0, 0, c.G.pad);
}

// per-RHS kappa on a multi-RHS handle: the clover term of the parent's gauge
// field for kappas[r], into the handle's per-RHS planes (FP64, FP32 and the
// FP16 copy), and the kappa tables the Dirac kernels read
void set_rhs_kappas(Ctx& c, const double* kappas, double csw) {
  if (!c.parent) throw Error(1, "per-RHS kappa needs a multi-RHS handle");
  c.sync_from_parent(false);
  if (!c.Ud) throw Error(4, "gauge field not loaded");
  const size_t n = (size_t)72 * spad(c.G);
  if (c.rhs_kappas.empty()) {  // graphs captured before read the parent's clover
    QWSG_CUDA(cudaStreamSynchronize(c.st));
    c.clear_graphs();
  }
  // each plane set on its own: one that failed to allocate is retried by the
  // next call, and no launch below runs before all of them exist
  auto want = [&](auto** p, size_t bytes) {
    if (*p) return;
    void* q = nullptr;
    QWSG_CUDA(cudaMalloc(&q, bytes));
    c.owned.push_back(q);
    *p = static_cast<std::remove_reference_t<decltype(**p)>*>(q);
  };
  want(&c.Cdr, sizeof(double) * n);
  want(&c.Csr, sizeof(float) * n);
  want(&c.Chr, sizeof(__half) * n);
  want(&c.kap_d, sizeof(double) * Ctx::kMaxRhs);
  want(&c.kap_s, sizeof(float) * Ctx::kMaxRhs);
  for (int r = 0; r < c.G.nr; r++)
    build_into(c, c.Ud, c.Cdr, c.Csr, csw * kappas[r], c.G.lgnr, r, spad(c.G));
  clover_s2h_entries(c.G, c.Chr, c.Csr, c.st);
  c.check_launch("clover_s2h_entries");
  double kd[Ctx::kMaxRhs];
  float ks[Ctx::kMaxRhs];
  for (int r = 0; r < c.G.nr; r++) {
    kd[r] = kappas[r];
    ks[r] = (float)kappas[r];
  }
  QWSG_CUDA(cudaMemcpyAsync(c.kap_d, kd, sizeof(double) * c.G.nr, cudaMemcpyHostToDevice, c.st));
  QWSG_CUDA(cudaMemcpyAsync(c.kap_s, ks, sizeof(float) * c.G.nr, cudaMemcpyHostToDevice, c.st));
  QWSG_CUDA(cudaStreamSynchronize(c.st));
  c.rhs_kappas.assign(kappas, kappas + c.G.nr);
}

}  // namespace qwsg
