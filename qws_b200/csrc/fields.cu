// Synthetic gauge, clover and source fields for benchmarks and tests
// (host code, OpenMP).  The reference only loads fields built elsewhere
// (BQCD, qws_bqcd.cc:125-382), so these conventions are ours; they are
// checked by properties (unitarity, Hermiticity, T * T^-1 = 1, free-field
// limit, plaquette) rather than against the reference.
//
// Random numbers: counter-based SplitMix64 streams keyed by (seed, site, mu,
// draw), so generation is parallel and independent of thread count.
//
// Conventions
//  * links: Gaussian complex 3x3 -> Gram-Schmidt on rows -> divided by a cube
//    root of the determinant (unit determinant), i.e. SU(3).
//  * APE-style smoothing: U' = Proj[(1-alpha) U + alpha/6 * sum of the six
//    staples], Proj = the same Gram-Schmidt + determinant-phase removal.
//  * gamma matrices: the Dirac basis implied by the hopping projectors of the
//    Wilson operator (see lattice.cuh): gamma_x, gamma_y, gamma_z as there,
//    gamma_t = diag(1,1,-1,-1).
//  * clover: F_{mu nu} = (Q - Q^dag)/(8i) from the four-leaf sum Q,
//    T = 1 - csw*kappa * sum_{mu<nu} sigma_{mu nu} F_{mu nu},
//    sigma_{mu nu} = (i/2)[gamma_mu, gamma_nu]; the stored per-site data are
//    the two 6x6 chiral blocks of T^-1 / 2 in QWS's packed format
//    (clover_def.h:88-284): with X = (s0+s2, s1+s3 | s0-s2, s1-s3) the clover
//    kernel computes s <- P^T diag(M0, M1) P s, so M_i = (P T P^T / 2)_i^-1 / 2.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/qwsg.h"
#include "ctx.h"

namespace qwsg {
namespace fields {

using cd = std::complex<double>;

static inline uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

struct Rng {
  uint64_t state;
  Rng(uint64_t seed, uint64_t a, uint64_t b)
      : state(splitmix64(seed ^ splitmix64(a * 0x100000001b3ull + b * 0x9e3779b97f4a7c15ull))) {}
  double uniform() {  // (0, 1]
    state += 0x9e3779b97f4a7c15ull;
    uint64_t z = splitmix64(state);
    return ((z >> 11) + 1) * (1.0 / 9007199254740992.0);
  }
  cd gauss() {  // unit-variance complex Gaussian (each part variance 1/2)
    double r = std::sqrt(-std::log(uniform()));
    double t = 2 * M_PI * uniform();
    return cd(r * std::cos(t), r * std::sin(t));
  }
};

struct M3 {
  cd a[3][3];
};

static inline M3 mul(const M3& x, const M3& y) {
  M3 r;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      cd s = 0;
      for (int k = 0; k < 3; k++) s += x.a[i][k] * y.a[k][j];
      r.a[i][j] = s;
    }
  return r;
}
static inline M3 dag(const M3& x) {
  M3 r;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) r.a[i][j] = std::conj(x.a[j][i]);
  return r;
}
static inline cd det(const M3& m) {
  const auto& a = m.a;
  return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
         a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
         a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
}

// Gram-Schmidt on the rows, then divide by a cube root of the determinant
static M3 project_su3(M3 m) {
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < i; j++) {
      cd p = 0;
      for (int k = 0; k < 3; k++) p += std::conj(m.a[j][k]) * m.a[i][k];
      for (int k = 0; k < 3; k++) m.a[i][k] -= p * m.a[j][k];
    }
    double n = 0;
    for (int k = 0; k < 3; k++) n += std::norm(m.a[i][k]);
    n = 1.0 / std::sqrt(n);
    for (int k = 0; k < 3; k++) m.a[i][k] *= n;
  }
  cd d = det(m);
  cd f = std::polar(1.0, -std::arg(d) / 3.0);
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++) m.a[i][k] *= f;
  return m;
}

struct Lat {
  int L[4];
  long V;
  long idx(const int x[4]) const {
    return x[0] + (long)L[0] * (x[1] + (long)L[1] * (x[2] + (long)L[2] * x[3]));
  }
  void coords(long s, int x[4]) const {
    x[0] = s % L[0];
    s /= L[0];
    x[1] = s % L[1];
    s /= L[1];
    x[2] = s % L[2];
    x[3] = (int)(s / L[2]);
  }
  long shift(long s, int mu, int d) const {
    int x[4];
    coords(s, x);
    x[mu] = (x[mu] + d + L[mu]) % L[mu];
    return idx(x);
  }
};

static inline M3 getU(const std::vector<M3>& U, const Lat& l, int mu, long s) { return U[mu * l.V + s]; }

static void staple_sum(const std::vector<M3>& U, const Lat& l, int mu, long s, M3& S) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) S.a[i][j] = 0;
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    long sp_mu = l.shift(s, mu, 1), sp_nu = l.shift(s, nu, 1), sm_nu = l.shift(s, nu, -1);
    long sm_nu_p_mu = l.shift(sm_nu, mu, 1);
    // U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag
    M3 a = mul(mul(getU(U, l, nu, s), getU(U, l, mu, sp_nu)), dag(getU(U, l, nu, sp_mu)));
    // U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu)
    M3 b = mul(mul(dag(getU(U, l, nu, sm_nu)), getU(U, l, mu, sm_nu)), getU(U, l, nu, sm_nu_p_mu));
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) S.a[i][j] += a.a[i][j] + b.a[i][j];
  }
}

static double plaquette(const std::vector<M3>& U, const Lat& l) {
  double tot = 0;
#pragma omp parallel for reduction(+ : tot) schedule(static)
  for (long s = 0; s < l.V; s++) {
    for (int mu = 0; mu < 4; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        M3 p = mul(mul(getU(U, l, mu, s), getU(U, l, nu, l.shift(s, mu, 1))),
                   mul(dag(getU(U, l, mu, l.shift(s, nu, 1))), dag(getU(U, l, nu, s))));
        tot += (p.a[0][0] + p.a[1][1] + p.a[2][2]).real() / 3.0;
      }
  }
  return tot / (6.0 * l.V);
}

// Q_{mu nu}(x): sum of the four plaquettes in the (mu,nu) plane touching x
static M3 leaf_sum(const std::vector<M3>& U, const Lat& l, long s, int mu, int nu) {
  long xpm = l.shift(s, mu, 1), xpn = l.shift(s, nu, 1);
  long xmm = l.shift(s, mu, -1), xmn = l.shift(s, nu, -1);
  long xmm_pn = l.shift(xmm, nu, 1), xmm_mn = l.shift(xmm, nu, -1), xmn_pm = l.shift(xmn, mu, 1);
  M3 q1 = mul(mul(getU(U, l, mu, s), getU(U, l, nu, xpm)),
              mul(dag(getU(U, l, mu, xpn)), dag(getU(U, l, nu, s))));
  M3 q2 = mul(mul(getU(U, l, nu, s), dag(getU(U, l, mu, xmm_pn))),
              mul(dag(getU(U, l, nu, xmm)), getU(U, l, mu, xmm)));
  M3 q3 = mul(mul(dag(getU(U, l, mu, xmm)), dag(getU(U, l, nu, xmm_mn))),
              mul(getU(U, l, mu, xmm_mn), getU(U, l, nu, xmn)));
  M3 q4 = mul(mul(dag(getU(U, l, nu, xmn)), getU(U, l, mu, xmn)),
              mul(getU(U, l, nu, xmn_pm), dag(getU(U, l, mu, s))));
  M3 r;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) r.a[i][j] = q1.a[i][j] + q2.a[i][j] + q3.a[i][j] + q4.a[i][j];
  return r;
}

static void gamma_matrices(cd g[4][4][4]) {
  const cd I(0, 1);
  std::memset((void*)g, 0, sizeof(cd) * 64);
  // gamma_x (from x+ projector h = (v0 - i v3, v1 - i v2))
  g[0][0][3] = I; g[0][1][2] = I; g[0][2][1] = -I; g[0][3][0] = -I;
  // gamma_y (h = (v0 - v3, v1 + v2))
  g[1][0][3] = 1; g[1][1][2] = -1; g[1][2][1] = -1; g[1][3][0] = 1;
  // gamma_z (h = (v0 - i v2, v1 + i v3))
  g[2][0][2] = I; g[2][1][3] = -I; g[2][2][0] = -I; g[2][3][1] = I;
  // gamma_t
  g[3][0][0] = 1; g[3][1][1] = 1; g[3][2][2] = -1; g[3][3][3] = -1;
}

// in-place inverse of an n x n complex matrix (Gauss-Jordan, partial pivoting)
static bool invert(cd* a, int n) {
  std::vector<cd> inv(n * n, 0.0);
  for (int i = 0; i < n; i++) inv[i * n + i] = 1;
  for (int c = 0; c < n; c++) {
    int p = c;
    for (int r = c + 1; r < n; r++)
      if (std::abs(a[r * n + c]) > std::abs(a[p * n + c])) p = r;
    if (std::abs(a[p * n + c]) == 0) return false;
    if (p != c)
      for (int k = 0; k < n; k++) {
        std::swap(a[p * n + k], a[c * n + k]);
        std::swap(inv[p * n + k], inv[c * n + k]);
      }
    cd d = 1.0 / a[c * n + c];
    for (int k = 0; k < n; k++) {
      a[c * n + k] *= d;
      inv[c * n + k] *= d;
    }
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      cd f = a[r * n + c];
      if (f == cd(0)) continue;
      for (int k = 0; k < n; k++) {
        a[r * n + k] -= f * a[c * n + k];
        inv[r * n + k] -= f * inv[c * n + k];
      }
    }
  }
  for (int i = 0; i < n * n; i++) a[i] = inv[i];
  return true;
}

}  // namespace fields

// sigma_{mu nu} (mu < nu, planes in the order 01 02 03 12 13 23) in the
// chiral basis of the packed clover: S[p][i][h][h2] = (Ps sigma Ps^T / 2)
// restricted to chirality block i, rows h / columns h2 of that block, with
// Ps rows (s0+s2, s1+s3 | s0-s2, s1-s3).  Returns the largest entry outside
// the two chirality blocks (zero: sigma is block diagonal there).
double clover_chiral_tables(double S[6][2][2][2][2]) {
  using namespace fields;
  cd g[4][4][4];
  gamma_matrices(g);
  const cd I(0, 1);
  const double Ps[4][4] = {{1, 0, 1, 0}, {0, 1, 0, 1}, {1, 0, -1, 0}, {0, 1, 0, -1}};
  double off = 0;
  int p = 0;
  for (int m = 0; m < 4; m++)
    for (int n = m + 1; n < 4; n++, p++) {
      cd sig[4][4];
      for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) {
          cd c = 0;
          for (int k = 0; k < 4; k++) c += g[m][a][k] * g[n][k][b] - g[n][a][k] * g[m][k][b];
          sig[a][b] = 0.5 * I * c;
        }
      for (int r = 0; r < 4; r++)
        for (int q = 0; q < 4; q++) {
          cd acc = 0;
          for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) acc += Ps[r][a] * sig[a][b] * Ps[q][b];
          acc *= 0.5;
          const int i = r / 2, j = q / 2;
          if (i != j) {
            off = std::max(off, std::abs(acc));
            continue;
          }
          S[p][i][r % 2][q % 2][0] = acc.real();
          S[p][i][r % 2][q % 2][1] = acc.imag();
        }
    }
  return off;
}

}  // namespace qwsg

using namespace qwsg::fields;

extern "C" {

// gauge: natural layout [4][V][3][3][2]
int qwsg_gen_gauge(double* U, const int L[4], unsigned long long seed, int n_smear, double alpha,
                   double* plaq) {
  try {
    Lat l{{L[0], L[1], L[2], L[3]}, (long)L[0] * L[1] * L[2] * L[3]};
    std::vector<M3> u(4 * l.V), w(4 * l.V);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < l.V; s++)
      for (int mu = 0; mu < 4; mu++) {
        Rng r(seed, (uint64_t)s, (uint64_t)mu);
        M3 m;
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) m.a[i][j] = r.gauss();
        u[mu * l.V + s] = project_su3(m);
      }
    for (int it = 0; it < n_smear; it++) {
#pragma omp parallel for schedule(static)
      for (long s = 0; s < l.V; s++)
        for (int mu = 0; mu < 4; mu++) {
          M3 S;
          staple_sum(u, l, mu, s, S);
          M3 m;
          const M3& o = u[mu * l.V + s];
          for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
              m.a[i][j] = (1 - alpha) * o.a[i][j] + (alpha / 6.0) * S.a[i][j];
          w[mu * l.V + s] = project_su3(m);
        }
      std::swap(u, w);
    }
    if (plaq) *plaq = plaquette(u, l);
#pragma omp parallel for schedule(static)
    for (long k = 0; k < 4 * l.V; k++)
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          U[k * 18 + 2 * (3 * i + j)] = u[k].a[i][j].real();
          U[k * 18 + 2 * (3 * i + j) + 1] = u[k].a[i][j].imag();
        }
    return 0;
  } catch (...) {
    return 3;
  }
}

int qwsg_plaquette(const double* U, const int L[4], double* plaq) {
  Lat l{{L[0], L[1], L[2], L[3]}, (long)L[0] * L[1] * L[2] * L[3]};
  std::vector<M3> u(4 * l.V);
#pragma omp parallel for schedule(static)
  for (long k = 0; k < 4 * l.V; k++)
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        u[k].a[i][j] = cd(U[k * 18 + 2 * (3 * i + j)], U[k * 18 + 2 * (3 * i + j) + 1]);
  *plaq = plaquette(u, l);
  return 0;
}

// clover: natural layout [V][72] = packed chiral blocks of T^-1 / 2; with
// T_out (optional, [V][12][12][2], spinor index 4*colour+spin) the clover
// term itself for tests.
int qwsg_gen_clover(double* C, const double* U, const int L[4], double csw, double kappa,
                    double* T_out) {
  Lat l{{L[0], L[1], L[2], L[3]}, (long)L[0] * L[1] * L[2] * L[3]};
  std::vector<M3> u(4 * l.V);
#pragma omp parallel for schedule(static)
  for (long k = 0; k < 4 * l.V; k++)
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        u[k].a[i][j] = cd(U[k * 18 + 2 * (3 * i + j)], U[k * 18 + 2 * (3 * i + j) + 1]);
  cd g[4][4][4];
  gamma_matrices(g);
  const cd I(0, 1);
  // sigma_{mu nu} = (i/2)[g_mu, g_nu]
  cd sig[4][4][4][4];
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++)
      for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) {
          cd c = 0;
          for (int k = 0; k < 4; k++) c += g[m][a][k] * g[n][k][b] - g[n][a][k] * g[m][k][b];
          sig[m][n][a][b] = 0.5 * I * c;
        }
  // chiral rotation X = P psi (12x12, spinor index 4*col+spin;
  // X index 6*i + k, k<3: colour k from spins (0,2); k>=3: colour k-3, spins (1,3))
  double P[12][12];
  std::memset(P, 0, sizeof(P));
  for (int c = 0; c < 3; c++) {
    P[c][4 * c + 0] = 1; P[c][4 * c + 2] = 1;
    P[3 + c][4 * c + 1] = 1; P[3 + c][4 * c + 3] = 1;
    P[6 + c][4 * c + 0] = 1; P[6 + c][4 * c + 2] = -1;
    P[9 + c][4 * c + 1] = 1; P[9 + c][4 * c + 3] = -1;
  }
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
  for (long s = 0; s < l.V; s++) {
    cd T[12][12];
    for (int i = 0; i < 12; i++)
      for (int j = 0; j < 12; j++) T[i][j] = (i == j) ? 1.0 : 0.0;
    for (int mu = 0; mu < 4; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        M3 q = leaf_sum(u, l, s, mu, nu);
        // F = (Q - Q^dag) / (8 i), made traceless
        M3 F;
        cd tr = 0;
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) F.a[i][j] = (q.a[i][j] - std::conj(q.a[j][i])) / (8.0 * I);
        for (int i = 0; i < 3; i++) tr += F.a[i][i];
        for (int i = 0; i < 3; i++) F.a[i][i] -= tr / 3.0;
        for (int a = 0; a < 4; a++)
          for (int b = 0; b < 4; b++) {
            cd sg = sig[mu][nu][a][b];
            if (sg == cd(0)) continue;
            for (int ci = 0; ci < 3; ci++)
              for (int cj = 0; cj < 3; cj++)
                T[4 * ci + a][4 * cj + b] -= csw * kappa * sg * F.a[ci][cj];
          }
      }
    if (T_out)
      for (int i = 0; i < 12; i++)
        for (int j = 0; j < 12; j++) {
          T_out[((s * 12 + i) * 12 + j) * 2] = T[i][j].real();
          T_out[((s * 12 + i) * 12 + j) * 2 + 1] = T[i][j].imag();
        }
    // Tc = P T P^T / 2 (block diagonal for a chirally symmetric T)
    cd Tc[12][12];
    for (int i = 0; i < 12; i++)
      for (int j = 0; j < 12; j++) {
        cd acc = 0;
        for (int a = 0; a < 12; a++) {
          if (P[i][a] == 0) continue;
          for (int b = 0; b < 12; b++)
            if (P[j][b] != 0) acc += P[i][a] * T[a][b] * P[j][b];
        }
        Tc[i][j] = 0.5 * acc;
      }
    for (int blk = 0; blk < 2; blk++) {
      cd m[36];
      for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) m[6 * i + j] = Tc[6 * blk + i][6 * blk + j];
      if (!invert(m, 6)) {
        bad++;
        continue;
      }
      double* out = C + 72 * s + 36 * blk;
      for (int j = 0; j < 6; j++) out[j] = 0.5 * m[6 * j + j].real();
      int n = 0;
      for (int j = 0; j < 6; j++)
        for (int k = j + 1; k < 6; k++, n++) {
          out[6 + 2 * n] = 0.5 * m[6 * j + k].real();
          out[7 + 2 * n] = 0.5 * m[6 * j + k].imag();
        }
    }
  }
  return bad ? 2 : 0;
}

// spinor sources, natural layout [V][24]
//  kind 0: Gaussian complex (unit variance per complex component)
//  kind 1: point source at the origin in (spin, colour) = (arg % 4, arg / 4)
//  kind 2: Z2 noise, (+-1 +- i)/sqrt(2) on every component
int qwsg_gen_source(double* S, const int L[4], unsigned long long seed, int kind, int arg) {
  long V = (long)L[0] * L[1] * L[2] * L[3];
  std::memset(S, 0, sizeof(double) * 24 * V);
  if (kind == 1) {
    int spin = arg % 4, col = arg / 4;
    S[8 * col + 2 * spin] = 1.0;
    return 0;
  }
#pragma omp parallel for schedule(static)
  for (long s = 0; s < V; s++) {
    Rng r(seed, (uint64_t)s, 1000 + (uint64_t)kind);
    for (int k = 0; k < 12; k++) {
      cd z;
      if (kind == 0) {
        z = r.gauss();
      } else {
        double a = r.uniform() < 0.5 ? -1 : 1, b = r.uniform() < 0.5 ? -1 : 1;
        z = cd(a, b) / std::sqrt(2.0);
      }
      S[24 * s + 2 * k] = z.real();
      S[24 * s + 2 * k + 1] = z.imag();
    }
  }
  return 0;
}

}  // extern "C"
