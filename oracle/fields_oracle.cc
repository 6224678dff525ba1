// Synthetic benchmark fields restated for the CPU checkers.
//
// TEST INFRASTRUCTURE ONLY: the reference arm of the benchmark and the
// parity tests build the reference's inputs with these functions, so the
// reference's own solver (oracle/_ref) runs without loading the product
// library.  The product generates the same fields on its side
// (qwsg_gen_gauge / qwsg_gen_clover / qwsg_gen_source); the tests check the
// two bit for bit, so both arms of a comparison consume identical arrays.
//
// The reference itself has no field generator: QWS loads links and a
// pre-inverted clover term built by BQCD (qws_bqcd.cc:125, :284).  These
// conventions are therefore the benchmark's, stated here in full:
//
//  * random numbers: SplitMix64 (Steele, Lea, Flood 2014) as a counter
//    generator; every (site, direction) owns a stream keyed by
//    (seed, site, direction), so the result does not depend on threads;
//    uniform u in (0, 1] from the top 53 bits; a complex Gaussian with
//    E|z|^2 = 1 by Box-Muller: sqrt(-log u1) * exp(2 pi i u2);
//  * links: 3x3 complex Gaussian matrix, rows orthonormalised in order
//    (Gram-Schmidt), then multiplied by exp(-i arg(det)/3): SU(3);
//  * smoothing: U' = Proj[(1 - alpha) U + alpha/6 * (sum of the 6 staples)];
//  * clover: leaf sum Q of the four plaquettes in each plane, F = (Q -
//    Q^dag)/(8 i) minus its trace/3, T = 1 - csw kappa sum_{mu<nu} sigma F
//    with sigma = (i/2)[gamma_mu, gamma_nu] in the basis the Dirac operator's
//    spin projectors imply (gamma_t = diag(1, 1, -1, -1)); stored: the two
//    6x6 chiral blocks of (X T X^T / 2)^-1 / 2, X the chiral rotation
//    (s0 + s2, s1 + s3 | s0 - s2, s1 - s3), packed as the reference's clover
//    kernel reads them (clover_def.h:88-284: 6 real diagonal entries, then the
//    15 upper off-diagonal entries row by row as re, im);
//  * sources: Gaussian (as above, per colour-spin component), a point
//    source at the origin, or Z2 noise (+-1 +- i)/sqrt(2).
//
// Bit-exactness: every floating-point operation below is written in the
// order the product's generator performs it, with std::complex arithmetic
// and no fused multiply-add (plain x86-64 code generation, no -march), so
// the two agree bit for bit on the same host.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

typedef std::complex<double> cplx;

struct SU3 {
  cplx e[3][3];
};

uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

class Draws {
 public:
  Draws(uint64_t seed, uint64_t site, uint64_t dir)
      : s_(mix64(seed ^ mix64(site * 0x100000001b3ull + dir * 0x9e3779b97f4a7c15ull))) {}
  double unit() {
    s_ += 0x9e3779b97f4a7c15ull;
    return ((mix64(s_) >> 11) + 1) * (1.0 / 9007199254740992.0);
  }
  cplx normal() {
    double rad = std::sqrt(-std::log(unit()));
    double ang = 2 * M_PI * unit();
    return cplx(rad * std::cos(ang), rad * std::sin(ang));
  }

 private:
  uint64_t s_;
};

SU3 prod(const SU3& A, const SU3& B) {
  SU3 C;
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) {
      cplx acc = 0;
      for (int k = 0; k < 3; k++) acc += A.e[r][k] * B.e[k][c];
      C.e[r][c] = acc;
    }
  return C;
}

SU3 adj(const SU3& A) {
  SU3 C;
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) C.e[r][c] = std::conj(A.e[c][r]);
  return C;
}

cplx det3(const SU3& A) {
  const cplx(*a)[3] = A.e;
  cplx m0 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
  cplx m1 = a[1][0] * a[2][2] - a[1][2] * a[2][0];
  cplx m2 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
  return a[0][0] * m0 - a[0][1] * m1 + a[0][2] * m2;
}

SU3 to_su3(SU3 A) {
  for (int r = 0; r < 3; r++) {
    for (int q = 0; q < r; q++) {
      cplx ov = 0;
      for (int k = 0; k < 3; k++) ov += std::conj(A.e[q][k]) * A.e[r][k];
      for (int k = 0; k < 3; k++) A.e[r][k] -= ov * A.e[q][k];
    }
    double n2 = 0;
    for (int k = 0; k < 3; k++) n2 += std::norm(A.e[r][k]);
    n2 = 1.0 / std::sqrt(n2);
    for (int k = 0; k < 3; k++) A.e[r][k] *= n2;
  }
  cplx phase = std::polar(1.0, -std::arg(det3(A)) / 3.0);
  for (int r = 0; r < 3; r++)
    for (int k = 0; k < 3; k++) A.e[r][k] *= phase;
  return A;
}

struct Geo {
  int n[4];
  long vol;
  long site(int x, int y, int z, int t) const {
    return x + (long)n[0] * (y + (long)n[1] * (z + (long)n[2] * t));
  }
  // neighbour of s displaced by d along mu (periodic)
  long nb(long s, int mu, int d) const {
    int c[4];
    long r = s;
    for (int m = 0; m < 3; m++) {
      c[m] = (int)(r % n[m]);
      r /= n[m];
    }
    c[3] = (int)r;
    c[mu] = (c[mu] + d + n[mu]) % n[mu];
    return site(c[0], c[1], c[2], c[3]);
  }
};

// sum over the six staples of link (s, mu)
SU3 staples(const std::vector<SU3>& U, const Geo& g, int mu, long s) {
  SU3 S;
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) S.e[r][c] = 0;
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    long up_mu = g.nb(s, mu, 1), up_nu = g.nb(s, nu, 1), dn_nu = g.nb(s, nu, -1);
    long dn_nu_up_mu = g.nb(dn_nu, mu, 1);
    SU3 fwd = prod(prod(U[nu * g.vol + s], U[mu * g.vol + up_nu]), adj(U[nu * g.vol + up_mu]));
    SU3 bwd = prod(prod(adj(U[nu * g.vol + dn_nu]), U[mu * g.vol + dn_nu]),
                   U[nu * g.vol + dn_nu_up_mu]);
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) S.e[r][c] += fwd.e[r][c] + bwd.e[r][c];
  }
  return S;
}

// the four plaquettes of plane (mu, nu) that touch s, summed
SU3 four_leaves(const std::vector<SU3>& U, const Geo& g, long s, int mu, int nu) {
  const long V = g.vol;
  long pm = g.nb(s, mu, 1), pn = g.nb(s, nu, 1);
  long mm = g.nb(s, mu, -1), mn = g.nb(s, nu, -1);
  long mm_pn = g.nb(mm, nu, 1), mm_mn = g.nb(mm, nu, -1), mn_pm = g.nb(mn, mu, 1);
  auto u = [&](int d, long x) -> const SU3& { return U[d * V + x]; };
  SU3 l1 = prod(prod(u(mu, s), u(nu, pm)), prod(adj(u(mu, pn)), adj(u(nu, s))));
  SU3 l2 = prod(prod(u(nu, s), adj(u(mu, mm_pn))), prod(adj(u(nu, mm)), u(mu, mm)));
  SU3 l3 = prod(prod(adj(u(mu, mm)), adj(u(nu, mm_mn))), prod(u(mu, mm_mn), u(nu, mn)));
  SU3 l4 = prod(prod(adj(u(nu, mn)), u(mu, mn)), prod(u(nu, mn_pm), adj(u(mu, s))));
  SU3 Q;
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) Q.e[r][c] = l1.e[r][c] + l2.e[r][c] + l3.e[r][c] + l4.e[r][c];
  return Q;
}

// Dirac matrices of the operator's spin projectors, [mu][row][col]
void dirac_gammas(cplx G[4][4][4]) {
  const cplx i1(0, 1);
  for (int m = 0; m < 4; m++)
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++) G[m][a][b] = 0;
  G[0][0][3] = i1;  G[0][1][2] = i1;  G[0][2][1] = -i1; G[0][3][0] = -i1;
  G[1][0][3] = 1;   G[1][1][2] = -1;  G[1][2][1] = -1;  G[1][3][0] = 1;
  G[2][0][2] = i1;  G[2][1][3] = -i1; G[2][2][0] = -i1; G[2][3][1] = i1;
  G[3][0][0] = 1;   G[3][1][1] = 1;   G[3][2][2] = -1;  G[3][3][3] = -1;
}

// Gauss-Jordan inverse with partial pivoting of an n x n row-major matrix,
// in place; false if singular
bool gj_inverse(cplx* M, int n) {
  std::vector<cplx> R(n * n, 0.0);
  for (int d = 0; d < n; d++) R[d * n + d] = 1;
  for (int c = 0; c < n; c++) {
    int piv = c;
    for (int r = c + 1; r < n; r++)
      if (std::abs(M[r * n + c]) > std::abs(M[piv * n + c])) piv = r;
    if (std::abs(M[piv * n + c]) == 0) return false;
    if (piv != c)
      for (int k = 0; k < n; k++) {
        std::swap(M[piv * n + k], M[c * n + k]);
        std::swap(R[piv * n + k], R[c * n + k]);
      }
    cplx inv_p = 1.0 / M[c * n + c];
    for (int k = 0; k < n; k++) {
      M[c * n + k] *= inv_p;
      R[c * n + k] *= inv_p;
    }
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      cplx f = M[r * n + c];
      if (f == cplx(0)) continue;
      for (int k = 0; k < n; k++) {
        M[r * n + k] -= f * M[c * n + k];
        R[r * n + k] -= f * R[c * n + k];
      }
    }
  }
  for (int k = 0; k < n * n; k++) M[k] = R[k];
  return true;
}

void unpack_links(const double* U, long nlinks, std::vector<SU3>& u) {
  u.resize(nlinks);
#pragma omp parallel for schedule(static)
  for (long k = 0; k < nlinks; k++)
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++)
        u[k].e[r][c] = cplx(U[18 * k + 6 * r + 2 * c], U[18 * k + 6 * r + 2 * c + 1]);
}

double mean_plaquette(const std::vector<SU3>& U, const Geo& g) {
  double sum = 0;
#pragma omp parallel for reduction(+ : sum) schedule(static)
  for (long s = 0; s < g.vol; s++)
    for (int mu = 0; mu < 4; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        SU3 p = prod(prod(U[mu * g.vol + s], U[nu * g.vol + g.nb(s, mu, 1)]),
                     prod(adj(U[mu * g.vol + g.nb(s, nu, 1)]), adj(U[nu * g.vol + s])));
        sum += (p.e[0][0] + p.e[1][1] + p.e[2][2]).real() / 3.0;
      }
  return sum / (6.0 * g.vol);
}

}  // namespace

extern "C" {

// links in natural layout U[mu][site][row][col][re,im]; returns the mean
// plaquette in *plaq (when non-null)
void orc_gen_gauge(double* Uout, const int L[4], unsigned long long seed, int n_smear,
                   double alpha, double* plaq) {
  Geo g{{L[0], L[1], L[2], L[3]}, (long)L[0] * L[1] * L[2] * L[3]};
  std::vector<SU3> cur(4 * g.vol), nxt(4 * g.vol);
#pragma omp parallel for schedule(static)
  for (long s = 0; s < g.vol; s++)
    for (int mu = 0; mu < 4; mu++) {
      Draws d(seed, (uint64_t)s, (uint64_t)mu);
      SU3 m;
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) m.e[r][c] = d.normal();
      cur[mu * g.vol + s] = to_su3(m);
    }
  for (int step = 0; step < n_smear; step++) {
#pragma omp parallel for schedule(static)
    for (long s = 0; s < g.vol; s++)
      for (int mu = 0; mu < 4; mu++) {
        SU3 st = staples(cur, g, mu, s);
        const SU3& old = cur[mu * g.vol + s];
        SU3 m;
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++)
            m.e[r][c] = (1 - alpha) * old.e[r][c] + (alpha / 6.0) * st.e[r][c];
        nxt[mu * g.vol + s] = to_su3(m);
      }
    cur.swap(nxt);
  }
  if (plaq) *plaq = mean_plaquette(cur, g);
#pragma omp parallel for schedule(static)
  for (long k = 0; k < 4 * g.vol; k++)
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) {
        Uout[18 * k + 6 * r + 2 * c] = cur[k].e[r][c].real();
        Uout[18 * k + 6 * r + 2 * c + 1] = cur[k].e[r][c].imag();
      }
}

double orc_plaquette(const double* U, const int L[4]) {
  Geo g{{L[0], L[1], L[2], L[3]}, (long)L[0] * L[1] * L[2] * L[3]};
  std::vector<SU3> u;
  unpack_links(U, 4 * g.vol, u);
  return mean_plaquette(u, g);
}

// clover term of the links U (natural layout) as the packed inverse
// C[site][2 blocks][36]; returns the number of singular blocks
int orc_gen_clover(double* C, const double* U, const int L[4], double csw, double kappa) {
  Geo g{{L[0], L[1], L[2], L[3]}, (long)L[0] * L[1] * L[2] * L[3]};
  std::vector<SU3> u;
  unpack_links(U, 4 * g.vol, u);
  cplx G[4][4][4];
  dirac_gammas(G);
  const cplx i1(0, 1);
  cplx sigma[4][4][4][4];  // [mu][nu][a][b] = (i/2)[G_mu, G_nu]
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++)
      for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) {
          cplx comm = 0;
          for (int k = 0; k < 4; k++) comm += G[m][a][k] * G[n][k][b] - G[n][a][k] * G[m][k][b];
          sigma[m][n][a][b] = 0.5 * i1 * comm;
        }
  // chiral rotation X: row 6h + k, k < 3 colour k of spins (0, 2), k >= 3
  // colour k - 3 of spins (1, 3); h = 0 sums, h = 1 differences
  double X[12][12];
  std::memset(X, 0, sizeof(X));
  for (int c = 0; c < 3; c++) {
    X[c][4 * c] = 1;      X[c][4 * c + 2] = 1;
    X[3 + c][4 * c + 1] = 1; X[3 + c][4 * c + 3] = 1;
    X[6 + c][4 * c] = 1;  X[6 + c][4 * c + 2] = -1;
    X[9 + c][4 * c + 1] = 1; X[9 + c][4 * c + 3] = -1;
  }
  int singular = 0;
#pragma omp parallel for schedule(static) reduction(+ : singular)
  for (long s = 0; s < g.vol; s++) {
    cplx T[12][12];  // spinor index 4 * colour + spin
    for (int i = 0; i < 12; i++)
      for (int j = 0; j < 12; j++) T[i][j] = (i == j) ? 1.0 : 0.0;
    for (int mu = 0; mu < 4; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        SU3 Q = four_leaves(u, g, s, mu, nu);
        SU3 F;
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) F.e[r][c] = (Q.e[r][c] - std::conj(Q.e[c][r])) / (8.0 * i1);
        cplx tr = 0;
        for (int r = 0; r < 3; r++) tr += F.e[r][r];
        for (int r = 0; r < 3; r++) F.e[r][r] -= tr / 3.0;
        for (int a = 0; a < 4; a++)
          for (int b = 0; b < 4; b++) {
            cplx sab = sigma[mu][nu][a][b];
            if (sab == cplx(0)) continue;
            for (int ci = 0; ci < 3; ci++)
              for (int cj = 0; cj < 3; cj++)
                T[4 * ci + a][4 * cj + b] -= csw * kappa * sab * F.e[ci][cj];
          }
      }
    cplx Tx[12][12];  // X T X^T / 2
    for (int i = 0; i < 12; i++)
      for (int j = 0; j < 12; j++) {
        cplx acc = 0;
        for (int a = 0; a < 12; a++) {
          if (X[i][a] == 0) continue;
          for (int b = 0; b < 12; b++)
            if (X[j][b] != 0) acc += X[i][a] * T[a][b] * X[j][b];
        }
        Tx[i][j] = 0.5 * acc;
      }
    for (int h = 0; h < 2; h++) {
      cplx blk[36];
      for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) blk[6 * i + j] = Tx[6 * h + i][6 * h + j];
      if (!gj_inverse(blk, 6)) {
        singular++;
        continue;
      }
      double* o = C + 72 * s + 36 * h;
      for (int d = 0; d < 6; d++) o[d] = 0.5 * blk[7 * d].real();
      int n = 0;
      for (int i = 0; i < 6; i++)
        for (int j = i + 1; j < 6; j++, n++) {
          o[6 + 2 * n] = 0.5 * blk[6 * i + j].real();
          o[7 + 2 * n] = 0.5 * blk[6 * i + j].imag();
        }
    }
  }
  return singular;
}

// spinor source S[site][colour][spin][re,im]: kind 0 Gaussian, 1 point source
// at the origin in component (spin, colour) = (arg % 4, arg / 4), 2 Z2 noise
void orc_gen_source(double* S, const int L[4], unsigned long long seed, int kind, int arg) {
  long V = (long)L[0] * L[1] * L[2] * L[3];
  std::memset(S, 0, sizeof(double) * 24 * V);
  if (kind == 1) {
    S[8 * (arg / 4) + 2 * (arg % 4)] = 1.0;
    return;
  }
#pragma omp parallel for schedule(static)
  for (long s = 0; s < V; s++) {
    Draws d(seed, (uint64_t)s, 1000 + (uint64_t)kind);
    for (int k = 0; k < 12; k++) {
      cplx z;
      if (kind == 0) {
        z = d.normal();
      } else {
        double re = d.unit() < 0.5 ? -1 : 1;
        double im = d.unit() < 0.5 ? -1 : 1;
        z = cplx(re, im) / std::sqrt(2.0);
      }
      S[24 * s + 2 * k] = z.real();
      S[24 * s + 2 * k + 1] = z.imag();
    }
  }
}

}  // extern "C"
