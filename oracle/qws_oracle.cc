// CPU restatement of QWS's domain-decomposed Wilson-clover solver path.
// TEST INFRASTRUCTURE ONLY (the checker; see qws_oracle.h for the rules,
// the layout and how it is pinned against the reference's goldens).
//
// Every function below restates one reference routine in plain loops over a
// natural, global lexicographic lattice.  SIMD lanes, MPI halo buffers and
// the x-half memory aliasing of the reference are replaced by their meaning:
//   * a "block" is one x-half of one rank's local volume;
//   * a halo face captured by ddd_out_pre_* is a snapshot of the source
//     field taken at the time of the pre call (the reference packs faces into
//     send buffers, ddd_out_s.cc:112-337, and ddd_out_pos_* reads only those
//     buffers, ddd_out_s.cc:341-629).
#include "qws_oracle.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <random>
#include <vector>

namespace {

template <typename T>
using cx = std::complex<T>;

}  // namespace

struct orc_lat {
  int L[4], NB[4], B[4];
  long V;
  int tbc;
  double kappa;
  std::vector<double> Ud, Cd;  // gauge [4][V][3][3][2], clover [V][72]
  std::vector<float> Us, Cs;
};

namespace {

inline void coords(const orc_lat* l, long s, int c[4]) {
  c[0] = (int)(s % l->L[0]);
  s /= l->L[0];
  c[1] = (int)(s % l->L[1]);
  s /= l->L[1];
  c[2] = (int)(s % l->L[2]);
  c[3] = (int)(s / l->L[2]);
}

inline long site_of(const orc_lat* l, const int c[4]) {
  return c[0] + (long)l->L[0] * (c[1] + (long)l->L[1] * (c[2] + (long)l->L[2] * c[3]));
}

inline int block_colour(const orc_lat* l, const int c[4]) {
  int s = 0;
  for (int mu = 0; mu < 4; mu++) s += c[mu] / l->B[mu];
  return s & 1;
}

inline bool selected(const orc_lat* l, long s, int kind, int sel) {
  int c[4];
  coords(l, s, c);
  if (kind == 0) return block_colour(l, c) == sel;
  return ((c[0] / l->B[0]) & 1) == sel;
}

template <typename T>
const T* gauge(const orc_lat* l);
template <>
const double* gauge<double>(const orc_lat* l) { return l->Ud.data(); }
template <>
const float* gauge<float>(const orc_lat* l) { return l->Us.data(); }
template <typename T>
const T* clover(const orc_lat* l);
template <>
const double* clover<double>(const orc_lat* l) { return l->Cd.data(); }
template <>
const float* clover<float>(const orc_lat* l) { return l->Cs.data(); }

// r = U h   (U row-major [3][3] complex, h two half-spinor components)
template <typename T>
inline void mul_u(const T* u, const cx<T> h[3][2], cx<T> r[3][2], bool dagger) {
  for (int a = 0; a < 3; a++)
    for (int k = 0; k < 2; k++) {
      cx<T> acc(0, 0);
      for (int b = 0; b < 3; b++) {
        cx<T> ub = dagger ? std::conj(cx<T>(u[2 * (3 * b + a)], u[2 * (3 * b + a) + 1]))
                          : cx<T>(u[2 * (3 * a + b)], u[2 * (3 * a + b) + 1]);
        acc += ub * h[b][k];
      }
      r[a][k] = acc;
    }
}

// Sum of the hopping terms into site s.  which: 1 = hops that stay inside
// the site's block (ddd_in_*: neighbour terms skipped at block faces,
// ddd_in_d.cc:91-190), 2 = hops that cross a block face (ddd_out_*),
// 3 = both.  Spin projections and reconstructions restate wilson_d.h /
// mult_all.h: x,y,z use (1 -+ gamma_mu) in QWS's Dirac basis, t uses
// gamma_4 = diag(1,1,-1,-1) with the factor 2 (and the antiperiodic phase
// fbc at the global t boundary, qws.cc:298-310, ddd_out_d.cc:214-219).
//
// pair_halves: model of the FP32 face packer's pairing when every rank passes
// the same domain index (ddd_out_s.cc:128-131 packs y/z/t faces from domain
// 1-idomain whenever npe[mu] > 1, which is the geometric neighbour only when
// neighbouring ranks work on opposite x-halves, as they do inside
// prec_ddd_s_).  With pair_halves set, a y/z/t hop that leaves the rank
// (NB[mu] > 1) lands on the same offset in the other x-half of the
// neighbouring rank.
//
// box: extents that define "inside" (default the SAP block; the even-odd
// operators use the rank's local volume).  dag: the adjoint hopping term
// H^dagger (deo_dag_*): a forward hop projects with (1 + gamma_mu) and a
// backward hop with (1 - gamma_mu), the links being used as in H.
//
// eo_index: model of the even-odd face packers (deo_out_d.cc:88-153): a y/z/t
// hop that leaves the rank box reads the other parity's site at the SAME
// compressed index x/2 of the wrapped row.  That is the geometric neighbour
// when the wrapped extent is even; with an odd extent the lattice is not
// bipartite across the wrap and the reference reads the adjacent x site.
template <typename T>
void hop_site(const orc_lat* l, const T* in, long s, int which, cx<T> acc[3][4],
              bool pair_halves = false, const int* box = nullptr, bool dag = false,
              bool eo_index = false) {
  const T* U = gauge<T>(l);
  const int* B = box ? box : l->B;
  int c[4];
  coords(l, s, c);
  for (int a = 0; a < 3; a++)
    for (int sp = 0; sp < 4; sp++) acc[a][sp] = cx<T>(0, 0);
  const cx<T> I(0, 1);
  for (int mu = 0; mu < 4; mu++) {
    for (int dir = 0; dir < 2; dir++) {  // 0 forward, 1 backward
      bool inner = dir == 0 ? (c[mu] % B[mu]) != B[mu] - 1 : (c[mu] % B[mu]) != 0;
      const int pd = dag ? 1 - dir : dir;  // projector/reconstruction of this hop
      if (!((inner && (which & 1)) || (!inner && (which & 2)))) continue;
      int cn[4] = {c[0], c[1], c[2], c[3]};
      cn[mu] = dir == 0 ? (c[mu] + 1) % l->L[mu] : (c[mu] - 1 + l->L[mu]) % l->L[mu];
      if (pair_halves && !inner && mu > 0 && l->NB[mu] > 1) {
        int B0 = l->B[0], base = (c[0] / (2 * B0)) * 2 * B0, h = (c[0] / B0) & 1;
        cn[0] = base + (1 - h) * B0 + c[0] % B0;
      }
      if (eo_index && !inner && mu > 0) {
        const int po = 1 - ((c[0] + c[1] + c[2] + c[3]) & 1);
        cn[0] = 2 * (c[0] / 2) + ((po + cn[1] + cn[2] + cn[3]) & 1);
      }
      long sn = site_of(l, cn);
      const T* v = in + 24 * sn;
      cx<T> h[3][2], r[3][2];
      for (int a = 0; a < 3; a++) {
        cx<T> v0(v[8 * a + 0], v[8 * a + 1]), v1(v[8 * a + 2], v[8 * a + 3]);
        cx<T> v2(v[8 * a + 4], v[8 * a + 5]), v3(v[8 * a + 6], v[8 * a + 7]);
        switch (mu * 2 + pd) {
          case 0: h[a][0] = v0 - I * v3; h[a][1] = v1 - I * v2; break;
          case 1: h[a][0] = v0 + I * v3; h[a][1] = v1 + I * v2; break;
          case 2: h[a][0] = v0 - v3; h[a][1] = v1 + v2; break;
          case 3: h[a][0] = v0 + v3; h[a][1] = v1 - v2; break;
          case 4: h[a][0] = v0 - I * v2; h[a][1] = v1 + I * v3; break;
          case 5: h[a][0] = v0 + I * v2; h[a][1] = v1 - I * v3; break;
          case 6: h[a][0] = v2; h[a][1] = v3; break;
          case 7: h[a][0] = v0; h[a][1] = v1; break;
        }
      }
      const T* u = dir == 0 ? U + 18 * ((long)mu * l->V + s) : U + 18 * ((long)mu * l->V + sn);
      mul_u<T>(u, h, r, dir == 1);
      if (mu == 3) {
        bool wrap = dir == 0 ? c[3] == l->L[3] - 1 : c[3] == 0;
        T f = wrap ? (T)(2 * l->tbc) : (T)2;
        for (int a = 0; a < 3; a++) {
          r[a][0] *= f;
          r[a][1] *= f;
        }
      }
      for (int a = 0; a < 3; a++) {
        cx<T> r0 = r[a][0], r1 = r[a][1];
        switch (mu * 2 + pd) {
          case 0: acc[a][0] += r0; acc[a][1] += r1; acc[a][2] += I * r1; acc[a][3] += I * r0; break;
          case 1: acc[a][0] += r0; acc[a][1] += r1; acc[a][2] -= I * r1; acc[a][3] -= I * r0; break;
          case 2: acc[a][0] += r0; acc[a][1] += r1; acc[a][2] += r1; acc[a][3] -= r0; break;
          case 3: acc[a][0] += r0; acc[a][1] += r1; acc[a][2] -= r1; acc[a][3] += r0; break;
          case 4: acc[a][0] += r0; acc[a][1] += r1; acc[a][2] += I * r0; acc[a][3] -= I * r1; break;
          case 5: acc[a][0] += r0; acc[a][1] += r1; acc[a][2] -= I * r0; acc[a][3] += I * r1; break;
          case 6: acc[a][2] += r0; acc[a][3] += r1; break;
          case 7: acc[a][0] += r0; acc[a][1] += r1; break;
        }
      }
    }
  }
}

// psi <- A^-1 psi with the per-site packed clover: rotate to the chiral basis
// without the factor 1/2, multiply each 6-vector by its packed Hermitian 6x6
// (a[0..5] real diagonal, a[6+2n], a[7+2n] = upper-triangle entry n in the
// order (0,1),(0,2),...,(4,5)), rotate back (clover_def.h:88-284).
template <typename T>
void clover_site(const T* a72, cx<T> v[3][4]) {
  cx<T> x[2][6], y[2][6];
  for (int a = 0; a < 3; a++) {
    x[0][a] = v[a][0] + v[a][2];
    x[0][3 + a] = v[a][1] + v[a][3];
    x[1][a] = v[a][0] - v[a][2];
    x[1][3 + a] = v[a][1] - v[a][3];
  }
  for (int i = 0; i < 2; i++) {
    const T* A = a72 + 36 * i;
    cx<T> M[6][6];
    int n = 0;
    for (int j = 0; j < 6; j++) M[j][j] = cx<T>(A[j], 0);
    for (int j = 0; j < 6; j++)
      for (int k = j + 1; k < 6; k++, n++) {
        M[j][k] = cx<T>(A[6 + 2 * n], A[7 + 2 * n]);
        M[k][j] = std::conj(M[j][k]);
      }
    for (int j = 0; j < 6; j++) {
      cx<T> acc(0, 0);
      for (int k = 0; k < 6; k++) acc += M[j][k] * x[i][k];
      y[i][j] = acc;
    }
  }
  for (int a = 0; a < 3; a++) {
    v[a][0] = y[0][a] + y[1][a];
    v[a][2] = y[0][a] - y[1][a];
    v[a][1] = y[0][3 + a] + y[1][3 + a];
    v[a][3] = y[0][3 + a] - y[1][3 + a];
  }
}

// ddd_in_{d,s}_: out = in - kappa A^-1 H_block in on the selected blocks
// (ddd_in_d.cc:66-196, ddd_in_s.cc:72-374; out = in + mkappa*tmp, :352-363).
template <typename T>
void ddd_in(const orc_lat* l, T* out, const T* in, int kind, int sel) {
  const T* C = clover<T>(l);
  const T mk = (T)(-l->kappa);
#pragma omp parallel for schedule(static)
  for (long s = 0; s < l->V; s++) {
    if (!selected(l, s, kind, sel)) continue;
    cx<T> acc[3][4];
    hop_site<T>(l, in, s, 1, acc);
    clover_site<T>(C + 72 * s, acc);
    for (int a = 0; a < 3; a++)
      for (int sp = 0; sp < 4; sp++) {
        long o = 24 * s + 8 * a + 2 * sp;
        out[o] = in[o] + mk * acc[a][sp].real();
        out[o + 1] = in[o + 1] + mk * acc[a][sp].imag();
      }
  }
}

// ddd_out_pre_* + ddd_out_pos_*: out += factor A^-1 H_face in on the selected
// blocks, `in` being the field as it was when the faces were packed
// (ddd_out_d.cc:84-235, ddd_out_s.cc:112-629; only face sites change).
// kind 2 = select by domain index with the FP32 packer's half pairing.
template <typename T>
void ddd_out(const orc_lat* l, T* out, const T* in, int kind, int sel, T factor) {
  const bool pair = kind == 2;
  if (pair) kind = 1;
  const T* C = clover<T>(l);
#pragma omp parallel for schedule(static)
  for (long s = 0; s < l->V; s++) {
    if (!selected(l, s, kind, sel)) continue;
    int c[4];
    coords(l, s, c);
    bool face = false;
    for (int mu = 0; mu < 4; mu++)
      if (c[mu] % l->B[mu] == 0 || c[mu] % l->B[mu] == l->B[mu] - 1) face = true;
    if (!face) continue;
    cx<T> acc[3][4];
    hop_site<T>(l, in, s, 2, acc, pair);
    clover_site<T>(C + 72 * s, acc);
    for (int a = 0; a < 3; a++)
      for (int sp = 0; sp < 4; sp++) {
        long o = 24 * s + 8 * a + 2 * sp;
        out[o] += acc[a][sp].real() * factor;
        out[o + 1] += acc[a][sp].imag() * factor;
      }
  }
}

template <typename T>
void copy_sel(const orc_lat* l, T* out, const T* in, int colour) {
  for (long s = 0; s < l->V; s++)
    if (selected(l, s, 0, colour)) std::memcpy(out + 24 * s, in + 24 * s, 24 * sizeof(T));
}
template <typename T>
void zero_sel(const orc_lat* l, T* out, int colour) {
  for (long s = 0; s < l->V; s++)
    if (selected(l, s, 0, colour)) std::memset(out + 24 * s, 0, 24 * sizeof(T));
}

// jinv_ddd_in_s_noprl_ (static_solver.cc:65-140): nm Richardson steps on
// D_block for the blocks of one colour; x0 = 2b - D b, x <- x + (b - D x).
void jinv_s(const orc_lat* l, float* x, const float* b, int colour, int nm, std::vector<float>& qs) {
  ddd_in<float>(l, qs.data(), b, 0, colour);
#pragma omp parallel for schedule(static)
  for (long s = 0; s < l->V; s++) {
    if (!selected(l, s, 0, colour)) continue;
    for (int j = 0; j < 24; j++) x[24 * s + j] = 2.0f * b[24 * s + j] - qs[24 * s + j];
  }
  for (int it = 1; it < nm; it++) {
    ddd_in<float>(l, qs.data(), x, 0, colour);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < l->V; s++) {
      if (!selected(l, s, 0, colour)) continue;
      for (int j = 0; j < 24; j++) x[24 * s + j] = x[24 * s + j] + (b[24 * s + j] - qs[24 * s + j]);
    }
  }
}

// s_c <- s_c + (in_c - tmp_c)   (accum_addsub_vols_s_noprl_, qws.cc:747-773)
void accum_addsub(const orc_lat* l, float* s, const float* in, const float* tmp, int colour) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < l->V; i++) {
    if (!selected(l, i, 0, colour)) continue;
    for (int j = 0; j < 24; j++) s[24 * i + j] += in[24 * i + j] - tmp[24 * i + j];
  }
}

bool sap_wrap(const orc_lat* l) { return l->NB[1] == 1 || l->NB[2] == 1 || l->NB[3] == 1; }

// The alternating sweeps shared by prec_ddd_s_ and prec_s_ (qws.cc:802-841,
// 954-965).  q's colour-O half must be zero on entry when the block grid wraps
// onto itself in y, z or t (qws.cc:806-808).
void sap_sweeps(const orc_lat* l, float* s, float* q, const float* in, int nsap, int nm,
                std::vector<float>& qs, std::vector<float>& snap, std::vector<float>& tmp) {
  const float kf = (float)l->kappa;
  const size_t nb = sizeof(float) * 24 * l->V;
  for (int isap = 0; isap < nsap; isap++) {
    for (int e = 0; e < 2; e++) {  // colour e, then colour 1-e
      int o = 1 - e;
      jinv_s(l, q, s, e, nm, qs);
      std::memcpy(snap.data(), q, nb);               // ddd_out_pre_s_(q, o)
      ddd_in<float>(l, tmp.data(), q, 0, e);         // q[o] = D_blk q[e]
      accum_addsub(l, s, in, tmp.data(), e);
      ddd_out<float>(l, s, snap.data(), 0, o, kf);   // ddd_out_pos_s_(s[o], q, o, kappa)
    }
  }
}

}  // namespace

extern "C" {

orc_lat* orc_create(const int L[4], const int NB[4], int tbc) {
  orc_lat* l = new orc_lat();
  l->V = 1;
  for (int mu = 0; mu < 4; mu++) {
    l->L[mu] = L[mu];
    l->NB[mu] = NB[mu];
    l->B[mu] = L[mu] / NB[mu];
    l->V *= L[mu];
  }
  l->tbc = tbc;
  l->kappa = 0;
  l->Ud.assign(4 * 18 * l->V, 0.0);
  l->Us.assign(4 * 18 * l->V, 0.0f);
  l->Cd.assign(72 * l->V, 0.0);
  l->Cs.assign(72 * l->V, 0.0f);
  return l;
}
void orc_destroy(orc_lat* l) { delete l; }
void orc_set_kappa(orc_lat* l, double kappa) { l->kappa = kappa; }
long orc_volume(const orc_lat* l) { return l->V; }

void orc_set_gauge_d(orc_lat* l, const double* U) {
  std::memcpy(l->Ud.data(), U, sizeof(double) * l->Ud.size());
  for (size_t i = 0; i < l->Us.size(); i++) l->Us[i] = (float)U[i];
}
void orc_set_clover_d(orc_lat* l, const double* C) {
  std::memcpy(l->Cd.data(), C, sizeof(double) * l->Cd.size());
  for (size_t i = 0; i < l->Cs.size(); i++) l->Cs[i] = (float)C[i];
}
void orc_set_gauge_s(orc_lat* l, const float* U) {
  std::memcpy(l->Us.data(), U, sizeof(float) * l->Us.size());
}
void orc_set_clover_s(orc_lat* l, const float* C) {
  std::memcpy(l->Cs.data(), C, sizeof(float) * l->Cs.size());
}

// main.cc:406-523: seeded mt19937(12345), normal_rand = sqrt(-log u1) *
// (cos, sin)(2 pi u2), link columns 0..1 random, column 2 from the
// determinant-style formula exactly as main.cc:449-473 writes it (including
// its `- u01i+u12r` imaginary parts, so the links are not unitary), clover
// entries Gaussian/10 with 1 added to the six diagonals of each block.
void orc_gen_main_fields(const int Ll[4], const int npe[4], double* U, double* C, int nsrc,
                         double* src) {
  std::mt19937 mt(12345);
  std::uniform_real_distribution<double> rand01(0.0, 1.0);
  auto normal_rand = [&](double* r0, double* r1) {
    double r = std::sqrt(-std::log(rand01(mt)));
    double t = 2.0 * 3.1415926535897932384626433832795028841971 * rand01(mt);
    *r0 = r * std::cos(t);
    *r1 = r * std::sin(t);
  };
  const long Vl = (long)Ll[0] * Ll[1] * Ll[2] * Ll[3];
  std::vector<double> ul(4 * 18 * Vl), cl(72 * Vl), sl(24 * Vl * (nsrc > 0 ? nsrc : 1));
  for (long s = 0; s < Vl; s++) {
    for (int mu = 0; mu < 4; mu++) {
      double* u = &ul[18 * (mu * Vl + s)];  // [row][col][ri]
      double r0, r1;
      for (int c1 = 0; c1 < 3; c1++)
        for (int c2 = 0; c2 < 2; c2++) {
          normal_rand(&r0, &r1);
          u[2 * (3 * c1 + c2)] = r0;  // QWS c[c2][c1] = U[row c1][col c2]
          u[2 * (3 * c1 + c2) + 1] = r1;
        }
      // QWS names u<ab> = c[a][b] = U[b][a]
      auto R = [&](int a, int b) { return u[2 * (3 * b + a)]; };
      auto Im = [&](int a, int b) { return u[2 * (3 * b + a) + 1]; };
      double u00r = R(0, 0), u00i = Im(0, 0), u01r = R(0, 1), u01i = Im(0, 1), u02r = R(0, 2), u02i = Im(0, 2);
      double u10r = R(1, 0), u10i = Im(1, 0), u11r = R(1, 1), u11i = Im(1, 1), u12r = R(1, 2), u12i = Im(1, 2);
      // c[2][k] = U[k][2]
      u[2 * (3 * 0 + 2)] = u01r * u12r - u01i * u12i - u02r * u11r + u02i * u11i;
      u[2 * (3 * 1 + 2)] = u02r * u10r - u02i * u10i - u00r * u12r + u00i * u12i;
      u[2 * (3 * 2 + 2)] = u00r * u11r - u00i * u11i - u01r * u10r + u01i * u10i;
      u[2 * (3 * 0 + 2) + 1] = -u01r * u12i - u01i + u12r + u02r * u11i + u02i * u11r;
      u[2 * (3 * 1 + 2) + 1] = -u02r * u10i - u02i + u10r + u00r * u12i + u00i * u12r;
      u[2 * (3 * 2 + 2) + 1] = -u00r * u11i - u00i + u11r + u01r * u10i + u01i * u10r;
    }
  }
  for (long s = 0; s < Vl; s++) {
    double* c = &cl[72 * s];
    for (int j = 0; j < 2; j++) {
      for (int k = 0; k < 18; k++) {
        double r0, r1;
        normal_rand(&r0, &r1);
        c[36 * j + 2 * k] = r0 / (double)10;
        c[36 * j + 2 * k + 1] = r1 / (double)10;
      }
      for (int k = 0; k < 6; k++) c[36 * j + k] += 1;
    }
  }
  for (int n = 0; n < nsrc; n++)
    for (long s = 0; s < Vl; s++)
      for (int c = 0; c < 3; c++)
        for (int sp = 0; sp < 4; sp++) {
          double r0, r1;
          normal_rand(&r0, &r1);
          sl[24 * (n * Vl + s) + 8 * c + 2 * sp] = r0;
          sl[24 * (n * Vl + s) + 8 * c + 2 * sp + 1] = r1;
        }
  // tile the local fields over the rank grid
  int L[4];
  for (int mu = 0; mu < 4; mu++) L[mu] = Ll[mu] * npe[mu];
  const long V = (long)L[0] * L[1] * L[2] * L[3];
  for (long g = 0; g < V; g++) {
    long r = g;
    int c[4];
    c[0] = r % L[0]; r /= L[0];
    c[1] = r % L[1]; r /= L[1];
    c[2] = r % L[2];
    c[3] = (int)(r / L[2]);
    long s = (c[0] % Ll[0]) + (long)Ll[0] * ((c[1] % Ll[1]) + (long)Ll[1] * ((c[2] % Ll[2]) + (long)Ll[2] * (c[3] % Ll[3])));
    for (int mu = 0; mu < 4; mu++)
      std::memcpy(&U[18 * (mu * V + g)], &ul[18 * (mu * Vl + s)], 18 * sizeof(double));
    std::memcpy(&C[72 * g], &cl[72 * s], 72 * sizeof(double));
    for (int n = 0; n < nsrc; n++)
      std::memcpy(&src[24 * (n * V + g)], &sl[24 * (n * Vl + s)], 24 * sizeof(double));
  }
}

void orc_ddd_in_d(orc_lat* l, double* out, const double* in, int kind, int sel) {
  ddd_in<double>(l, out, in, kind, sel);
}
void orc_ddd_out_d(orc_lat* l, double* out, const double* in, int kind, int sel, double factor) {
  ddd_out<double>(l, out, in, kind, sel, factor);
}
void orc_ddd_in_s(orc_lat* l, float* out, const float* in, int kind, int sel) {
  ddd_in<float>(l, out, in, kind, sel);
}
void orc_ddd_out_s(orc_lat* l, float* out, const float* in, int kind, int sel, float factor) {
  ddd_out<float>(l, out, in, kind, sel, factor);
}

// ddd_d_ (qws.cc:625-632): for each domain, block-interior part then faces.
void orc_ddd_d(orc_lat* l, double* out, const double* in) {
  for (int d = 0; d < 2; d++) {
    ddd_in<double>(l, out, in, 1, d);
    ddd_out<double>(l, out, in, 1, d, -l->kappa);
  }
}
// ddd_s_ (qws.cc:634-644): ddd_eo_s_ on domain_e then domain_o.
void orc_ddd_s(orc_lat* l, float* out, const float* in) {
  for (int c = 0; c < 2; c++) {
    ddd_in<float>(l, out, in, 0, c);
    ddd_out<float>(l, out, in, 0, c, (float)(-l->kappa));
  }
}

// clvd_vm_/clv_s_ semantics on every site (qws.cc:390-425)
void orc_clover_d(orc_lat* l, double* v) {
#pragma omp parallel for schedule(static)
  for (long s = 0; s < l->V; s++) {
    cx<double> a[3][4];
    for (int c = 0; c < 3; c++)
      for (int sp = 0; sp < 4; sp++) a[c][sp] = cx<double>(v[24 * s + 8 * c + 2 * sp], v[24 * s + 8 * c + 2 * sp + 1]);
    clover_site<double>(l->Cd.data() + 72 * s, a);
    for (int c = 0; c < 3; c++)
      for (int sp = 0; sp < 4; sp++) {
        v[24 * s + 8 * c + 2 * sp] = a[c][sp].real();
        v[24 * s + 8 * c + 2 * sp + 1] = a[c][sp].imag();
      }
  }
}
void orc_clover_s(orc_lat* l, float* v) {
#pragma omp parallel for schedule(static)
  for (long s = 0; s < l->V; s++) {
    cx<float> a[3][4];
    for (int c = 0; c < 3; c++)
      for (int sp = 0; sp < 4; sp++) a[c][sp] = cx<float>(v[24 * s + 8 * c + 2 * sp], v[24 * s + 8 * c + 2 * sp + 1]);
    clover_site<float>(l->Cs.data() + 72 * s, a);
    for (int c = 0; c < 3; c++)
      for (int sp = 0; sp < 4; sp++) {
        v[24 * s + 8 * c + 2 * sp] = a[c][sp].real();
        v[24 * s + 8 * c + 2 * sp + 1] = a[c][sp].imag();
      }
  }
}

void orc_jinv_s(orc_lat* l, float* x, const float* b, int colour, int nm) {
  std::vector<float> qs(24 * l->V, 0.0f);
  jinv_s(l, x, b, colour, nm, qs);
}

// prec_ddd_s_ (qws.cc:776-926): out = D M_SAP in.
void orc_prec_ddd_s(orc_lat* l, float* out, const float* in, int nsap, int nm) {
  const long n = 24 * l->V;
  std::vector<float> s(in, in + n), q(n, 0.0f), qs(n, 0.0f), snap(n), tmp(n, 0.0f);
  const float kf = (float)l->kappa, mkf = (float)(-l->kappa);
  const int E = 0, O = 1;
  const bool wrap = sap_wrap(l);
  if (wrap) zero_sel(l, q.data(), O);
  sap_sweeps(l, s.data(), q.data(), in, nsap, nm, qs, snap, tmp);
  if (wrap) zero_sel(l, q.data(), O);
  jinv_s(l, q.data(), s.data(), E, nm, qs);
  std::memcpy(snap.data(), q.data(), sizeof(float) * n);  // ddd_out_pre_s_(q, O)
  ddd_in<float>(l, out, q.data(), 0, E);
  if (wrap) {  // qws.cc:860-891
    ddd_out<float>(l, s.data(), snap.data(), 0, O, kf);
    jinv_s(l, q.data(), s.data(), O, nm, qs);
    std::memcpy(snap.data(), q.data(), sizeof(float) * n);  // pre(q, E)
    ddd_in<float>(l, out, q.data(), 0, O);
    ddd_out<float>(l, out, snap.data(), 0, E, mkf);
    ddd_out<float>(l, out, snap.data(), 0, O, mkf);  // pre(q, O) captures the same q
  } else {     // qws.cc:892-920
    zero_sel(l, out, O);
    ddd_out<float>(l, out, snap.data(), 0, O, mkf);
    for (long i = 0; i < l->V; i++)
      if (selected(l, i, 0, O))
        for (int j = 0; j < 24; j++) s[24 * i + j] -= out[24 * i + j];
    jinv_s(l, q.data(), s.data(), O, nm, qs);
    std::memcpy(snap.data(), q.data(), sizeof(float) * n);  // pre(q, E)
    ddd_in<float>(l, s.data(), q.data(), 0, O);
    for (long i = 0; i < l->V; i++)
      if (selected(l, i, 0, O))
        for (int j = 0; j < 24; j++) out[24 * i + j] += s[24 * i + j];
    ddd_out<float>(l, out, snap.data(), 0, E, mkf);
  }
}

// prec_s_ (qws.cc:929-975): out = M_SAP in.
void orc_prec_s(orc_lat* l, float* out, const float* in, int nsap, int nm) {
  const long n = 24 * l->V;
  std::vector<float> s(in, in + n), q(n, 0.0f), qs(n, 0.0f), snap(n), tmp(n, 0.0f);
  const float kf = (float)l->kappa;
  const bool wrap = sap_wrap(l);
  if (wrap) zero_sel(l, q.data(), 1);
  sap_sweeps(l, s.data(), q.data(), in, nsap, nm, qs, snap, tmp);
  if (wrap) zero_sel(l, out, 1);
  jinv_s(l, out, s.data(), 0, nm, qs);
  std::memcpy(snap.data(), out, sizeof(float) * n);
  ddd_out<float>(l, s.data(), snap.data(), 0, 1, kf);
  jinv_s(l, out, s.data(), 1, nm, qs);
}

double orc_norm2_d(const double* v, long n) {
  double r = 0;
#pragma omp parallel for reduction(+ : r)
  for (long i = 0; i < n; i++) r += v[i] * v[i];
  return r;
}
double orc_norm2_s(const float* v, long n) {
  double r = 0;
#pragma omp parallel for reduction(+ : r)
  for (long i = 0; i < n; i++) r += (double)v[i] * (double)v[i];
  return r;
}

}  // extern "C"

namespace {

// <a,b> = sum conj(a) b over all sites, accumulated in double
template <typename T>
cx<double> cdot(const T* a, const T* b, long n) {
  double re = 0, im = 0;
#pragma omp parallel for reduction(+ : re, im)
  for (long i = 0; i < n; i += 2) {
    re += (double)a[i] * b[i] + (double)a[i + 1] * b[i + 1];
    im += (double)a[i] * b[i + 1] - (double)a[i + 1] * b[i];
  }
  return cx<double>(re, im);
}

}  // namespace

extern "C" {

// bicgstab_precdd_s_ (bicgstab_precdd_s.cc:85-559): right-preconditioned
// BiCGStab on (D M) x = b from x = 0, single-precision scalars.
int orc_bicgstab_precdd_s(orc_lat* l, float* x, const float* b, double tol, int maxiter, int nsap,
                          int nm, double* final_rel) {
  const long n = 24 * l->V;
  std::vector<float> q(n), r(b, b + n), p(b, b + n), t(n), r0(b, b + n);
  std::memset(x, 0, sizeof(float) * n);
  float bnorm = (float)orc_norm2_s(b, n);
  cx<float> rho0(bnorm, 0), rho, beta, omega, alpha, ctmp;
  float rnorm = bnorm;
  int iter, done = maxiter;
  for (iter = 0; iter < maxiter; iter++) {
    orc_prec_ddd_s(l, q.data(), p.data(), nsap, nm);
    cx<double> d = cdot(r0.data(), q.data(), n);
    ctmp = cx<float>((float)d.real(), (float)d.imag());
    alpha = rho0 / ctmp;
    if (std::abs(ctmp) == 0) alpha = 0;
    float ar = alpha.real(), ai = alpha.imag();
    for (long i = 0; i < n; i += 2) {
      float pr = p[i], pi = p[i + 1], qr = q[i], qi = q[i + 1];
      x[i] = x[i] + ar * pr - ai * pi;
      x[i + 1] = x[i + 1] + ar * pi + ai * pr;
      r[i] = r[i] - ar * qr + ai * qi;
      r[i + 1] = r[i + 1] - ar * qi - ai * qr;
    }
    rnorm = (float)orc_norm2_s(r.data(), n);
    if (std::sqrt(rnorm / bnorm) < tol) { done = iter + 1; break; }
    orc_prec_ddd_s(l, t.data(), r.data(), nsap, nm);
    double tt = orc_norm2_s(t.data(), n);
    cx<double> tr = cdot(t.data(), r.data(), n);
    float redu0 = (float)tt, redu1 = (float)tr.real(), redu2 = (float)tr.imag();
    omega = cx<float>(redu1 / redu0, redu2 / redu0);
    if (redu0 == 0) omega = 0;
    ar = omega.real();
    ai = omega.imag();
    for (long i = 0; i < n; i += 2) {
      float rr = r[i], ri = r[i + 1], tr_ = t[i], ti = t[i + 1];
      x[i] = x[i] + ar * rr - ai * ri;
      x[i + 1] = x[i + 1] + ar * ri + ai * rr;
      r[i] = rr - ar * tr_ + ai * ti;
      r[i + 1] = ri - ar * ti - ai * tr_;
    }
    rnorm = (float)orc_norm2_s(r.data(), n);
    cx<double> rr0 = cdot(r0.data(), r.data(), n);
    rho = cx<float>((float)rr0.real(), (float)rr0.imag());
    if (std::sqrt(rnorm / bnorm) < tol) { done = iter + 1; break; }
    beta = alpha * rho / (rho0 * omega);
    rho0 = rho;
    if (std::abs(omega) == 0 || std::abs(rho0) == 0) beta = 0;
    ar = omega.real();
    ai = omega.imag();
    float br = beta.real(), bi = beta.imag();
    for (long i = 0; i < n; i += 2) {
      float cr = p[i] - ar * q[i] + ai * q[i + 1];
      float ci = p[i + 1] - ar * q[i + 1] - ai * q[i];
      p[i] = br * cr - bi * ci + r[i];
      p[i + 1] = br * ci + bi * cr + r[i + 1];
    }
  }
  if (final_rel) *final_rel = std::sqrt((double)rnorm / (double)bnorm);
  return done;
}

}  // extern "C"

namespace {

// approx_inv_dirac_op (bicgstab_dd_mix.cc:76-102) with the renormalising
// converters of reordering.cc:108-204.
int approx_inv(orc_lat* l, double* x, const double* b, double tol_s, int maxiter_s, int nsap, int nm) {
  const long n = 24 * l->V;
  double bn = std::sqrt(orc_norm2_d(b, n));
  double inv = 1.0 / bn;
  std::vector<float> bs(n), ts(n), xs(n);
  for (long i = 0; i < n; i++) bs[i] = (float)(b[i] * inv);
  int it = orc_bicgstab_precdd_s(l, ts.data(), bs.data(), tol_s, maxiter_s, nsap, nm, nullptr);
  orc_prec_s(l, xs.data(), ts.data(), nsap, nm);
  for (long i = 0; i < n; i++) x[i] = ((double)xs[i]) * bn;
  return it;
}

}  // namespace

extern "C" {

// A breakdown planted for tests: at outer iteration g_breakdown_at (0: never)
// the outer loop takes <r0, q> as exactly zero, so the reference's guard
// (alpha = 0 when |<r0, q>| == 0, bicgstab_dd_mix.cc:192) decides the step.
static int g_breakdown_at = 0;
void orc_plant_breakdown(int outer_iter) { g_breakdown_at = outer_iter; }

// bicgstab_dd_mix_ (bicgstab_dd_mix.cc:105-388): flexible BiCGStab in FP64
// with the single-precision SAP-preconditioned solve as variable
// preconditioner; iter runs 1..maxiter-1.
void orc_bicgstab_dd_mix(orc_lat* l, double* x, const double* b, double tol, int maxiter,
                         double tol_s, int maxiter_s, int nsap, int nm, double* stats, double* hist) {
  const long n = 24 * l->V;
  std::vector<double> q(n), r(n), p(n), t(n), u(n), r0(n);
  if (hist)
    for (int i = 0; i < 2 * maxiter; i++) hist[i] = NAN;
  orc_ddd_d(l, q.data(), x);
  for (long i = 0; i < n; i++) {
    r[i] = b[i] - q[i];
    p[i] = r[i];
    r0[i] = r[i];
  }
  double bnorm = orc_norm2_d(b, n);
  cx<double> rho0(orc_norm2_d(r.data(), n), 0), rho, beta, omega, alpha, ctmp;
  double rnorm = rho0.real();
  long inner = 0;
  int iter, h = 0;
  for (iter = 1; iter < maxiter; iter++) {
    inner += approx_inv(l, u.data(), p.data(), tol_s, maxiter_s, nsap, nm);
    orc_ddd_d(l, q.data(), u.data());
    ctmp = cdot(r0.data(), q.data(), n);
    if (iter == g_breakdown_at) ctmp = 0;
    alpha = rho0 / ctmp;
    if (std::abs(ctmp) == 0) alpha = 0;
    double ar = alpha.real(), ai = alpha.imag();
    for (long i = 0; i < n; i += 2) {
      x[i] = x[i] + ar * u[i] - ai * u[i + 1];
      x[i + 1] = x[i + 1] + ar * u[i + 1] + ai * u[i];
      r[i] = r[i] - ar * q[i] + ai * q[i + 1];
      r[i + 1] = r[i + 1] - ar * q[i + 1] - ai * q[i];
    }
    rnorm = orc_norm2_d(r.data(), n);
    if (hist) hist[h++] = std::sqrt(rnorm / bnorm);
    if (std::sqrt(rnorm / bnorm) < tol) break;
    inner += approx_inv(l, u.data(), r.data(), tol_s, maxiter_s, nsap, nm);
    orc_ddd_d(l, t.data(), u.data());
    double tt = orc_norm2_d(t.data(), n);
    cx<double> tr = cdot(t.data(), r.data(), n);
    omega = cx<double>(tr.real() / tt, tr.imag() / tt);
    if (tt == 0) omega = 0;
    ar = omega.real();
    ai = omega.imag();
    for (long i = 0; i < n; i += 2) {
      x[i] = x[i] + ar * u[i] - ai * u[i + 1];
      x[i + 1] = x[i + 1] + ar * u[i + 1] + ai * u[i];
      r[i] = r[i] - ar * t[i] + ai * t[i + 1];
      r[i + 1] = r[i + 1] - ar * t[i + 1] - ai * t[i];
    }
    rnorm = orc_norm2_d(r.data(), n);
    if (hist) hist[h++] = std::sqrt(rnorm / bnorm);
    if (std::sqrt(rnorm / bnorm) < tol) break;
    rho = cdot(r0.data(), r.data(), n);
    beta = alpha * rho / (rho0 * omega);
    rho0 = rho;
    if (std::abs(omega) == 0 || std::abs(rho0) == 0) beta = 0;
    ar = omega.real();
    ai = omega.imag();
    double br = beta.real(), bi = beta.imag();
    for (long i = 0; i < n; i += 2) {
      double cr = p[i] - ar * q[i] + ai * q[i + 1];
      double ci = p[i + 1] - ar * q[i + 1] - ai * q[i];
      p[i] = br * cr - bi * ci + r[i];
      p[i + 1] = br * ci + bi * cr + r[i + 1];
    }
  }
  if (stats) {
    stats[0] = iter;
    stats[1] = (double)inner;
    stats[2] = rnorm / bnorm;
  }
}

}  // extern "C"

namespace {

// assign_mult_mSAP_s_h_ in exact(er) arithmetic: prec_s_ with nsap-1 sweeps
void prec_s_h_fp32(orc_lat* l, float* out, const float* in, int nsap, int nm) {
  orc_prec_s(l, out, in, nsap - 1, nm);
}

}  // namespace

extern "C" {

// bicgstab_precdd_s_h_ (bicgstab_precdd_s_h.cc:83-369): flexible BiCGStab,
// w = M p, q = D w, x += alpha w, breakdown guards |ctmp| <= 1e-15 and
// |t|^2 <= 1e-30 (:165, :250).
int orc_bicgstab_precdd_s_h(orc_lat* l, float* x, const float* b, double tol, int maxiter,
                            int nsap, int nm, double* final_rel) {
  const long n = 24 * l->V;
  std::vector<float> q(n), r(b, b + n), p(b, b + n), t(n), r0(b, b + n), w(n);
  std::memset(x, 0, sizeof(float) * n);
  float bnorm = (float)orc_norm2_s(b, n);
  cx<float> rho0(bnorm, 0), rho, beta, omega, alpha, ctmp;
  float rnorm = bnorm;
  int done = maxiter;
  for (int iter = 0; iter < maxiter; iter++) {
    prec_s_h_fp32(l, w.data(), p.data(), nsap, nm);
    orc_ddd_s(l, q.data(), w.data());
    cx<double> d = cdot(r0.data(), q.data(), n);
    ctmp = cx<float>((float)d.real(), (float)d.imag());
    alpha = rho0 / ctmp;
    if (std::abs(ctmp) <= 1e-15f) alpha = 0;
    float ar = alpha.real(), ai = alpha.imag();
    for (long i = 0; i < n; i += 2) {
      x[i] += ar * w[i] - ai * w[i + 1];
      x[i + 1] += ar * w[i + 1] + ai * w[i];
      r[i] += -ar * q[i] + ai * q[i + 1];
      r[i + 1] += -ar * q[i + 1] - ai * q[i];
    }
    rnorm = (float)orc_norm2_s(r.data(), n);
    if (std::sqrt(rnorm / bnorm) < tol) { done = iter + 1; break; }
    prec_s_h_fp32(l, w.data(), r.data(), nsap, nm);
    orc_ddd_s(l, t.data(), w.data());
    double tt = orc_norm2_s(t.data(), n);
    cx<double> tr = cdot(t.data(), r.data(), n);
    float redu0 = (float)tt, redu1 = (float)tr.real(), redu2 = (float)tr.imag();
    omega = cx<float>(redu1 / redu0, redu2 / redu0);
    if (redu0 <= 1e-30f) omega = 0;
    ar = omega.real();
    ai = omega.imag();
    for (long i = 0; i < n; i += 2) {
      x[i] += ar * w[i] - ai * w[i + 1];
      x[i + 1] += ar * w[i + 1] + ai * w[i];
      r[i] += -ar * t[i] + ai * t[i + 1];
      r[i + 1] += -ar * t[i + 1] - ai * t[i];
    }
    rnorm = (float)orc_norm2_s(r.data(), n);
    if (std::sqrt(rnorm / bnorm) < tol) { done = iter + 1; break; }
    cx<double> rr0 = cdot(r0.data(), r.data(), n);
    rho = cx<float>((float)rr0.real(), (float)rr0.imag());
    beta = alpha * rho / (rho0 * omega);
    rho0 = rho;
    if (std::abs(omega) == 0 || std::abs(rho0) == 0) beta = 0;
    ar = omega.real();
    ai = omega.imag();
    float br = beta.real(), bi = beta.imag();
    for (long i = 0; i < n; i += 2) {
      float cr = p[i] - ar * q[i] + ai * q[i + 1];
      float ci = p[i + 1] - ar * q[i + 1] - ai * q[i];
      p[i] = br * cr - bi * ci + r[i];
      p[i + 1] = br * ci + bi * cr + r[i + 1];
    }
  }
  if (final_rel) *final_rel = std::sqrt((double)rnorm / (double)bnorm);
  return done;
}

// bicgstab_dd_mix2_hf_ (bicgstab_dd_mix2_hf.cc:110-373) around it: the
// approximate inverse has no trailing prec_s_ (approx_inv_dirac_op_hf,
// :88-107); iter = 0..maxiter-1 and conviter = the iteration of convergence.
void orc_bicgstab_dd_mix2_hf(orc_lat* l, double* x, const double* b, double tol, int maxiter,
                             double tol_s, int maxiter_s, int nsap, int nm, double* stats) {
  const long n = 24 * l->V;
  std::vector<double> q(n), r(n), p(n), t(n), u(n), r0(n);
  std::vector<float> bs(n), xs(n);
  auto approx = [&](double* out, const double* in) {
    double bn = std::sqrt(orc_norm2_d(in, n)), inv = 1.0 / bn;
    for (long i = 0; i < n; i++) bs[i] = (float)(in[i] * inv);
    int it = orc_bicgstab_precdd_s_h(l, xs.data(), bs.data(), tol_s, maxiter_s, nsap, nm, nullptr);
    for (long i = 0; i < n; i++) out[i] = (double)xs[i] * bn;
    return it;
  };
  orc_ddd_d(l, q.data(), x);
  for (long i = 0; i < n; i++) r[i] = p[i] = r0[i] = b[i] - q[i];
  double bnorm = orc_norm2_d(b, n);
  cx<double> rho0(orc_norm2_d(r.data(), n), 0), rho, beta, omega, alpha, ctmp;
  double rnorm = rho0.real();
  long inner = 0;
  int iter, conv = maxiter;
  for (iter = 0; iter < maxiter; iter++) {
    inner += approx(u.data(), p.data());
    orc_ddd_d(l, q.data(), u.data());
    ctmp = cdot(r0.data(), q.data(), n);
    alpha = rho0 / ctmp;
    if (std::abs(ctmp) == 0) alpha = 0;
    double ar = alpha.real(), ai = alpha.imag();
    for (long i = 0; i < n; i += 2) {
      x[i] += ar * u[i] - ai * u[i + 1];
      x[i + 1] += ar * u[i + 1] + ai * u[i];
      r[i] += -ar * q[i] + ai * q[i + 1];
      r[i + 1] += -ar * q[i + 1] - ai * q[i];
    }
    rnorm = orc_norm2_d(r.data(), n);
    if (std::sqrt(rnorm / bnorm) < tol) { conv = iter; break; }
    inner += approx(u.data(), r.data());
    orc_ddd_d(l, t.data(), u.data());
    double tt = orc_norm2_d(t.data(), n);
    cx<double> tr = cdot(t.data(), r.data(), n);
    omega = cx<double>(tr.real() / tt, tr.imag() / tt);
    if (tt == 0) omega = 0;
    ar = omega.real();
    ai = omega.imag();
    for (long i = 0; i < n; i += 2) {
      x[i] += ar * u[i] - ai * u[i + 1];
      x[i + 1] += ar * u[i + 1] + ai * u[i];
      r[i] += -ar * t[i] + ai * t[i + 1];
      r[i + 1] += -ar * t[i + 1] - ai * t[i];
    }
    rnorm = orc_norm2_d(r.data(), n);
    if (std::sqrt(rnorm / bnorm) < tol) { conv = iter; break; }
    rho = cdot(r0.data(), r.data(), n);
    beta = alpha * rho / (rho0 * omega);
    rho0 = rho;
    if (std::abs(omega) == 0 || std::abs(rho0) == 0) beta = 0;
    ar = omega.real();
    ai = omega.imag();
    double br = beta.real(), bi = beta.imag();
    for (long i = 0; i < n; i += 2) {
      double cr = p[i] - ar * q[i] + ai * q[i + 1];
      double ci = p[i + 1] - ar * q[i + 1] - ai * q[i];
      p[i] = br * cr - bi * ci + r[i];
      p[i + 1] = br * ci + bi * cr + r[i + 1];
    }
  }
  if (stats) {
    stats[0] = conv;
    stats[1] = (double)inner;
    stats[2] = rnorm / bnorm;
  }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Even-odd (site parity) operators, deo_in_d.cc:65-445, deo_out_d.cc:88-286,
// deo_dag_in.cc, deo_dag_out.cc, deo_in_s.cc, deo_out_s.cc, and their
// compositions in qws.cc:518-605.  Sites of parity pe = (x+y+z+t)%2 receive
// hops from the other parity.  "in" hops stay inside the rank's local box
// (L/npe, npe = (NB0/2, NB1, NB2, NB3)); "out" hops cross its faces (halo).
// ---------------------------------------------------------------------------
namespace {

template <typename T>
void deo_t(const orc_lat* l, T* out, const T* in, int pe, int which, int dag, int clov, int mode,
           T factor, const T* in0) {
  const T* C = clover<T>(l);
  int box[4] = {l->L[0] / (l->NB[0] / 2), l->L[1] / l->NB[1], l->L[2] / l->NB[2],
                l->L[3] / l->NB[3]};
#pragma omp parallel for schedule(static)
  for (long s = 0; s < l->V; s++) {
    int c[4];
    coords(l, s, c);
    if (((c[0] + c[1] + c[2] + c[3]) & 1) != pe) continue;
    cx<T> acc[3][4];
    hop_site<T>(l, in, s, which, acc, false, box, dag != 0, true);
    if (clov) clover_site<T>(C + 72 * s, acc);
    for (int a = 0; a < 3; a++)
      for (int sp = 0; sp < 4; sp++) {
        long o = 24 * s + 8 * a + 2 * sp;
        T re = acc[a][sp].real(), im = acc[a][sp].imag();
        if (mode == 0) {  // __store_sc
          out[o] = re;
          out[o + 1] = im;
        } else if (mode == 1) {  // __store_add_sc(out, tmp, factor)
          out[o] += re * factor;
          out[o + 1] += im * factor;
        } else {  // __load_sc(out, in0); __store_add_sc(out, tmp, factor)
          out[o] = in0[o] + re * factor;
          out[o + 1] = in0[o + 1] + im * factor;
        }
      }
  }
}

// parity-pe clover multiplication (clvd_vm_/clv_s_, qws.cc:390-425)
template <typename T>
void clv_parity(const orc_lat* l, T* out, const T* in, int pe) {
  const T* C = clover<T>(l);
#pragma omp parallel for schedule(static)
  for (long s = 0; s < l->V; s++) {
    int c[4];
    coords(l, s, c);
    if (((c[0] + c[1] + c[2] + c[3]) & 1) != pe) continue;
    cx<T> a[3][4];
    for (int cc = 0; cc < 3; cc++)
      for (int sp = 0; sp < 4; sp++)
        a[cc][sp] = cx<T>(in[24 * s + 8 * cc + 2 * sp], in[24 * s + 8 * cc + 2 * sp + 1]);
    clover_site<T>(C + 72 * s, a);
    for (int cc = 0; cc < 3; cc++)
      for (int sp = 0; sp < 4; sp++) {
        out[24 * s + 8 * cc + 2 * sp] = a[cc][sp].real();
        out[24 * s + 8 * cc + 2 * sp + 1] = a[cc][sp].imag();
      }
  }
}

}  // namespace

extern "C" {

void orc_deo_d(orc_lat* l, double* out, const double* in, int pe, int which, int dag, int clov,
               int mode, double factor, const double* in0) {
  deo_t<double>(l, out, in, pe, which, dag, clov, mode, factor, in0);
}
void orc_deo_s(orc_lat* l, float* out, const float* in, int pe, int which, int dag, int clov,
               int mode, float factor, const float* in0) {
  deo_t<float>(l, out, in, pe, which, dag, clov, mode, factor, in0);
}
void orc_clv_d(orc_lat* l, double* out, const double* in, int pe) { clv_parity<double>(l, out, in, pe); }
void orc_clv_s(orc_lat* l, float* out, const float* in, int pe) { clv_parity<float>(l, out, in, pe); }

// mtilde_vm_ (qws.cc:551-556): out_e = in_e - kappa^2 A_ee^-1 H_eo A_oo^-1 H_oe in_e
// (pce = 0, pco = 1 as main.cc:163-164 passes them)
void orc_mtilde_d(orc_lat* l, double* out, const double* in) {
  std::vector<double> tmp(24 * l->V, 0.0);
  deo_t<double>(l, tmp.data(), in, 1, 3, 0, 1, 0, 0.0, nullptr);
  deo_t<double>(l, out, tmp.data(), 0, 3, 0, 1, 2, -l->kappa * l->kappa, in);
}
// mtilde_dag_vm_ (qws.cc:557-565)
void orc_mtilde_dag_d(orc_lat* l, double* out, const double* in) {
  std::vector<double> t0(24 * l->V, 0.0), t1(24 * l->V, 0.0);
  clv_parity<double>(l, t0.data(), in, 0);
  deo_t<double>(l, t1.data(), t0.data(), 1, 3, 1, 1, 0, 0.0, nullptr);
  deo_t<double>(l, out, t1.data(), 0, 3, 1, 0, 2, -l->kappa * l->kappa, in);
}

// bicgstab_vm_ (bicgstab.cc:68-333): BiCGStab on mtilde_vm_ for the even
// parity, iter = 1..maxiter-1, stops when sqrt(|r|^2/|b|^2) < 1e-14 after the
// omega step; returns the iteration count.
int orc_bicgstab_vm(orc_lat* l, double* x, const double* b, int maxiter) {
  const long n = 24 * l->V;
  std::vector<double> q(n, 0.0), r(n, 0.0), p(n, 0.0), t(n, 0.0), r0(n, 0.0);
  auto even = [&](long s) {
    int c[4];
    coords(l, s, c);
    return ((c[0] + c[1] + c[2] + c[3]) & 1) == 0;
  };
  std::vector<char> ev(l->V);
  for (long s = 0; s < l->V; s++) ev[s] = even(s);
  auto dot = [&](const double* a, const double* bb) {
    double re = 0, im = 0;
    for (long s = 0; s < l->V; s++)
      if (ev[s])
        for (int k = 0; k < 24; k += 2) {
          long i = 24 * s + k;
          re += a[i] * bb[i] + a[i + 1] * bb[i + 1];
          im += a[i] * bb[i + 1] - a[i + 1] * bb[i];
        }
    return cx<double>(re, im);
  };
  orc_mtilde_d(l, q.data(), x);
  for (long s = 0; s < l->V; s++)
    if (ev[s])
      for (int k = 0; k < 24; k++) {
        long i = 24 * s + k;
        r[i] = b[i] - q[i];
        p[i] = r0[i] = r[i];
      }
  double bnorm = dot(b, b).real();
  cx<double> rho0(dot(r.data(), r.data()).real(), 0), rho, beta, omega, alpha, ctmp;
  int iter;
  for (iter = 1; iter < maxiter; iter++) {
    orc_mtilde_d(l, q.data(), p.data());
    ctmp = dot(r0.data(), q.data());
    alpha = rho0 / ctmp;
    for (long s = 0; s < l->V; s++)
      if (ev[s])
        for (int k = 0; k < 24; k += 2) {
          long i = 24 * s + k;
          cx<double> xv(x[i], x[i + 1]), pv(p[i], p[i + 1]), rv(r[i], r[i + 1]), qv(q[i], q[i + 1]);
          xv += alpha * pv;
          rv -= alpha * qv;
          x[i] = xv.real(); x[i + 1] = xv.imag();
          r[i] = rv.real(); r[i + 1] = rv.imag();
        }
    orc_mtilde_d(l, t.data(), r.data());
    double tt = dot(t.data(), t.data()).real();
    cx<double> tr = dot(t.data(), r.data());
    omega = cx<double>(tr.real() / tt, tr.imag() / tt);
    for (long s = 0; s < l->V; s++)
      if (ev[s])
        for (int k = 0; k < 24; k += 2) {
          long i = 24 * s + k;
          cx<double> xv(x[i], x[i + 1]), rv(r[i], r[i + 1]), tv(t[i], t[i + 1]);
          xv += omega * rv;
          rv -= omega * tv;
          x[i] = xv.real(); x[i + 1] = xv.imag();
          r[i] = rv.real(); r[i + 1] = rv.imag();
        }
    double rnorm = dot(r.data(), r.data()).real();
    if (std::sqrt(rnorm / bnorm) < 1e-14) break;
    rho = dot(r0.data(), r.data());
    beta = alpha * rho / (rho0 * omega);
    rho0 = rho;
    for (long s = 0; s < l->V; s++)
      if (ev[s])
        for (int k = 0; k < 24; k += 2) {
          long i = 24 * s + k;
          cx<double> pv(p[i], p[i + 1]), qv(q[i], q[i + 1]), rv(r[i], r[i + 1]);
          pv = rv + beta * (pv - omega * qv);
          p[i] = pv.real(); p[i + 1] = pv.imag();
        }
  }
  return iter;
}

// mtdagmt_vm_ (qws.cc:566-571)
void orc_mtdagmt_d(orc_lat* l, double* out, const double* in) {
  std::vector<double> t(24 * l->V, 0.0);
  orc_mtilde_d(l, t.data(), in);
  orc_mtilde_dag_d(l, out, t.data());
}

namespace {
// real inner products over the even sites (the parity the eo solvers use)
struct EvenSites {
  std::vector<long> idx;
  explicit EvenSites(const orc_lat* l) {
    for (long s = 0; s < l->V; s++) {
      int c[4];
      coords(l, s, c);
      if (((c[0] + c[1] + c[2] + c[3]) & 1) == 0) idx.push_back(s);
    }
  }
  double dot(const double* a, const double* b) const {  // Re <a, b>
    double acc = 0;
    for (long s : idx)
      for (int k = 0; k < 24; k++) acc += a[24 * s + k] * b[24 * s + k];
    return acc;
  }
};
}  // namespace

// cg_vm_ (cg.cc:65-172): CG on mtdagmt_vm_ for the even parity, x = initial
// guess in / solution out, iter = 1..maxiter-1, stops when
// sqrt(|r|^2/|b|^2) < 1e-14 after the x/r update; returns the last iter
int orc_cg_vm(orc_lat* l, double* x, const double* b, int maxiter) {
  const long n = 24 * l->V;
  EvenSites ev(l);
  std::vector<double> q(n, 0.0), r(n, 0.0), p(n, 0.0);
  orc_mtdagmt_d(l, q.data(), x);
  for (long s : ev.idx)
    for (int k = 0; k < 24; k++) {
      long i = 24 * s + k;
      r[i] = b[i] - q[i];
      p[i] = r[i];
    }
  const double bnorm = ev.dot(b, b);
  double rho0 = ev.dot(r.data(), r.data());
  int iter;
  for (iter = 1; iter < maxiter; iter++) {
    orc_mtdagmt_d(l, q.data(), p.data());
    const double alpha = rho0 / ev.dot(p.data(), q.data());
    for (long s : ev.idx)
      for (int k = 0; k < 24; k++) {
        long i = 24 * s + k;
        x[i] += alpha * p[i];
        r[i] -= alpha * q[i];
      }
    const double rnorm = ev.dot(r.data(), r.data());
    if (std::sqrt(rnorm / bnorm) < 1e-14) break;
    const double beta = rnorm / rho0;
    rho0 = rnorm;
    for (long s : ev.idx)
      for (int k = 0; k < 24; k++) {
        long i = 24 * s + k;
        p[i] = r[i] + beta * p[i];
      }
  }
  return iter;
}

// mcg_vm_ (mcg.cc:65-219): multi-shift CG, (mtdagmt + sigma_k) x_k = b,
// x_k from zero (X: n natural-layout fields back to back); the shifted
// coefficients follow mcg.cc:141-147 and 196-200; returns the last iter.
// One deliberate difference: a shift whose residual |zeta_k| |r| / |b| is
// below 1e-14 stops being updated.  The reference updates it to the end,
// and once zeta_k underflows to zero its next ratio is 0/0 and the
// solution turns into NaN; before that point the two agree.
int orc_mcg_vm(orc_lat* l, double* X, const double* b, int n, const double* sigma, int maxiter) {
  const long N = 24 * l->V;
  EvenSites ev(l);
  std::vector<double> q(N, 0.0), r(N, 0.0), p(N, 0.0), pp((size_t)N * n, 0.0);
  for (long s : ev.idx)
    for (int k = 0; k < 24; k++) r[24 * s + k] = p[24 * s + k] = b[24 * s + k];
  for (long i = 0; i < N * n; i++) X[i] = 0.0;
  for (int k = 0; k < n; k++)
    for (long i = 0; i < N; i++) pp[(size_t)k * N + i] = r[i];
  const double bnorm = ev.dot(b, b);
  double rho0 = bnorm, alpha0 = 1.0, beta = 0.0;
  std::vector<double> z0(n, 1.0), z1(n, 1.0), z2(n);
  std::vector<char> active(n, 1);
  int iter;
  for (iter = 1; iter < maxiter; iter++) {
    orc_mtdagmt_d(l, q.data(), p.data());
    const double alpha = -rho0 / ev.dot(p.data(), q.data());
    for (long s : ev.idx)
      for (int k = 0; k < 24; k++) r[24 * s + k] += alpha * q[24 * s + k];
    const double rnorm = ev.dot(r.data(), r.data());
    for (int k = 0; k < n; k++) {
      if (!active[k]) continue;
      z2[k] = z1[k] * z0[k] * alpha0 /
              (alpha * beta * (z0[k] - z1[k]) + z0[k] * alpha0 * (1.0 - sigma[k] * alpha));
      const double c = alpha * z2[k] / z1[k];
      double* xk = X + (size_t)k * N;
      const double* pk = pp.data() + (size_t)k * N;
      for (long s : ev.idx)
        for (int j = 0; j < 24; j++) xk[24 * s + j] -= c * pk[24 * s + j];
      if (std::fabs(z2[k]) * std::sqrt(rnorm / bnorm) < 1e-14) active[k] = 0;
    }
    if (std::sqrt(rnorm / bnorm) < 1e-14) break;
    beta = rnorm / rho0;
    rho0 = rnorm;
    for (long s : ev.idx)
      for (int k = 0; k < 24; k++) p[24 * s + k] = r[24 * s + k] + beta * p[24 * s + k];
    for (int k = 0; k < n; k++) {
      if (!active[k]) continue;
      const double d = beta * (z2[k] / z1[k]) * (z2[k] / z1[k]);
      double* pk = pp.data() + (size_t)k * N;
      for (long s : ev.idx)
        for (int j = 0; j < 24; j++) pk[24 * s + j] = d * pk[24 * s + j] + z2[k] * r[24 * s + j];
      z0[k] = z1[k];
      z1[k] = z2[k];
    }
    alpha0 = alpha;
  }
  return iter;
}

}  // extern "C"
