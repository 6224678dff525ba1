// Multi-RHS solvers: the reference's BiCGStab loops (bicgstab_precdd_s.cc:85-559,
// bicgstab_precdd_s_h.cc:83-369, bicgstab_dd_mix.cc:76-388,
// bicgstab_dd_mix2_hf.cc:88-373) run on a context whose spinor fields hold
// G.nr right-hand sides of one gauge field.  Every operator application is
// one launch over all RHS (each link and clover load serves every RHS, see
// lattice.cuh); the scalars alpha, omega, beta are per RHS and reach the
// update kernels as a small device table.  A RHS that has converged is
// frozen: its coefficients are zero from then on, so its iterate is exactly
// the one a single-RHS solve stops at, and the loop runs until every RHS has
// converged or the iteration limit is reached.
#include <cmath>
#include <complex>
#include <cstring>

#include "ctx.h"

namespace qwsg {

namespace {

constexpr int kMax = Ctx::kMaxRhs;

struct Table {
  double v[4 * kMax];
  Table() { std::memset(v, 0, sizeof(v)); }
};

// bicgstab_precdd_s_ / bicgstab_precdd_s_h_ on all RHS.  flexible = false:
// q = prec_ddd_s(p) (right-preconditioned form); true: w = M_h p, q = D w and
// x is updated with w (the half-precision pair's flexible form).  RHS with
// active[r] false on entry (or |b_r| = 0) are left at x_r = 0.  iters[r]: the
// reference's count for each RHS.
int inner_solve(Ctx& c, float* x, const float* b, double tol, int maxiter, int nsap, int nm,
                bool flexible, const bool* active_in, int* iters) {
  const Geom& G = c.G;
  const int nr = G.nr;
  float *q = c.in_q, *r = c.in_r, *p = c.in_p, *t = c.in_t, *r0 = c.in_r0, *w = c.in_w;
  blas_zero<float>(G, x, 0, G.V, c.st);
  blas_bicg_init<float>(G, b, nullptr, r, p, r0, c.d_res, c.rb, c.st);
  const double* h = c.fetch(4 * nr);
  using cf = std::complex<float>;
  float bnorm[kMax], rnorm[kMax];
  cf rho0[kMax], rho[kMax], alpha[kMax], omega[kMax], beta[kMax];
  bool act[kMax];
  int nact = 0;
  for (int k = 0; k < nr; k++) {
    bnorm[k] = (float)h[4 * k];
    rnorm[k] = bnorm[k];
    rho0[k] = cf(bnorm[k], 0);
    act[k] = (active_in ? active_in[k] : true) && bnorm[k] > 0;
    iters[k] = act[k] ? maxiter : 0;
    nact += act[k];
  }
  int iter;
  for (iter = 0; iter < maxiter && nact > 0; iter++) {
    c.n_inner_iter++;
    if (flexible) {
      prec_s_h(c, w, p, nsap, nm);
      dslash_full_s(c, q, w);
    } else {
      prec_ddd_s(c, q, p, nsap, nm);
    }
    blas_cdot<float>(G, r0, q, c.d_res, c.rb, c.st);
    h = c.fetch(4 * nr);
    Table ta;
    for (int k = 0; k < nr; k++) {
      alpha[k] = 0;
      if (!act[k]) continue;
      const cf ctmp((float)h[4 * k], (float)h[4 * k + 1]);
      alpha[k] = rho0[k] / ctmp;
      if (flexible ? std::abs(ctmp) <= 1e-15f : std::abs(ctmp) == 0) alpha[k] = 0;
      ta.v[4 * k] = alpha[k].real();
      ta.v[4 * k + 1] = alpha[k].imag();
    }
    blas_bicg_update<float>(G, x, r, flexible ? w : p, q, 0, 0, nullptr, c.d_res, c.rb, c.st,
                            c.put_coefs(ta.v));
    h = c.fetch(4 * nr);
    for (int k = 0; k < nr; k++) {
      if (!act[k]) continue;
      rnorm[k] = (float)h[4 * k];
      if (!std::isfinite(rnorm[k])) throw Error(3, "solver: non-finite residual norm");
      if (std::sqrt(rnorm[k] / bnorm[k]) < tol) {
        iters[k] = iter + 1;
        act[k] = false;
        nact--;
      }
    }
    if (nact == 0) break;
    if (flexible) {
      prec_s_h(c, w, r, nsap, nm);
      dslash_full_s(c, t, w);
    } else {
      prec_ddd_s(c, t, r, nsap, nm);
    }
    blas_norm_cdot<float>(G, t, r, c.d_res, c.rb, c.st);
    h = c.fetch(4 * nr);
    Table to;
    for (int k = 0; k < nr; k++) {
      omega[k] = 0;
      if (!act[k]) continue;
      const float redu0 = (float)h[4 * k], redu1 = (float)h[4 * k + 1], redu2 = (float)h[4 * k + 2];
      omega[k] = cf(redu1 / redu0, redu2 / redu0);
      if (flexible ? redu0 <= 1e-30f : redu0 == 0) omega[k] = 0;
      to.v[4 * k] = omega[k].real();
      to.v[4 * k + 1] = omega[k].imag();
    }
    blas_bicg_update<float>(G, x, r, flexible ? w : r, t, 0, 0, r0, c.d_res, c.rb, c.st,
                            c.put_coefs(to.v));
    h = c.fetch(4 * nr);
    Table tb;
    for (int k = 0; k < nr; k++) {
      if (!act[k]) continue;  // frozen: p = r (beta = omega = 0), harmless
      rnorm[k] = (float)h[4 * k];
      if (!std::isfinite(rnorm[k])) throw Error(3, "solver: non-finite residual norm");
      rho[k] = cf((float)h[4 * k + 1], (float)h[4 * k + 2]);
      if (std::sqrt(rnorm[k] / bnorm[k]) < tol) {
        iters[k] = iter + 1;
        act[k] = false;
        nact--;
        continue;
      }
      beta[k] = alpha[k] * rho[k] / (rho0[k] * omega[k]);
      rho0[k] = rho[k];
      if (std::abs(omega[k]) == 0 || std::abs(rho0[k]) == 0) beta[k] = 0;
      tb.v[4 * k] = beta[k].real();
      tb.v[4 * k + 1] = beta[k].imag();
      tb.v[4 * k + 2] = omega[k].real();
      tb.v[4 * k + 3] = omega[k].imag();
    }
    if (nact == 0) break;
    blas_bicg_p<float>(G, p, r, q, 0, 0, 0, 0, c.st, c.put_coefs(tb.v));
  }
  c.check_launch("bicgstab_precdd_s (multi-RHS)");
  int most = 0;
  for (int k = 0; k < nr; k++) most = iters[k] > most ? iters[k] : most;
  return most;
}

// approx_inv_dirac_op / approx_inv_dirac_op_hf on all RHS: each RHS is
// normalised by its own norm (fermi_reorder_d2s_dd_renorm_); RHS with
// active[r] false get x_r = 0 and cost no inner iterations.
int approx_inv(Ctx& c, double* x, const double* b, double tol_s, int maxiter_s, int nsap, int nm,
               bool hf, const bool* active) {
  const int nr = c.G.nr;
  blas_norm2<double>(c.G, b, c.d_res, c.rb, c.st);
  const double* h = c.fetch(4 * nr);
  Table down, up;
  bool act[kMax];
  for (int k = 0; k < nr; k++) {
    const double bn = std::sqrt(h[4 * k]);
    act[k] = active[k] && bn > 0;
    down.v[4 * k] = act[k] ? 1.0 / bn : 0.0;
    up.v[4 * k] = act[k] ? bn : 0.0;
  }
  blas_d2s(c.G, c.ai_b, b, 0, c.st, c.put_coefs(down.v));
  int its[kMax], it;
  if (hf) {
    it = inner_solve(c, c.ai_x, c.ai_b, tol_s, maxiter_s, nsap, nm, true, act, its);
  } else {
    it = inner_solve(c, c.ai_t, c.ai_b, tol_s, maxiter_s, nsap, nm, false, act, its);
    prec_s(c, c.ai_x, c.ai_t, nsap, nm);
  }
  blas_s2d(c.G, x, c.ai_x, 0, c.st, c.put_coefs(up.v));
  return it;
}

// the flexible FP64 outer BiCGStab on all RHS, iter in [iter_begin, iter_end);
// conv[r]: the reference's conviter of each RHS (iter_end when not reached).
// RHS r stops at its own tolerance when the handle has per-RHS ones.
void outer_loop(Ctx& c, double* x, const double* b, double tol, int iter_begin, int iter_end,
                double tol_s, int maxiter_s, int nsap, int nm, bool hf, const bool* active_in,
                int* conv, long* inner_out, double* rel_out) {
  const Geom& G = c.G;
  const int nr = G.nr;
  double *q = c.out_q, *r = c.out_r, *p = c.out_p, *t = c.out_t, *u = c.out_u, *r0 = c.out_r0;
  using cd = std::complex<double>;
  dslash_full_d(c, q, x);
  blas_bicg_init<double>(G, b, q, r, p, r0, c.d_res, c.rb, c.st);
  const double* h = c.fetch(4 * nr);
  double bnorm[kMax], rnorm[kMax];
  cd rho0[kMax], rho[kMax], alpha[kMax], omega[kMax], beta[kMax];
  bool act[kMax];
  int nact = 0;
  for (int k = 0; k < nr; k++) {
    bnorm[k] = h[4 * k];
    rnorm[k] = h[4 * k + 1];
    rho0[k] = cd(h[4 * k + 1], 0);
    act[k] = active_in[k] && bnorm[k] > 0;
    conv[k] = iter_end;
    nact += act[k];
  }
  double tolk[kMax];  // each RHS's own stopping tolerance
  for (int k = 0; k < nr; k++) tolk[k] = c.rhs_tols.empty() ? tol : c.rhs_tols[k];
  long inner = 0;
  for (int iter = iter_begin; iter < iter_end && nact > 0; iter++) {
    inner += approx_inv(c, u, p, tol_s, maxiter_s, nsap, nm, hf, act);
    dslash_full_d(c, q, u);
    blas_cdot<double>(G, r0, q, c.d_res, c.rb, c.st);
    h = c.fetch(4 * nr);
    Table ta;
    for (int k = 0; k < nr; k++) {
      alpha[k] = 0;
      if (!act[k]) continue;
      const cd ctmp(h[4 * k], h[4 * k + 1]);
      alpha[k] = rho0[k] / ctmp;
      if (std::abs(ctmp) == 0) alpha[k] = 0;
      ta.v[4 * k] = alpha[k].real();
      ta.v[4 * k + 1] = alpha[k].imag();
    }
    blas_bicg_update<double>(G, x, r, u, q, 0, 0, nullptr, c.d_res, c.rb, c.st,
                             c.put_coefs(ta.v));
    h = c.fetch(4 * nr);
    for (int k = 0; k < nr; k++) {
      if (!act[k]) continue;
      rnorm[k] = h[4 * k];
      if (!std::isfinite(rnorm[k])) throw Error(3, "solver: non-finite residual norm");
      if (std::sqrt(rnorm[k] / bnorm[k]) < tolk[k]) {
        conv[k] = iter;
        act[k] = false;
        nact--;
      }
    }
    if (nact == 0) break;
    inner += approx_inv(c, u, r, tol_s, maxiter_s, nsap, nm, hf, act);
    dslash_full_d(c, t, u);
    blas_norm_cdot<double>(G, t, r, c.d_res, c.rb, c.st);
    h = c.fetch(4 * nr);
    Table to;
    for (int k = 0; k < nr; k++) {
      omega[k] = 0;
      if (!act[k]) continue;
      omega[k] = cd(h[4 * k + 1] / h[4 * k], h[4 * k + 2] / h[4 * k]);
      if (h[4 * k] == 0) omega[k] = 0;
      to.v[4 * k] = omega[k].real();
      to.v[4 * k + 1] = omega[k].imag();
    }
    blas_bicg_update<double>(G, x, r, u, t, 0, 0, r0, c.d_res, c.rb, c.st, c.put_coefs(to.v));
    h = c.fetch(4 * nr);
    Table tb;
    for (int k = 0; k < nr; k++) {
      if (!act[k]) continue;
      rnorm[k] = h[4 * k];
      if (!std::isfinite(rnorm[k])) throw Error(3, "solver: non-finite residual norm");
      rho[k] = cd(h[4 * k + 1], h[4 * k + 2]);
      if (std::sqrt(rnorm[k] / bnorm[k]) < tolk[k]) {
        conv[k] = iter;
        act[k] = false;
        nact--;
        continue;
      }
      beta[k] = alpha[k] * rho[k] / (rho0[k] * omega[k]);
      rho0[k] = rho[k];
      if (std::abs(omega[k]) == 0 || std::abs(rho0[k]) == 0) beta[k] = 0;
      tb.v[4 * k] = beta[k].real();
      tb.v[4 * k + 1] = beta[k].imag();
      tb.v[4 * k + 2] = omega[k].real();
      tb.v[4 * k + 3] = omega[k].imag();
    }
    if (nact == 0) break;
    blas_bicg_p<double>(G, p, r, q, 0, 0, 0, 0, c.st, c.put_coefs(tb.v));
  }
  *inner_out += inner;
  for (int k = 0; k < nr; k++) rel_out[k] = bnorm[k] > 0 ? std::sqrt(rnorm[k] / bnorm[k]) : 0;
}

}  // namespace

void true_residual_mrhs(Ctx& c, const double* x, const double* b, double* rel) {
  c.ensure_outer();
  dslash_full_d(c, c.out_t, x);
  blas_bicg_init<double>(c.G, b, c.out_t, c.out_q, c.out_p, c.out_r0, c.d_res, c.rb, c.st);
  const double* h = c.fetch(4 * c.G.nr);
  for (int k = 0; k < c.G.nr; k++) rel[k] = h[4 * k] > 0 ? std::sqrt(h[4 * k + 1] / h[4 * k]) : 0;
}

int bicgstab_precdd_s_mrhs(Ctx& c, float* x, const float* b, double tol, int maxiter, int nsap,
                           int nm, int* iters) {
  Region region_("bicgstab_precdd_s");
  c.ensure_inner();
  return inner_solve(c, x, b, tol, maxiter, nsap, nm, false, nullptr, iters);
}

int bicgstab_precdd_s_h_mrhs(Ctx& c, float* x, const float* b, double tol, int maxiter, int nsap,
                             int nm, int* iters) {
  Region region_("bicgstab_precdd_s_h");
  c.ensure_hp();
  return inner_solve(c, x, b, tol, maxiter, nsap, nm, true, nullptr, iters);
}

// bicgstab_dd_mix_ on all RHS (iter = 1 .. maxiter-1); per-RHS statistics
void bicgstab_dd_mix_mrhs(Ctx& c, double* x, const double* b, double tol, int maxiter,
                          double tol_s, int maxiter_s, int nsap, int nm, SolveStats* st) {
  Region region_("bicgstab_dd_mix");
  c.ensure_outer();
  const int nr = c.G.nr;
  bool act[kMax];
  int conv[kMax];
  double rel[kMax];
  for (int k = 0; k < nr; k++) act[k] = true;
  long inner = 0;
  outer_loop(c, x, b, tol, 1, maxiter, tol_s, maxiter_s, nsap, nm, false, act, conv, &inner, rel);
  for (int k = 0; k < nr; k++) {
    st[k].outer_iters = conv[k];
    st[k].inner_iters = inner;
    st[k].rel_resid_recursive = rel[k];
    st[k].rel_resid_true = -1;
  }
  c.check_launch("bicgstab_dd_mix (multi-RHS)");
}

// bicgstab_dd_mix2_hf_ on all RHS with reliable restarts: after each pass the
// FP64 true residual of every RHS is recomputed and only the RHS above tol
// are restarted.
void bicgstab_dd_mix2_hf_mrhs(Ctx& c, double* x, const double* b, double tol, int maxiter,
                              double tol_s, int maxiter_s, int nsap, int nm, int reliable,
                              SolveStats* st) {
  Region region_("bicgstab_dd_mix2_hf");
  c.ensure_outer();
  c.ensure_hp();
  const int nr = c.G.nr;
  bool act[kMax];
  int conv[kMax], total[kMax];
  double rel[kMax], truerel[kMax];
  for (int k = 0; k < nr; k++) {
    act[k] = true;
    total[k] = 0;
    truerel[k] = -1;
    rel[k] = 0;
  }
  long inner = 0;
  for (int pass = 0; pass <= reliable; pass++) {
    double rel_pass[kMax];
    outer_loop(c, x, b, tol, 0, maxiter, tol_s, maxiter_s, nsap, nm, true, act, conv, &inner,
               rel_pass);
    int left = 0;
    for (int k = 0; k < nr; k++) {
      if (!act[k]) continue;
      rel[k] = rel_pass[k];
      total[k] += (conv[k] < maxiter ? conv[k] + 1 : maxiter);
    }
    if (reliable <= 0) break;
    true_residual_mrhs(c, x, b, truerel);
    for (int k = 0; k < nr; k++) {
      if (act[k] && truerel[k] < (c.rhs_tols.empty() ? tol : c.rhs_tols[k])) act[k] = false;
      left += act[k];
    }
    if (left == 0) break;
  }
  for (int k = 0; k < nr; k++) {
    st[k].outer_iters = reliable > 0 ? total[k] : conv[k];
    st[k].inner_iters = inner;
    st[k].rel_resid_recursive = rel[k];
    st[k].rel_resid_true = truerel[k];
  }
  c.check_launch("bicgstab_dd_mix2_hf (multi-RHS)");
}

}  // namespace qwsg
