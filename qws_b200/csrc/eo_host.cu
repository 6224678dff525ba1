// Host side of the even-odd (site parity) operator family and its solver
// (deo_*/dee_*/one_minus_*, clvd_vm_/clv_s_, mtilde_vm_, mtilde_dag_vm_,
// mtilde_s_ of qws.cc:390-605 and bicgstab_vm_ of bicgstab.cc:68-333).
// Parity fields live in the library's DD-order planes; a parity-p vector is
// a full field whose other-parity sites are zero.
#include <cmath>
#include <complex>
#include <string>
#include <vector>

#include "ctx.h"

namespace qwsg {

[[noreturn]] void throw_unsupported_eo() {
  throw Error(2, "even-odd operator: unsupported combination of hop set / adjoint / clover / mode");
}

void Ctx::ensure_eo() {
  // each buffer on its own (a failed allocation is retried by the next call)
  for (int i = 0; i < 6; i++)
    if (!eo_d[i]) eo_d[i] = alloc_spinor<double>();
  for (int i = 0; i < 2; i++)
    if (!eo_s[i]) eo_s[i] = alloc_spinor<float>();
}

template <typename R>
static EoArgs<R> eo_args(Ctx& c, int pe);
template <>
EoArgs<double> eo_args<double>(Ctx& c, int pe) {
  EoArgs<double> a{};
  a.G = c.G;
  a.U = c.eoUd ? c.eoUd : c.Ud;
  a.C = c.eoCd ? c.eoCd : c.Cd;
  a.pe = pe;
  return a;
}
template <>
EoArgs<float> eo_args<float>(Ctx& c, int pe) {
  EoArgs<float> a{};
  a.G = c.G;
  a.U = c.eoUs ? c.eoUs : c.Us;
  a.C = c.eoCs ? c.eoCs : c.Cs;
  a.pe = pe;
  return a;
}

template <typename R>
void deo(Ctx& c, R* out, const R* in, int pe, int which, int dag, int clov, int mode,
         double factor, const R* in0) {
  if (pe != 0 && pe != 1) throw Error(1, "parity must be 0 or 1");
  if (mode == 2 && !in0) throw Error(1, "mode 2 needs in0");
  auto a = eo_args<R>(c, pe);
  if (!a.U || !a.C) throw Error(4, "gauge/clover fields not loaded");
  a.src = in;
  a.out = out;
  a.in0 = in0;
  a.coef = (R)factor;
  // the reference's rank box: each rank holds two x-halves (NB = 2*npe0, ...)
  a.box[0] = c.G.L[0] / (c.G.NB[0] / 2);
  for (int mu = 1; mu < 4; mu++) a.box[mu] = c.G.L[mu] / c.G.NB[mu];
  launch_eo<R>(which, dag, clov, mode, a, c.st);
  c.check_launch("deo");
}
template void deo<float>(Ctx&, float*, const float*, int, int, int, int, int, double, const float*);
template void deo<double>(Ctx&, double*, const double*, int, int, int, int, int, double,
                          const double*);

template <typename R>
void clv(Ctx& c, R* out, const R* in, int pe) {
  auto a = eo_args<R>(c, pe);
  if (!a.C) throw Error(4, "clover field not loaded");
  a.src = in;
  a.out = out;
  launch_clv<R>(a, c.st);
  c.check_launch("clv");
}
template void clv<float>(Ctx&, float*, const float*, int);
template void clv<double>(Ctx&, double*, const double*, int);

// mtilde_vm_: out_e = in_e - kappa^2 A_ee^-1 H_eo A_oo^-1 H_oe in_e
// (dee_deo_vm_(pco, pce) then one_minus_dee_deo_vm_(pce, pco))
void mtilde_d(Ctx& c, double* out, const double* in) {
  c.ensure_eo();
  double* tmp = c.eo_d[0];
  deo<double>(c, tmp, in, c.pco, 3, 0, 1, 0, 0.0, nullptr);
  deo<double>(c, out, tmp, c.pce, 3, 0, 1, 2, -c.kappa * c.kappa, in);
  c.n_mtilde++;
}

// mtilde_dag_vm_: clvd_vm2_(pce), dee_deo_dag_vm_(pco, pce), one_minus_deo_dag_vm_(pce, pco)
void mtilde_dag_d(Ctx& c, double* out, const double* in) {
  c.ensure_eo();
  double *t0 = c.eo_d[0], *t1 = c.eo_d[1];
  clv<double>(c, t0, in, c.pce);
  deo<double>(c, t1, t0, c.pco, 3, 1, 1, 0, 0.0, nullptr);
  deo<double>(c, out, t1, c.pce, 3, 1, 0, 2, -c.kappa * c.kappa, in);
}

void mtilde_s(Ctx& c, float* out, const float* in) {
  c.ensure_eo();
  float* tmp = c.eo_s[0];
  deo<float>(c, tmp, in, c.pco, 3, 0, 1, 0, 0.0, nullptr);
  deo<float>(c, out, tmp, c.pce, 3, 0, 1, 2, -(double)(float)(c.kappa * c.kappa), in);
}

// bicgstab_vm_ (bicgstab.cc:68-333): BiCGStab on mtilde for the pce parity,
// iter = 1..maxiter-1, converged when sqrt(|r|^2/|b|^2) < 1e-14 after the
// omega step.  x: initial guess in, solution out.  Returns conviter.
int bicgstab_vm(Ctx& c, double* x, const double* b, int maxiter) {
  c.ensure_eo();
  c.ensure_outer();
  const Geom& G = c.G;
  double *q = c.eo_d[2], *r = c.eo_d[3], *p = c.eo_d[4], *t = c.eo_d[5], *r0 = c.out_r0,
         *bb = c.out_q, *xx = c.out_p;
  // vectors of one parity: the other parity's sites are held at zero
  parity_select<double>(G, bb, b, c.pce, c.st);
  parity_select<double>(G, xx, x, c.pce, c.st);
  mtilde_d(c, q, xx);
  blas_bicg_init<double>(G, bb, q, r, p, r0, c.d_res, c.rb, c.st);
  const double* h = c.fetch(2);
  const double bnorm = h[0];
  std::complex<double> rho0(h[1], 0), rho, beta, omega, alpha, ctmp;
  int iter;
  for (iter = 1; iter < maxiter; iter++) {
    mtilde_d(c, q, p);
    blas_cdot<double>(G, r0, q, c.d_res, c.rb, c.st);
    h = c.fetch(2);
    ctmp = std::complex<double>(h[0], h[1]);
    alpha = rho0 / ctmp;
    blas_bicg_update<double>(G, xx, r, p, q, alpha.real(), alpha.imag(), nullptr, c.d_res, c.rb,
                             c.st);
    mtilde_d(c, t, r);
    blas_norm_cdot<double>(G, t, r, c.d_res, c.rb, c.st);
    h = c.fetch(3);
    omega = std::complex<double>(h[1] / h[0], h[2] / h[0]);
    blas_bicg_update<double>(G, xx, r, r, t, omega.real(), omega.imag(), r0, c.d_res, c.rb, c.st);
    h = c.fetch(3);
    const double rnorm = h[0];
    rho = std::complex<double>(h[1], h[2]);
    if (std::sqrt(rnorm / bnorm) < 1e-14) break;
    beta = alpha * rho / (rho0 * omega);
    rho0 = rho;
    blas_bicg_p<double>(G, p, r, q, beta.real(), beta.imag(), omega.real(), omega.imag(), c.st);
  }
  blas_copy<double>(G, x, xx, 0, G.V, c.st);
  c.check_launch("bicgstab_vm");
  return iter;
}

// mtdagmt_vm_: mtilde_dag(mtilde(in))
void mtdagmt_d(Ctx& c, double* out, const double* in) {
  c.ensure_eo();
  double* t = c.eo_d[5];
  mtilde_d(c, t, in);
  mtilde_dag_d(c, out, t);
}

static void check_finite(double v, const char* what) {
  if (!std::isfinite(v)) throw Error(3, std::string(what) + ": non-finite residual norm");
}

// cg_vm_ (cg.cc:65-172): CG on mtdagmt for the pce parity; x: initial guess
// in, solution out.  iter = 1..maxiter-1; converged when
// sqrt(|r|^2/|b|^2) < 1e-14 after the x/r update.  Returns the last iter
// (the reference does not report it).  A zero source returns x = 0 at
// iteration 0 (the reference divides 0 by 0 there).
int cg_vm(Ctx& c, double* x, const double* b, int maxiter) {
  c.ensure_eo();
  c.ensure_outer();
  const Geom& G = c.G;
  double *q = c.eo_d[2], *r = c.eo_d[3], *p = c.eo_d[4], *r0 = c.out_r0, *bb = c.out_q,
         *xx = c.out_p;
  parity_select<double>(G, bb, b, c.pce, c.st);
  parity_select<double>(G, xx, x, c.pce, c.st);
  mtdagmt_d(c, q, xx);
  blas_bicg_init<double>(G, bb, q, r, p, r0, c.d_res, c.rb, c.st);
  const double* h = c.fetch(2);
  const double bnorm = h[0];
  double rho0 = h[1];
  if (bnorm == 0) {
    blas_zero<double>(G, x, 0, G.V, c.st);
    return 0;
  }
  int iter;
  for (iter = 1; iter < maxiter; iter++) {
    mtdagmt_d(c, q, p);
    blas_cdot<double>(G, p, q, c.d_res, c.rb, c.st);
    h = c.fetch(1);
    const double alpha = rho0 / h[0];
    blas_bicg_update<double>(G, xx, r, p, q, alpha, 0.0, nullptr, c.d_res, c.rb, c.st);
    h = c.fetch(1);
    const double rnorm = h[0];
    check_finite(rnorm, "cg_vm");
    if (std::sqrt(rnorm / bnorm) < 1e-14) break;
    const double beta = rnorm / rho0;
    rho0 = rnorm;
    blas_bicg_p<double>(G, p, r, q, beta, 0.0, 0.0, 0.0, c.st);
  }
  blas_copy<double>(G, x, xx, 0, G.V, c.st);
  c.check_launch("cg_vm");
  return iter;
}

// mcg_vm_ (mcg.cc:65-219): multi-shift CG for (mtdagmt + sigma_k) x_k = b,
// k < n, all x_k from zero, sharing the Krylov space of the unshifted
// system; the shifted coefficients follow the recurrence of mcg.cc:141-147
// (zeta ratios z_k) and every iteration's shift updates run in one kernel.
// Same stopping rule as cg_vm on the unshifted residual.  Returns the last
// iter.  A shift whose residual |z_k| |r| / |b| fell below 1e-14 is no
// longer updated (the reference keeps updating it until z_k underflows and
// 0/0 turns its solution into NaN; up to that point the two agree).
int mcg_vm(Ctx& c, double* X, const double* b, int n, const double* sigma, int maxiter) {
  if (n < 1 || n > Ctx::kMaxRhs) throw Error(1, "mcg_vm: number of shifts must be 1..32");
  if (c.G.nr != 1) throw Error(1, "mcg_vm: single right-hand side only");
  c.ensure_eo();
  c.ensure_outer();
  const Geom& G = c.G;
  if (c.ms_n < n) {
    c.ms_p = nullptr;
    QWSG_CUDA(cudaMalloc(&c.ms_p, sizeof(double) * c.spinor_elems() * n));
    c.owned.push_back(c.ms_p);
    c.ms_n = n;
  }
  double *q = c.eo_d[2], *r = c.eo_d[3], *p = c.eo_d[4], *r0 = c.out_r0, *bb = c.out_q;
  parity_select<double>(G, bb, b, c.pce, c.st);
  blas_bicg_init<double>(G, bb, nullptr, r, p, r0, c.d_res, c.rb, c.st);
  const double* h = c.fetch(1);
  const double bnorm = h[0];
  double rho0 = bnorm;
  for (int k = 0; k < n; k++) {
    blas_zero<double>(G, X + k * c.spinor_elems(), 0, G.V, c.st);
    blas_copy<double>(G, c.ms_p + k * c.spinor_elems(), r, 0, G.V, c.st);
  }
  if (bnorm == 0) return 0;
  std::vector<double> z0(n, 1.0), z1(n, 1.0), z2(n, 0.0), cf(4 * n, 0.0);
  std::vector<char> active(n, 1);
  double alpha0 = 1.0, beta = 0.0;
  int iter;
  for (iter = 1; iter < maxiter; iter++) {
    mtdagmt_d(c, q, p);
    blas_cdot<double>(G, p, q, c.d_res, c.rb, c.st);
    h = c.fetch(1);
    const double alpha = -rho0 / h[0];
    blas_axpy_norm<double>(G, r, q, alpha, c.d_res, c.rb, c.st);
    h = c.fetch(1);
    const double rnorm = h[0];
    check_finite(rnorm, "mcg_vm");
    const bool done = std::sqrt(rnorm / bnorm) < 1e-14;
    const double beta_new = rnorm / rho0;
    for (int k = 0; k < n; k++) {
      cf[4 * k + 3] = active[k];
      if (!active[k]) continue;
      z2[k] = z1[k] * z0[k] * alpha0 /
              (alpha * beta * (z0[k] - z1[k]) + z0[k] * alpha0 * (1.0 - sigma[k] * alpha));
      const double ratio = z2[k] / z1[k];
      cf[4 * k + 0] = alpha * ratio;           // x_k -= alpha z2/z1 pp_k
      cf[4 * k + 1] = z2[k];                   // pp_k = z2 r + ...
      cf[4 * k + 2] = beta_new * ratio * ratio;  // ... + beta (z2/z1)^2 pp_k
    }
    blas_mshift(G, X, c.ms_p, n, r, p, beta_new, c.put_coefs(cf.data(), 4 * n), !done, c.st);
    if (done) break;
    beta = beta_new;
    rho0 = rnorm;
    for (int k = 0; k < n; k++) {
      if (!active[k]) continue;
      // converged shifts: their x_k is final after this iteration's update
      if (std::fabs(z2[k]) * std::sqrt(rnorm / bnorm) < 1e-14) active[k] = 0;
      z0[k] = z1[k];
      z1[k] = z2[k];
    }
    alpha0 = alpha;
  }
  c.check_launch("mcg_vm");
  return iter;
}

}  // namespace qwsg
