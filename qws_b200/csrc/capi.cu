// Native qwsg_* C ABI (include/qwsg.h).
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/qwsg.h"
#include "ctx.h"

namespace qwsg {

static thread_local std::string g_last_error;

void set_error(const std::string& m) { g_last_error = m; }

template <typename F>
static int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return 3;
  }
}

// the handle's device staging buffer for host<->device conversions
static void* staging(Ctx& c, size_t n) {
  if (n > c.stage_bytes) {
    QWSG_CUDA(cudaStreamSynchronize(c.st));
    if (c.stage) cudaFree(c.stage);
    c.stage = nullptr;
    c.stage_bytes = 0;
    QWSG_CUDA(cudaMalloc(&c.stage, n));
    c.stage_bytes = n;
  }
  return c.stage;
}

static void check_ctx(qwsg_lattice* l) {
  if (!l || !l->c) throw Error(4, "lattice handle is NULL");
}

template <typename Rin, typename R>
static void load_gauge_t(Ctx& c, R* dst, const Rin* U) {
  size_t n = sizeof(Rin) * 72 * (size_t)c.G.V;
  void* d = staging(c, n);
  QWSG_CUDA(cudaMemcpyAsync(d, U, n, cudaMemcpyHostToDevice, c.st));
  nat_to_planes_gauge<Rin, R>(c.G, dst, (const Rin*)d, c.st);
  c.check_launch("load_gauge");
  QWSG_CUDA(cudaStreamSynchronize(c.st));
}
template <typename Rin, typename R>
static void load_clover_t(Ctx& c, R* dst, const Rin* C) {
  size_t n = sizeof(Rin) * 72 * (size_t)c.G.V;
  void* d = staging(c, n);
  QWSG_CUDA(cudaMemcpyAsync(d, C, n, cudaMemcpyHostToDevice, c.st));
  nat_to_planes_clover<Rin, R>(c.G, dst, (const Rin*)d, c.st);
  c.check_launch("load_clover");
  QWSG_CUDA(cudaStreamSynchronize(c.st));
}

template <typename R>
static void sp_to_dev(Ctx& c, R* dev, const R* host) {
  size_t n = sizeof(R) * 24 * (size_t)c.G.V;
  void* d = staging(c, n);
  QWSG_CUDA(cudaMemcpyAsync(d, host, n, cudaMemcpyHostToDevice, c.st));
  nat_to_planes_spinor<R>(c.G, dev, (const R*)d, c.st);
  c.check_launch("spinor_to_device");
  QWSG_CUDA(cudaStreamSynchronize(c.st));
}
template <typename R>
static void sp_to_host(Ctx& c, R* host, const R* dev) {
  size_t n = sizeof(R) * 24 * (size_t)c.G.V;
  void* d = staging(c, n);
  planes_to_nat_spinor<R>(c.G, (R*)d, dev, c.st);
  c.check_launch("spinor_to_host");
  QWSG_CUDA(cudaMemcpyAsync(host, d, n, cudaMemcpyDeviceToHost, c.st));
  QWSG_CUDA(cudaStreamSynchronize(c.st));
}

}  // namespace qwsg

using namespace qwsg;

extern "C" {

const char* qwsg_last_error(void) { return g_last_error.c_str(); }
const char* qwsg_version(void) { return "qws_b200 0.1 (sm_100a)"; }

int qwsg_create(qwsg_lattice** out, const int L[4], const int NB[4], int tbc) {
  return guarded([&] {
    if (!out || !L || !NB) throw Error(1, "qwsg_create: NULL argument");
    if (tbc != 1 && tbc != -1) throw Error(1, "qwsg_create: tbc must be +1 or -1");
    *out = new qwsg_lattice{new Ctx(L, NB, tbc)};
  });
}

int qwsg_destroy(qwsg_lattice* l) {
  return guarded([&] {
    if (!l) return;
    delete l->c;
    delete l;
  });
}

int qwsg_set_stream(qwsg_lattice* l, void* stream) {
  return guarded([&] {
    check_ctx(l);
    Ctx& c = *l->c;
    QWSG_CUDA(cudaStreamSynchronize(c.st));
    if (c.own_stream) cudaStreamDestroy(c.st);
    c.own_stream = false;
    c.st = (cudaStream_t)stream;  // NULL = the legacy default stream
  });
}

int qwsg_set_kappa(qwsg_lattice* l, double kappa) {
  return guarded([&] {
    check_ctx(l);
    l->c->kappa = kappa;
  });
}

int qwsg_geometry(const qwsg_lattice* l, int* volume, int* pad) {
  return guarded([&] {
    if (!l || !l->c) throw Error(4, "lattice handle is NULL");
    if (volume) *volume = l->c->G.V;
    if (pad) *pad = l->c->G.pad;
  });
}

int qwsg_sync(qwsg_lattice* l) {
  return guarded([&] {
    check_ctx(l);
    QWSG_CUDA(cudaStreamSynchronize(l->c->st));
  });
}

int qwsg_load_gauge(qwsg_lattice* l, const double* U) {
  return guarded([&] {
    check_ctx(l);
    Ctx& c = *l->c;
    c.ensure_fields_d();
    c.ensure_fields_s();
    load_gauge_t<double, double>(c, c.Ud, U);
    load_gauge_t<double, float>(c, c.Us, U);
  });
}
int qwsg_load_clover(qwsg_lattice* l, const double* C) {
  return guarded([&] {
    check_ctx(l);
    Ctx& c = *l->c;
    c.ensure_fields_d();
    c.ensure_fields_s();
    load_clover_t<double, double>(c, c.Cd, C);
    load_clover_t<double, float>(c, c.Cs, C);
  });
}
int qwsg_load_gauge_s(qwsg_lattice* l, const float* U) {
  return guarded([&] {
    check_ctx(l);
    Ctx& c = *l->c;
    c.ensure_fields_s();
    load_gauge_t<float, float>(c, c.Us, U);
  });
}
int qwsg_load_clover_s(qwsg_lattice* l, const float* C) {
  return guarded([&] {
    check_ctx(l);
    Ctx& c = *l->c;
    c.ensure_fields_s();
    load_clover_t<float, float>(c, c.Cs, C);
  });
}

int qwsg_spinor_to_device_d(qwsg_lattice* l, double* dev, const double* host) {
  return guarded([&] {
    check_ctx(l);
    sp_to_dev<double>(*l->c, dev, host);
  });
}
int qwsg_spinor_to_host_d(qwsg_lattice* l, double* host, const double* dev) {
  return guarded([&] {
    check_ctx(l);
    sp_to_host<double>(*l->c, host, dev);
  });
}
int qwsg_spinor_to_device_s(qwsg_lattice* l, float* dev, const float* host) {
  return guarded([&] {
    check_ctx(l);
    sp_to_dev<float>(*l->c, dev, host);
  });
}
int qwsg_spinor_to_host_s(qwsg_lattice* l, float* host, const float* dev) {
  return guarded([&] {
    check_ctx(l);
    sp_to_host<float>(*l->c, host, dev);
  });
}

static void need_fields(Ctx& c, bool dbl) {
  if (dbl ? !c.Ud : !c.Us) throw Error(4, "gauge/clover fields not loaded");
}

int qwsg_ddd_d(qwsg_lattice* l, double* out, const double* in) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, true);
    dslash_full_d(*l->c, out, in);
  });
}
int qwsg_ddd_s(qwsg_lattice* l, float* out, const float* in) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    dslash_full_s(*l->c, out, in);
  });
}
int qwsg_ddd_in_d(qwsg_lattice* l, double* out, const double* in, int colour) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, true);
    if (colour != 0 && colour != 1) throw Error(1, "colour must be 0 or 1");
    dslash_inner<double>(*l->c, out, in, colour, -1);
  });
}
int qwsg_ddd_in_s(qwsg_lattice* l, float* out, const float* in, int colour) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    if (colour != 0 && colour != 1) throw Error(1, "colour must be 0 or 1");
    dslash_inner<float>(*l->c, out, in, colour, -1);
  });
}
int qwsg_ddd_out_d(qwsg_lattice* l, double* out, const double* in, int colour, double factor) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, true);
    if (colour != 0 && colour != 1) throw Error(1, "colour must be 0 or 1");
    dslash_outer<double>(*l->c, out, in, colour, -1, factor, -1);
  });
}
int qwsg_ddd_out_s(qwsg_lattice* l, float* out, const float* in, int colour, double factor) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    if (colour != 0 && colour != 1) throw Error(1, "colour must be 0 or 1");
    dslash_outer<float>(*l->c, out, in, colour, -1, factor, -1);
  });
}
int qwsg_jinv_s(qwsg_lattice* l, float* x, const float* b, int colour, int nm) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    if (colour != 0 && colour != 1) throw Error(1, "colour must be 0 or 1");
    jinv_s(*l->c, x, b, colour, nm);
  });
}
int qwsg_prec_ddd_s(qwsg_lattice* l, float* out, const float* in, int nsap, int nm) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    prec_ddd_s(*l->c, out, in, nsap, nm);
  });
}
int qwsg_prec_s(qwsg_lattice* l, float* out, const float* in, int nsap, int nm) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    prec_s(*l->c, out, in, nsap, nm);
  });
}
int qwsg_bicgstab_precdd_s(qwsg_lattice* l, float* x, const float* b, double tol, int maxiter,
                           int nsap, int nm, int* iters, double* final_rel) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    int it = bicgstab_precdd_s(*l->c, x, b, tol, maxiter, nsap, nm, final_rel);
    if (iters) *iters = it;
  });
}
int qwsg_bicgstab_dd_mix(qwsg_lattice* l, double* x, const double* b, double tol, int maxiter,
                         double tol_s, int maxiter_s, int nsap, int nm, qwsg_solve_stats* st) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, true);
    need_fields(*l->c, false);
    SolveStats s;
    bicgstab_dd_mix(*l->c, x, b, tol, maxiter, tol_s, maxiter_s, nsap, nm, &s, nullptr, 0);
    if (st) {
      st->outer_iters = s.outer_iters;
      st->inner_iters = s.inner_iters;
      st->rel_resid_recursive = s.rel_resid_recursive;
      st->rel_resid_true = s.rel_resid_true;
    }
  });
}
int qwsg_prec_s_h(qwsg_lattice* l, float* out, const float* in, int nsap, int nm) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    prec_s_h(*l->c, out, in, nsap, nm);
  });
}
int qwsg_bicgstab_precdd_s_h(qwsg_lattice* l, float* x, const float* b, double tol, int maxiter,
                             int nsap, int nm, int* iters, double* final_rel) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    int it = bicgstab_precdd_s_h(*l->c, x, b, tol, maxiter, nsap, nm, final_rel);
    if (iters) *iters = it;
  });
}
int qwsg_bicgstab_dd_mix2_hf(qwsg_lattice* l, double* x, const double* b, double tol, int maxiter,
                             double tol_s, int maxiter_s, int nsap, int nm, int reliable,
                             qwsg_solve_stats* st) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, true);
    need_fields(*l->c, false);
    SolveStats s;
    bicgstab_dd_mix2_hf(*l->c, x, b, tol, maxiter, tol_s, maxiter_s, nsap, nm, reliable, &s);
    if (st) {
      st->outer_iters = s.outer_iters;
      st->inner_iters = s.inner_iters;
      st->rel_resid_recursive = s.rel_resid_recursive;
      st->rel_resid_true = s.rel_resid_true;
    }
  });
}
int qwsg_set_parities(qwsg_lattice* l, int pce, int pco) {
  return guarded([&] {
    check_ctx(l);
    if (pce < 0 || pce > 1 || pco != 1 - pce) throw Error(1, "parities must be (0,1) or (1,0)");
    l->c->pce = pce;
    l->c->pco = pco;
  });
}
int qwsg_deo_d(qwsg_lattice* l, double* out, const double* in, int pe, int which, int dag,
               int clov, int mode, double factor, const double* in0) {
  return guarded([&] {
    check_ctx(l);
    deo<double>(*l->c, out, in, pe, which, dag, clov, mode, factor, in0);
  });
}
int qwsg_deo_s(qwsg_lattice* l, float* out, const float* in, int pe, int which, int dag, int clov,
               int mode, double factor, const float* in0) {
  return guarded([&] {
    check_ctx(l);
    deo<float>(*l->c, out, in, pe, which, dag, clov, mode, factor, in0);
  });
}
int qwsg_clv_d(qwsg_lattice* l, double* out, const double* in, int pe) {
  return guarded([&] {
    check_ctx(l);
    clv<double>(*l->c, out, in, pe);
  });
}
int qwsg_clv_s(qwsg_lattice* l, float* out, const float* in, int pe) {
  return guarded([&] {
    check_ctx(l);
    clv<float>(*l->c, out, in, pe);
  });
}
int qwsg_mtilde_d(qwsg_lattice* l, double* out, const double* in) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, true);
    mtilde_d(*l->c, out, in);
  });
}
int qwsg_mtilde_dag_d(qwsg_lattice* l, double* out, const double* in) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, true);
    mtilde_dag_d(*l->c, out, in);
  });
}
int qwsg_mtilde_s(qwsg_lattice* l, float* out, const float* in) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    mtilde_s(*l->c, out, in);
  });
}
int qwsg_bicgstab_vm(qwsg_lattice* l, double* x, const double* b, int maxiter, int* iters) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, true);
    int it = bicgstab_vm(*l->c, x, b, maxiter);
    if (iters) *iters = it;
  });
}
int qwsg_true_residual(qwsg_lattice* l, const double* x, const double* b, double* rel) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, true);
    double r = true_residual(*l->c, x, b);
    if (rel) *rel = r;
  });
}
int qwsg_kernel_timing(qwsg_lattice* l, int enable) {
  return guarded([&] {
    check_ctx(l);
    Ctx& c = *l->c;
    QWSG_CUDA(cudaStreamSynchronize(c.st));
    c.recs.clear();
    c.ev_next = 0;
    c.timing = enable != 0;
  });
}
int qwsg_kernel_stats(qwsg_lattice* l, int* nkind, long* launches, double* ms, double* bytes) {
  return guarded([&] {
    check_ctx(l);
    if (!nkind || *nkind < K_NKIND) {
      if (nkind) *nkind = K_NKIND;
      throw Error(1, "qwsg_kernel_stats: arrays must hold K_NKIND entries");
    }
    *nkind = K_NKIND;
    for (int k = 0; k < K_NKIND; k++) {
      launches[k] = 0;
      ms[k] = 0;
      bytes[k] = 0;
    }
    kernel_stats(*l->c, launches, ms, bytes);
  });
}
const char* qwsg_kernel_name(int kind) { return kernel_kind_name(kind); }

int qwsg_counters(qwsg_lattice* l, long* prec_ddd, long* prec_s_, long* jinv, long* inner,
                  long* ddd_d) {
  return guarded([&] {
    check_ctx(l);
    Ctx& c = *l->c;
    if (prec_ddd) *prec_ddd = c.n_prec_ddd;
    if (prec_s_) *prec_s_ = c.n_prec_s;
    if (jinv) *jinv = c.n_jinv;
    if (inner) *inner = c.n_inner_iter;
    if (ddd_d) *ddd_d = c.n_dslash_d;
  });
}

}  // extern "C"
