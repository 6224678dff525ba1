// Native qwsg_* C ABI (include/qwsg.h).
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/qwsg.h"

#include "ctx.h"

namespace qwsg {

std::atomic<long> g_kernel_launches{0};
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
  if (l->c->parent) l->c->sync_from_parent(false);
}
// operations defined for one right-hand side only
static void single_rhs(qwsg_lattice* l, const char* what) {
  if (l->c->G.nr != 1)
    throw Error(1, std::string(what) + ": not available on a multi-RHS handle");
}
// fields live on the parent lattice of a multi-RHS handle
static void not_batch(qwsg_lattice* l, const char* what) {
  if (l->c->parent)
    throw Error(1, std::string(what) + ": load fields on the parent lattice of a multi-RHS handle");
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

// host: G.nr natural-layout spinors back to back ([nr][V][24])
template <typename R>
static void sp_to_dev(Ctx& c, R* dev, const R* host) {
  const size_t n = sizeof(R) * 24 * (size_t)c.G.V;
  R* d = (R*)staging(c, n * c.G.nr);
  QWSG_CUDA(cudaMemcpyAsync(d, host, n * c.G.nr, cudaMemcpyHostToDevice, c.st));
  for (int r = 0; r < c.G.nr; r++)
    nat_to_planes_spinor<R>(c.G, dev, d + (size_t)r * 24 * c.G.V, c.st, r);
  c.check_launch("spinor_to_device");
  QWSG_CUDA(cudaStreamSynchronize(c.st));
}
template <typename R>
static void sp_to_host(Ctx& c, R* host, const R* dev) {
  const size_t n = sizeof(R) * 24 * (size_t)c.G.V;
  R* d = (R*)staging(c, n * c.G.nr);
  for (int r = 0; r < c.G.nr; r++)
    planes_to_nat_spinor<R>(c.G, d + (size_t)r * 24 * c.G.V, dev, c.st, r);
  c.check_launch("spinor_to_host");
  QWSG_CUDA(cudaMemcpyAsync(host, d, n * c.G.nr, cudaMemcpyDeviceToHost, c.st));
  QWSG_CUDA(cudaStreamSynchronize(c.st));
}

static void copy_stats(const SolveStats& s, qwsg_solve_stats* st) {
  st->outer_iters = s.outer_iters;
  st->inner_iters = s.inner_iters;
  st->rel_resid_recursive = s.rel_resid_recursive;
  st->rel_resid_true = s.rel_resid_true;
}
// the summary of a multi-RHS solve: the most outer iterations and the largest
// residuals over the RHS
static SolveStats worst(const std::vector<SolveStats>& v) {
  SolveStats w;
  for (const auto& s : v) {
    w.outer_iters = s.outer_iters > w.outer_iters ? s.outer_iters : w.outer_iters;
    w.inner_iters = s.inner_iters;
    w.rel_resid_recursive =
        s.rel_resid_recursive > w.rel_resid_recursive ? s.rel_resid_recursive : w.rel_resid_recursive;
    w.rel_resid_true = s.rel_resid_true > w.rel_resid_true ? s.rel_resid_true : w.rel_resid_true;
  }
  return w;
}

}  // namespace qwsg

using namespace qwsg;

// ---- BQCD-format arrays, reordered on the device (bqcd.cu) --------------------
// staging: the raw array (n reals) and, if given, the site map after it
static const int* bqcd_stage(Ctx& c, const double* const* parts, const size_t* sizes, int nparts,
                             const int* site_map, double** data) {
  size_t n = 0;
  for (int k = 0; k < nparts; k++) n += sizes[k];
  const size_t map_off = (sizeof(double) * n + 255) / 256 * 256;
  char* d = (char*)staging(c, map_off + (site_map ? sizeof(int) * (size_t)c.G.V : 0));
  size_t off = 0;
  for (int k = 0; k < nparts; k++) {
    if (parts[k])
      QWSG_CUDA(cudaMemcpyAsync(d + sizeof(double) * off, parts[k], sizeof(double) * sizes[k],
                                cudaMemcpyHostToDevice, c.st));
    off += sizes[k];
  }
  *data = (double*)d;
  if (!site_map) return nullptr;
  QWSG_CUDA(cudaMemcpyAsync(d + map_off, site_map, sizeof(int) * (size_t)c.G.V,
                            cudaMemcpyHostToDevice, c.st));
  return (const int*)(d + map_off);
}

// a site map must send the sites of parity eo to slots [eo*V/2, (eo+1)*V/2),
// each slot once (std_xyzt2i_ numbers the sites of each parity 1..V/2)
static void check_site_map(const Ctx& c, const int* site_map) {
  if (!site_map) return;
  const int* L = c.G.L;
  const int V = c.G.V, Vh = V / 2;
  std::vector<char> seen(V, 0);
  for (int n = 0; n < V; n++) {
    const int x = n % L[0], y = (n / L[0]) % L[1], z = (n / (L[0] * L[1])) % L[2],
              t = n / (L[0] * L[1] * L[2]);
    const int eo = (x + y + z + t) & 1, s = site_map[n];
    if (s < eo * Vh || s >= (eo + 1) * Vh || seen[s])
      throw Error(1, "BQCD site map: not a per-parity permutation of the slots");
    seen[s] = 1;
  }
}

template <typename R>
static void spinor_from_bqcd(Ctx& c, R* dev, const double* even, const double* odd,
                             const int* site_map) {
  if (!dev || !even || !odd) throw Error(1, "spinor_from_bqcd: NULL argument");
  check_site_map(c, site_map);
  const size_t half = (size_t)12 * c.G.V;  // reals of one parity array
  const double* parts[2] = {even, odd};
  const size_t sizes[2] = {half, half};
  for (int r = 0; r < c.G.nr; r++) {
    double* d;
    const double* pr[2] = {parts[0] + r * half, parts[1] + r * half};
    const int* map = bqcd_stage(c, pr, sizes, 2, site_map, &d);
    bqcd_to_planes_spinor<R>(c.G, dev, d, map, r, c.st);
    c.check_launch("spinor_from_bqcd");
    QWSG_CUDA(cudaStreamSynchronize(c.st));
  }
}
template <typename R>
static void spinor_to_bqcd(Ctx& c, double* even, double* odd, const R* dev, const int* site_map) {
  if (!dev || !even || !odd) throw Error(1, "spinor_to_bqcd: NULL argument");
  check_site_map(c, site_map);
  const size_t half = (size_t)12 * c.G.V;
  const double* none[2] = {nullptr, nullptr};
  const size_t sizes[2] = {half, half};
  for (int r = 0; r < c.G.nr; r++) {
    double* d;
    const int* map = bqcd_stage(c, none, sizes, 2, site_map, &d);
    planes_to_bqcd_spinor<R>(c.G, d, dev, map, r, c.st);
    c.check_launch("spinor_to_bqcd");
    QWSG_CUDA(cudaMemcpyAsync(even + r * half, d, sizeof(double) * half, cudaMemcpyDeviceToHost,
                              c.st));
    QWSG_CUDA(cudaMemcpyAsync(odd + r * half, d + half, sizeof(double) * half,
                              cudaMemcpyDeviceToHost, c.st));
    QWSG_CUDA(cudaStreamSynchronize(c.st));
  }
}
extern "C" {

const char* qwsg_last_error(void) { return g_last_error.c_str(); }
const char* qwsg_version(void) { return "qws_b200 0.1 (sm_100a)"; }
long qwsg_launch_count(void) { return g_kernel_launches.load(); }

int qwsg_create(qwsg_lattice** out, const int L[4], const int NB[4], int tbc) {
  return guarded([&] {
    if (!out || !L || !NB) throw Error(1, "qwsg_create: NULL argument");
    if (tbc != 1 && tbc != -1) throw Error(1, "qwsg_create: tbc must be +1 or -1");
    *out = new qwsg_lattice{new Ctx(L, NB, tbc)};
  });
}

int qwsg_create_batch(qwsg_lattice** out, qwsg_lattice* parent, int nrhs) {
  return guarded([&] {
    if (!out) throw Error(1, "qwsg_create_batch: NULL argument");
    check_ctx(parent);
    if (parent->c->parent) throw Error(1, "qwsg_create_batch: the parent must be a lattice");
    const Geom& G = parent->c->G;
    auto* c = new Ctx(G.L, G.NB, G.tbc, nrhs);
    c->G.hop_threads = G.hop_threads;
    c->owns_fields = false;
    c->parent = parent->c;
    try {
      c->sync_from_parent(false);
    } catch (...) {
      delete c;
      throw;
    }
    *out = new qwsg_lattice{c};
  });
}

int qwsg_batch_set_parent(qwsg_lattice* l, qwsg_lattice* parent) {
  return guarded([&] {
    // (the old parent may be gone: nothing of it is touched)
    if (!l || !l->c || !parent || !parent->c) throw Error(4, "lattice handle is NULL");
    Ctx& c = *l->c;
    Ctx& p = *parent->c;
    if (!c.parent) throw Error(1, "qwsg_batch_set_parent: not a multi-RHS handle");
    if (p.parent) throw Error(1, "qwsg_batch_set_parent: the parent must be a lattice");
    for (int mu = 0; mu < 4; mu++)
      if (p.G.L[mu] != c.G.L[mu] || p.G.NB[mu] != c.G.NB[mu])
        throw Error(1, "qwsg_batch_set_parent: the lattice must have the same extents and block grid");
    if (p.G.tbc != c.G.tbc) throw Error(1, "qwsg_batch_set_parent: the time boundary differs");
    QWSG_CUDA(cudaStreamSynchronize(c.st));  // the handle's running work
    c.graph_gen++;  // the graphs hold the old fields' addresses: update before use
    c.rhs_kappas.clear();                    // per-RHS clover terms of the old gauge field
    c.rhs_tols.clear();
    c.parent = &p;
    c.G.hop_threads = p.G.hop_threads;
    c.links12_valid = false;
    c.sync_from_parent(false);
  });
}

int qwsg_batch_set_kappas(qwsg_lattice* l, const double* kappas, double csw) {
  return guarded([&] {
    check_ctx(l);
    if (!kappas) throw Error(1, "qwsg_batch_set_kappas: NULL argument");
    for (int r = 0; r < l->c->G.nr; r++)
      if (!(kappas[r] > 0) || !std::isfinite(kappas[r]))
        throw Error(1, "qwsg_batch_set_kappas: kappa must be positive and finite");
    set_rhs_kappas(*l->c, kappas, csw);
  });
}

int qwsg_batch_set_tols(qwsg_lattice* l, const double* tols) {
  return guarded([&] {
    check_ctx(l);
    Ctx& c = *l->c;
    if (!tols) {
      c.rhs_tols.clear();
      return;
    }
    for (int r = 0; r < c.G.nr; r++)
      if (!std::isfinite(tols[r])) throw Error(1, "qwsg_batch_set_tols: tolerance must be finite");
    c.rhs_tols.assign(tols, tols + c.G.nr);
  });
}

int qwsg_inject_breakdown(qwsg_lattice* l, int outer_iter) {
  return guarded([&] {
    check_ctx(l);
    if (outer_iter < 0) throw Error(1, "qwsg_inject_breakdown: outer_iter must be >= 0");
    l->c->breakdown_at = outer_iter;
  });
}

int qwsg_nrhs(const qwsg_lattice* l, int* nrhs) {
  return guarded([&] {
    if (!l || !l->c) throw Error(4, "lattice handle is NULL");
    if (nrhs) *nrhs = l->c->G.nr;
  });
}

int qwsg_batch_stats(qwsg_lattice* l, qwsg_solve_stats* per_rhs, int* iters_per_rhs) {
  return guarded([&] {
    if (!l || !l->c) throw Error(4, "lattice handle is NULL");
    Ctx& c = *l->c;
    for (int r = 0; r < c.G.nr; r++) {
      if (per_rhs && r < (int)c.last_stats.size()) copy_stats(c.last_stats[r], per_rhs + r);
      if (iters_per_rhs && r < (int)c.last_iters.size()) iters_per_rhs[r] = c.last_iters[r];
    }
  });
}

int qwsg_build_clover(qwsg_lattice* l, double csw) {
  return guarded([&] {
    check_ctx(l);
    not_batch(l, "qwsg_build_clover");
    build_clover(*l->c, csw);
  });
}

int qwsg_gen_gauge_device(qwsg_lattice* l, unsigned long long seed, int n_smear, double alpha,
                          double* plaq) {
  return guarded([&] {
    check_ctx(l);
    not_batch(l, "qwsg_gen_gauge_device");
    double p = gen_gauge_device(*l->c, seed, n_smear, alpha);
    if (plaq) *plaq = p;
  });
}

int qwsg_set_graphs(qwsg_lattice* l, int enable) {
  return guarded([&] {
    check_ctx(l);
    Ctx& c = *l->c;
    QWSG_CUDA(cudaStreamSynchronize(c.st));
    c.use_graphs = enable != 0;
    if (!c.use_graphs) c.clear_graphs();
  });
}

int qwsg_set_link_compression(qwsg_lattice* l, int mode) {
  return guarded([&] {
    check_ctx(l);
    not_batch(l, "qwsg_set_link_compression");
    if (mode != 0 && mode != 1) throw Error(1, "qwsg_set_link_compression: mode must be 0 or 1");
    Ctx& c = *l->c;
    QWSG_CUDA(cudaStreamSynchronize(c.st));
    c.link_compress = mode;
    c.links12_valid = false;
    c.ensure_links12();
  });
}
int qwsg_link_compression(qwsg_lattice* l, int* active) {
  return guarded([&] {
    check_ctx(l);
    Ctx& c = *l->c;
    c.ensure_links12();
    if (active) *active = c.links12_on ? 1 : 0;
  });
}

int qwsg_set_hop_threads(qwsg_lattice* l, int threads) {
  return guarded([&] {
    check_ctx(l);
    if (threads != 64 && threads != 128 && threads != 256)
      throw Error(1, "qwsg_set_hop_threads: threads must be 64, 128 or 256");
    Ctx& c = *l->c;
    QWSG_CUDA(cudaStreamSynchronize(c.st));
    c.clear_graphs();  // captured launches carry the old shape
    c.G.hop_threads = threads;
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

int qwsg_own_stream(qwsg_lattice* l, int priority, void** stream) {
  return guarded([&] {
    check_ctx(l);
    Ctx& c = *l->c;
    QWSG_CUDA(cudaStreamSynchronize(c.st));
    cudaStream_t s = nullptr;
    QWSG_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, priority));
    if (c.own_stream) cudaStreamDestroy(c.st);
    c.st = s;
    c.own_stream = true;
    if (stream) *stream = (void*)s;
  });
}

int qwsg_set_kappa(qwsg_lattice* l, double kappa) {
  return guarded([&] {
    check_ctx(l);
    not_batch(l, "qwsg_set_kappa");
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
    not_batch(l, "qwsg_load_gauge");
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
    not_batch(l, "qwsg_load_clover");
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
    not_batch(l, "qwsg_load_gauge_s");
    Ctx& c = *l->c;
    c.ensure_fields_s();
    load_gauge_t<float, float>(c, c.Us, U);
  });
}
int qwsg_load_clover_s(qwsg_lattice* l, const float* C) {
  return guarded([&] {
    check_ctx(l);
    not_batch(l, "qwsg_load_clover_s");
    Ctx& c = *l->c;
    c.ensure_fields_s();
    load_clover_t<float, float>(c, c.Cs, C);
  });
}

int qwsg_load_gauge_bqcd(qwsg_lattice* l, const double* u, const int* site_map) {
  return guarded([&] {
    check_ctx(l);
    not_batch(l, "qwsg_load_gauge_bqcd");
    if (!u) throw Error(1, "qwsg_load_gauge_bqcd: NULL argument");
    Ctx& c = *l->c;
    check_site_map(c, site_map);
    c.ensure_fields_d();
    c.ensure_fields_s();
    const size_t n = (size_t)72 * c.G.V;
    double* d;
    const int* map = bqcd_stage(c, &u, &n, 1, site_map, &d);
    bqcd_to_planes_gauge<double>(c.G, c.Ud, d, map, c.st);
    bqcd_to_planes_gauge<float>(c.G, c.Us, d, map, c.st);
    c.check_launch("load_gauge_bqcd");
    QWSG_CUDA(cudaStreamSynchronize(c.st));
  });
}
int qwsg_load_clover_bqcd(qwsg_lattice* l, const double* cl, const int* site_map) {
  return guarded([&] {
    check_ctx(l);
    not_batch(l, "qwsg_load_clover_bqcd");
    if (!cl) throw Error(1, "qwsg_load_clover_bqcd: NULL argument");
    Ctx& c = *l->c;
    check_site_map(c, site_map);
    c.ensure_fields_d();
    c.ensure_fields_s();
    const size_t n = (size_t)72 * c.G.V;
    double* d;
    const int* map = bqcd_stage(c, &cl, &n, 1, site_map, &d);
    bqcd_to_planes_clover<double>(c.G, c.Cd, d, map, c.st);
    bqcd_to_planes_clover<float>(c.G, c.Cs, d, map, c.st);
    c.check_launch("load_clover_bqcd");
    QWSG_CUDA(cudaStreamSynchronize(c.st));
  });
}
int qwsg_spinor_from_bqcd_d(qwsg_lattice* l, double* dev, const double* even, const double* odd,
                            const int* site_map) {
  return guarded([&] {
    check_ctx(l);
    spinor_from_bqcd<double>(*l->c, dev, even, odd, site_map);
  });
}
int qwsg_spinor_from_bqcd_s(qwsg_lattice* l, float* dev, const double* even, const double* odd,
                            const int* site_map) {
  return guarded([&] {
    check_ctx(l);
    spinor_from_bqcd<float>(*l->c, dev, even, odd, site_map);
  });
}
int qwsg_spinor_to_bqcd_d(qwsg_lattice* l, double* even, double* odd, const double* dev,
                          const int* site_map) {
  return guarded([&] {
    check_ctx(l);
    spinor_to_bqcd<double>(*l->c, even, odd, dev, site_map);
  });
}
int qwsg_spinor_to_bqcd_s(qwsg_lattice* l, double* even, double* odd, const float* dev,
                          const int* site_map) {
  return guarded([&] {
    check_ctx(l);
    spinor_to_bqcd<float>(*l->c, even, odd, dev, site_map);
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
    Ctx& c = *l->c;
    int it;
    if (c.G.nr > 1) {
      c.last_iters.assign(c.G.nr, 0);
      it = bicgstab_precdd_s_mrhs(c, x, b, tol, maxiter, nsap, nm, c.last_iters.data());
      if (final_rel) *final_rel = -1;
    } else {
      it = bicgstab_precdd_s(c, x, b, tol, maxiter, nsap, nm, final_rel);
    }
    if (iters) *iters = it;
  });
}
int qwsg_bicgstab_dd_mix(qwsg_lattice* l, double* x, const double* b, double tol, int maxiter,
                         double tol_s, int maxiter_s, int nsap, int nm, qwsg_solve_stats* st) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, true);
    need_fields(*l->c, false);
    Ctx& c = *l->c;
    SolveStats s;
    if (c.G.nr > 1) {
      c.last_stats.assign(c.G.nr, SolveStats{});
      bicgstab_dd_mix_mrhs(c, x, b, tol, maxiter, tol_s, maxiter_s, nsap, nm,
                           c.last_stats.data());
      s = worst(c.last_stats);
    } else {
      bicgstab_dd_mix(c, x, b, tol, maxiter, tol_s, maxiter_s, nsap, nm, &s, nullptr, 0);
    }
    if (st) copy_stats(s, st);
  });
}
int qwsg_prec_s_h(qwsg_lattice* l, float* out, const float* in, int nsap, int nm) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    prec_s_h(*l->c, out, in, nsap, nm);
  });
}
int qwsg_ddd_in_h(qwsg_lattice* l, float* out, const float* in, int colour) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    sap_kernel(*l->c, out, in, nullptr, 0, colour, 0, 0.0, true);
  });
}
int qwsg_jinv_h(qwsg_lattice* l, float* x, const float* b, int colour, int nm) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    sap_kernel(*l->c, x, b, nullptr, 1, colour, nm, 0.0, true);
  });
}
int qwsg_ddd_out_h(qwsg_lattice* l, float* out, const float* in, int colour, double factor) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    sap_kernel(*l->c, out, in, nullptr, 2, colour, 0, factor, true);
  });
}
int qwsg_sap_update_s(qwsg_lattice* l, float* s, const float* a, const float* in, int colour) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    sap_kernel(*l->c, s, a, in, 3, colour, 0, 0.0, false);
  });
}
int qwsg_sap_update_h(qwsg_lattice* l, float* s, const float* a, const float* in, int colour) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    sap_kernel(*l->c, s, a, in, 3, colour, 0, 0.0, true);
  });
}
int qwsg_store_h(qwsg_lattice* l, float* out, const float* in) {
  return guarded([&] {
    check_ctx(l);
    Ctx& c = *l->c;
    if (!c.h_b) c.h_b = c.alloc_spinor_h();
    spinor_s2h(c.G, c.h_b, in, c.st);
    spinor_h2s(c.G, out, c.h_b, c.st);
    c.check_launch("qwsg_store_h");
  });
}
int qwsg_bicgstab_precdd_s_h(qwsg_lattice* l, float* x, const float* b, double tol, int maxiter,
                             int nsap, int nm, int* iters, double* final_rel) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, false);
    Ctx& c = *l->c;
    int it;
    if (c.G.nr > 1) {
      c.last_iters.assign(c.G.nr, 0);
      it = bicgstab_precdd_s_h_mrhs(c, x, b, tol, maxiter, nsap, nm, c.last_iters.data());
      if (final_rel) *final_rel = -1;
    } else {
      it = bicgstab_precdd_s_h(c, x, b, tol, maxiter, nsap, nm, final_rel);
    }
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
    Ctx& c = *l->c;
    SolveStats s;
    if (c.G.nr > 1) {
      c.last_stats.assign(c.G.nr, SolveStats{});
      bicgstab_dd_mix2_hf_mrhs(c, x, b, tol, maxiter, tol_s, maxiter_s, nsap, nm, reliable,
                               c.last_stats.data());
      s = worst(c.last_stats);
    } else {
      bicgstab_dd_mix2_hf(c, x, b, tol, maxiter, tol_s, maxiter_s, nsap, nm, reliable, &s);
    }
    if (st) copy_stats(s, st);
  });
}
int qwsg_group_bicgstab_dd_mix2_hf(qwsg_group_item* items, int n, void* stream,
                                   qwsg_group_stats* gst) {
  return guarded([&] {
    if (n < 0 || (n > 0 && !items)) throw Error(1, "group solve: no items");
    if (n == 0) return;
    std::vector<GroupItem> v(n);
    for (int i = 0; i < n; i++) {
      qwsg_group_item& it = items[i];
      check_ctx(it.lat);
      need_fields(*it.lat->c, true);
      need_fields(*it.lat->c, false);
      if (!it.x || !it.b) throw Error(1, "group solve: x and b must be set");
      v[i] = GroupItem{it.lat->c, it.x, it.b, it.tol, it.maxiter, it.tol_s, it.maxiter_s,
                       it.nsap, it.nm, it.reliable, SolveStats{}, -1, std::string()};
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : v[0].c->st;
    GroupStats gs{};
    std::string first_error;
    try {
      group_bicgstab_dd_mix2_hf(v, st, &gs);
    } catch (...) {
      for (int i = 0; i < n; i++) items[i].status = v[i].status < 0 ? 3 : v[i].status;
      throw;
    }
    int code = 0;
    for (int i = 0; i < n; i++) {
      items[i].status = v[i].status;
      copy_stats(v[i].stats, &items[i].stats);
      if (v[i].status != 0 && code == 0) {
        code = v[i].status;
        first_error = "group solve, item " + std::to_string(i) + ": " + v[i].error;
      }
    }
    if (gst) {
      gst->rounds = gs.rounds;
      gst->merged_launches = gs.merged_launches;
      gst->member_launches = gs.member_launches;
      gst->t_members = gs.t_members;
      gst->t_merge = gs.t_merge;
      gst->t_launch = gs.t_launch;
      gst->t_gpu_wait = gs.t_gpu_wait;
    }
    if (code) throw Error(code, first_error);
  });
}
int qwsg_set_parities(qwsg_lattice* l, int pce, int pco) {
  return guarded([&] {
    check_ctx(l);
    single_rhs(l, "qwsg_set_parities");
    if (pce < 0 || pce > 1 || pco != 1 - pce) throw Error(1, "parities must be (0,1) or (1,0)");
    l->c->pce = pce;
    l->c->pco = pco;
  });
}
int qwsg_deo_d(qwsg_lattice* l, double* out, const double* in, int pe, int which, int dag,
               int clov, int mode, double factor, const double* in0) {
  return guarded([&] {
    check_ctx(l);
    single_rhs(l, "qwsg_deo_d");
    deo<double>(*l->c, out, in, pe, which, dag, clov, mode, factor, in0);
  });
}
int qwsg_deo_s(qwsg_lattice* l, float* out, const float* in, int pe, int which, int dag, int clov,
               int mode, double factor, const float* in0) {
  return guarded([&] {
    check_ctx(l);
    single_rhs(l, "qwsg_deo_s");
    deo<float>(*l->c, out, in, pe, which, dag, clov, mode, factor, in0);
  });
}
int qwsg_clv_d(qwsg_lattice* l, double* out, const double* in, int pe) {
  return guarded([&] {
    check_ctx(l);
    single_rhs(l, "qwsg_clv_d");
    clv<double>(*l->c, out, in, pe);
  });
}
int qwsg_clv_s(qwsg_lattice* l, float* out, const float* in, int pe) {
  return guarded([&] {
    check_ctx(l);
    single_rhs(l, "qwsg_clv_s");
    clv<float>(*l->c, out, in, pe);
  });
}
int qwsg_mtilde_d(qwsg_lattice* l, double* out, const double* in) {
  return guarded([&] {
    check_ctx(l);
    single_rhs(l, "qwsg_mtilde_d");
    need_fields(*l->c, true);
    mtilde_d(*l->c, out, in);
  });
}
int qwsg_mtilde_dag_d(qwsg_lattice* l, double* out, const double* in) {
  return guarded([&] {
    check_ctx(l);
    single_rhs(l, "qwsg_mtilde_dag_d");
    need_fields(*l->c, true);
    mtilde_dag_d(*l->c, out, in);
  });
}
int qwsg_mtilde_s(qwsg_lattice* l, float* out, const float* in) {
  return guarded([&] {
    check_ctx(l);
    single_rhs(l, "qwsg_mtilde_s");
    need_fields(*l->c, false);
    mtilde_s(*l->c, out, in);
  });
}
int qwsg_bicgstab_vm(qwsg_lattice* l, double* x, const double* b, int maxiter, int* iters) {
  return guarded([&] {
    check_ctx(l);
    single_rhs(l, "qwsg_bicgstab_vm");
    need_fields(*l->c, true);
    int it = bicgstab_vm(*l->c, x, b, maxiter);
    if (iters) *iters = it;
  });
}
int qwsg_mtdagmt_d(qwsg_lattice* l, double* out, const double* in) {
  return guarded([&] {
    check_ctx(l);
    single_rhs(l, "qwsg_mtdagmt_d");
    need_fields(*l->c, true);
    mtdagmt_d(*l->c, out, in);
  });
}
int qwsg_cg_vm(qwsg_lattice* l, double* x, const double* b, int maxiter, int* iters) {
  return guarded([&] {
    check_ctx(l);
    single_rhs(l, "qwsg_cg_vm");
    need_fields(*l->c, true);
    int it = cg_vm(*l->c, x, b, maxiter);
    if (iters) *iters = it;
  });
}
int qwsg_mcg_vm(qwsg_lattice* l, double* x, const double* b, int nshift, const double* sigma,
                int maxiter, int* iters) {
  return guarded([&] {
    check_ctx(l);
    single_rhs(l, "qwsg_mcg_vm");
    if (!x || !b || !sigma) throw Error(1, "qwsg_mcg_vm: NULL argument");
    need_fields(*l->c, true);
    int it = mcg_vm(*l->c, x, b, nshift, sigma, maxiter);
    if (iters) *iters = it;
  });
}
int qwsg_true_residual(qwsg_lattice* l, const double* x, const double* b, double* rel) {
  return guarded([&] {
    check_ctx(l);
    need_fields(*l->c, true);
    Ctx& c = *l->c;
    if (c.G.nr > 1) {  // rel holds one value per RHS
      if (!rel) throw Error(1, "qwsg_true_residual: rel must hold one value per RHS");
      true_residual_mrhs(c, x, b, rel);
    } else {
      double r = true_residual(c, x, b);
      if (rel) *rel = r;
    }
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
