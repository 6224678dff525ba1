// Drop-in implementation of the reference's C entry points (include/qws_dropin.h).
//
// Host arrays keep QWS's layout; every call stages them through the handle's
// device buffer, converts to planes on the GPU, runs the CUDA path and
// converts back.  Fields are uploaded lazily (dirty flag).
#include <omp.h>
#include <sys/time.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/qws_dropin.h"
#include "../../include/qwsg.h"
#include "ctx.h"

// reference-compatible globals (qws.cc:74-127)
extern "C" {
pglud_t glud = nullptr;
pglus_t glus = nullptr;
pclvd_t clvd = nullptr;
pclvs_t clvs = nullptr;
double kappa = 0, kappa2 = 0, mkappa = 0;
int nx = 0, ny = 0, nz = 0, nt = 0, nxh = 0, nxd = 0, nxs = 0, vold = 0, vols = 0;
int rank = 0, npe[4] = {1, 1, 1, 1}, domain_e = 0, domain_o = 1;
double fbc[4][2];
FILE* para_outputfile = nullptr;
// supplied by the host program in BQCD (qws_bqcd.cc:56-57); optional here
int std_xyzt2i_(int*) __attribute__((weak));
int e_o_(int*) __attribute__((weak));
}

namespace {

using namespace qwsg;

struct Dropin {
  qwsg_lattice* lat = nullptr;
  int vlend = 8, vlens = 16;
  bool fields_dirty = true;
  bool always_upload = false;
  double* pd[3] = {nullptr, nullptr, nullptr};  // FP64 planes: 0,1 work, 2 face snapshot
  float* ps[3] = {nullptr, nullptr, nullptr};   // FP32 planes
  double t_solver = 0;
  long n_calls_dd_mix = 0;
  // even-odd family: the even-odd reading of the same host fields, and work
  // planes (0 out, 1 in, 2 in0, 3 the face snapshot of deo_out_pre)
  bool eo_dirty = true;
  double* eUd = nullptr;
  double* eCd = nullptr;
  float* eUs = nullptr;
  float* eCs = nullptr;
  double* ed[4] = {};
  float* es[4] = {};
  int pce = 0, pco = 1;
};
Dropin g;
int g_vlend_req = 0, g_vlens_req = 0;

// the host fields changed: both readings must be uploaded again
void mark_dirty() {
  g.fields_dirty = true;
  g.eo_dirty = true;
}

Ctx& ctx() {
  if (!g.lat) {
    fprintf(stderr, "qws_b200: called before qws_init_\n");
    std::exit(1);
  }
  return *g.lat->c;
}

[[noreturn]] void die(const std::string& m) {
  fprintf(stderr, "qws_b200: %s\n", m.c_str());
  std::exit(1);
}

// QWS ends the program on errors (exit(1)); with QWSG_NO_EXIT set in the
// environment the entry point returns instead, leaving the message in
// qwsg_last_error() and its outputs unspecified
template <typename F>
void guard(const char* name, F&& f) {
  try {
    f();
  } catch (const std::exception& e) {
    set_error(std::string(name) + ": " + e.what());
    static const bool no_exit = std::getenv("QWSG_NO_EXIT") != nullptr;
    if (no_exit) {
      fprintf(stderr, "qws_b200: %s: %s\n", name, e.what());
      return;
    }
    die(std::string(name) + ": " + e.what());
  }
}

void* stage(Ctx& c, size_t n) {
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

void ensure_planes(Ctx& c) {
  for (int i = 0; i < 3; i++) {
    if (!g.pd[i]) g.pd[i] = c.alloc_spinor<double>();
    if (!g.ps[i]) g.ps[i] = c.alloc_spinor<float>();
  }
}

// upload the resident fields from the host globals when dirty
void sync_fields(Ctx& c) {
  c.kappa = kappa;
  if (!g.fields_dirty && !g.always_upload) return;
  c.ensure_fields_d();
  c.ensure_fields_s();
  const size_t V = (size_t)c.G.V;
  void* d = stage(c, sizeof(double) * 72 * V);
  QWSG_CUDA(cudaMemcpyAsync(d, glud, sizeof(double) * 72 * V, cudaMemcpyHostToDevice, c.st));
  qws_to_planes_gauge<double>(c.G, c.Ud, (const double*)d, g.vlend, c.st);
  QWSG_CUDA(cudaMemcpyAsync(d, clvd, sizeof(double) * 72 * V, cudaMemcpyHostToDevice, c.st));
  qws_to_planes_clover<double>(c.G, c.Cd, (const double*)d, g.vlend, c.st);
  QWSG_CUDA(cudaMemcpyAsync(d, glus, sizeof(float) * 72 * V, cudaMemcpyHostToDevice, c.st));
  qws_to_planes_gauge<float>(c.G, c.Us, (const float*)d, g.vlens, c.st);
  QWSG_CUDA(cudaMemcpyAsync(d, clvs, sizeof(float) * 72 * V, cudaMemcpyHostToDevice, c.st));
  qws_to_planes_clover<float>(c.G, c.Cs, (const float*)d, g.vlens, c.st);
  c.check_launch("field upload");
  QWSG_CUDA(cudaStreamSynchronize(c.st));
  g.fields_dirty = false;
}

// host QWS spinor array (whole lattice when dom < 0, else the half array of
// domain dom) -> device planes
template <typename R>
void up(Ctx& c, R* planes, const void* host, int dom, int vlen) {
  const size_t Vh = (size_t)c.G.Vh;
  size_t off = dom < 0 ? 0 : (size_t)dom * Vh * 24;
  size_t n = dom < 0 ? 2 * Vh * 24 : Vh * 24;
  R* d = (R*)stage(c, sizeof(R) * 2 * Vh * 24);
  QWSG_CUDA(cudaMemcpyAsync(d + off, host, sizeof(R) * n, cudaMemcpyHostToDevice, c.st));
  qws_to_planes_spinor<R>(c.G, planes, d, vlen, dom < 0 ? 0 : dom * c.G.Vh,
                          dom < 0 ? c.G.V : c.G.Vh, c.st);
  c.check_launch("spinor upload");
}

template <typename R>
void down(Ctx& c, void* host, const R* planes, int dom, int vlen) {
  const size_t Vh = (size_t)c.G.Vh;
  size_t off = dom < 0 ? 0 : (size_t)dom * Vh * 24;
  size_t n = dom < 0 ? 2 * Vh * 24 : Vh * 24;
  R* d = (R*)stage(c, sizeof(R) * 2 * Vh * 24);
  planes_to_qws_spinor<R>(c.G, d, planes, vlen, dom < 0 ? 0 : dom * c.G.Vh,
                          dom < 0 ? c.G.V : c.G.Vh, c.st);
  c.check_launch("spinor download");
  QWSG_CUDA(cudaMemcpyAsync(host, d + off, sizeof(R) * n, cudaMemcpyDeviceToHost, c.st));
  QWSG_CUDA(cudaStreamSynchronize(c.st));
}

// the even-odd operators read glud/clvd/glus/clvs with the parity split
// (qws_bqcd.cc:66-85): upload that reading next to the DD one when dirty
void sync_eo(Ctx& c) {
  sync_fields(c);
  const size_t n = (size_t)72 * c.G.pad;
  // every buffer on its own (a failed allocation is retried by the next call)
  for (double** p : {&g.eUd, &g.eCd})
    if (!*p) {
      QWSG_CUDA(cudaMalloc(p, sizeof(double) * n));
      g.eo_dirty = true;
    }
  for (float** p : {&g.eUs, &g.eCs})
    if (!*p) {
      QWSG_CUDA(cudaMalloc(p, sizeof(float) * n));
      g.eo_dirty = true;
    }
  for (int i = 0; i < 4; i++) {
    if (!g.ed[i]) g.ed[i] = c.alloc_spinor<double>();
    if (!g.es[i]) g.es[i] = c.alloc_spinor<float>();
  }
  if (g.eo_dirty || g.always_upload) {
    const size_t V = (size_t)c.G.V;
    void* d = stage(c, sizeof(double) * 72 * V);
    QWSG_CUDA(cudaMemcpyAsync(d, glud, sizeof(double) * 72 * V, cudaMemcpyHostToDevice, c.st));
    qws_to_planes_gauge<double>(c.G, g.eUd, (const double*)d, g.vlend, c.st, true);
    QWSG_CUDA(cudaMemcpyAsync(d, clvd, sizeof(double) * 72 * V, cudaMemcpyHostToDevice, c.st));
    qws_to_planes_clover<double>(c.G, g.eCd, (const double*)d, g.vlend, c.st, true);
    QWSG_CUDA(cudaMemcpyAsync(d, glus, sizeof(float) * 72 * V, cudaMemcpyHostToDevice, c.st));
    qws_to_planes_gauge<float>(c.G, g.eUs, (const float*)d, g.vlens, c.st, true);
    QWSG_CUDA(cudaMemcpyAsync(d, clvs, sizeof(float) * 72 * V, cudaMemcpyHostToDevice, c.st));
    qws_to_planes_clover<float>(c.G, g.eCs, (const float*)d, g.vlens, c.st, true);
    c.check_launch("even-odd field upload");
    QWSG_CUDA(cudaStreamSynchronize(c.st));
    g.eo_dirty = false;
  }
  c.eoUd = g.eUd;
  c.eoCd = g.eCd;
  c.eoUs = g.eUs;
  c.eoCs = g.eCs;
  c.pce = g.pce;
  c.pco = g.pco;
}

// host half array of parity p (vol elements, even-odd layout) <-> planes
template <typename R>
void up_eo(Ctx& c, R* planes, const void* host, int p, int vlen) {
  const size_t n = (size_t)c.G.Vh * 24;
  R* d = (R*)stage(c, sizeof(R) * n);
  QWSG_CUDA(cudaMemcpyAsync(d, host, sizeof(R) * n, cudaMemcpyHostToDevice, c.st));
  qws_eo_to_planes_spinor<R>(c.G, planes, d, vlen, p, c.st);
  c.check_launch("even-odd spinor upload");
}

template <typename R>
void down_eo(Ctx& c, void* host, const R* planes, int p, int vlen) {
  const size_t n = (size_t)c.G.Vh * 24;
  R* d = (R*)stage(c, sizeof(R) * n);
  planes_to_qws_eo_spinor<R>(c.G, d, planes, vlen, p, c.st);
  c.check_launch("even-odd spinor download");
  QWSG_CUDA(cudaMemcpyAsync(host, d, sizeof(R) * n, cudaMemcpyDeviceToHost, c.st));
  QWSG_CUDA(cudaStreamSynchronize(c.st));
}

int xyzt2i(int* j) {
  if (std_xyzt2i_) return std_xyzt2i_(j);
  int lex = j[0] + nx * (j[1] + ny * (j[2] + nz * j[3]));
  return lex / 2 + 1;
}
int eo_of(int* j) {
  if (e_o_) return e_o_(j);
  return (j[0] + j[1] + j[2] + j[3]) % 2;
}

// QWS host-layout element / lane of site (x,y,z,t) for lane width vlen
inline size_t qws_elem(int x, int y, int z, int t, int vlen, size_t* lane) {
  int nxv = nxh / vlen;
  size_t vol = (size_t)nxv * ny * nz * nt;
  int dom = x / nxh, xh = x % nxh;
  *lane = xh % vlen;
  return dom * vol + xh / vlen + (size_t)nxv * (y + (size_t)ny * (z + (size_t)nz * t));
}

double wall() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

}  // namespace

extern "C" {

int qwsg_set_host_vlen(int vlend, int vlens) {
  if (vlend <= 0 || vlens <= 0) return 1;
  g_vlend_req = vlend;
  g_vlens_req = vlens;
  return 0;
}

int qwsg_mark_fields_dirty(void) {
  mark_dirty();
  return 0;
}

qwsg_lattice* qwsg_dropin_lattice(void) { return g.lat; }

// qws.cc:130-316 for one process holding the whole lattice
void qws_init_(int* lx, int* ly, int* lz, int* lt, int* npe_f, int* fbc_f, int* pce_f,
               int* pco_f, int* block_size) {
  (void)block_size;  // unused by the reference as well (qws.cc:121-122)
  // the parities of mtilde_vm_/mtilde_s_/bicgstab_vm_ (qws.cc:134-135)
  if (!((*pce_f == 0 && *pco_f == 1) || (*pce_f == 1 && *pco_f == 0)))
    die("qws_init_: pce/pco must be (0,1) or (1,0)");
  g.pce = *pce_f;
  g.pco = *pco_f;
  const char* e;
  g.vlend = g_vlend_req ? g_vlend_req : ((e = getenv("QWSG_VLEND")) ? atoi(e) : 8);
  g.vlens = g_vlens_req ? g_vlens_req : ((e = getenv("QWSG_VLENS")) ? atoi(e) : 16);
  g.always_upload = (e = getenv("QWSG_ALWAYS_UPLOAD")) && atoi(e) != 0;
  for (int i = 0; i < 4; i++) {
    npe[i] = npe_f[i];
    if (npe[i] != 1)
      die("qws_init_: the drop-in runs one GPU holding the whole lattice; npe must be 1 1 1 1 "
          "(use qwsg_create with NB = (2*npe0, npe1, npe2, npe3) for the reference's partition "
          "of a rank grid)");
  }
  nx = *lx;
  ny = *ly;
  nz = *lz;
  nt = *lt;
  nxh = nx / 2;
  nxd = nxh / g.vlend;
  nxs = nxh / g.vlens;
  if (nxd == 0 || nxh % g.vlend) die("qws_init_: nx/2 must be a positive multiple of VLEND");
  if (nxs == 0 || nxh % g.vlens) die("qws_init_: nx/2 must be a positive multiple of VLENS");
  vold = nxd * ny * nz * nt;
  vols = nxs * ny * nz * nt;
  rank = 0;
  domain_e = 0;
  domain_o = 1;
  // fbc (qws.cc:298-310) for a single rank: the t phase is applied on both faces
  for (int mu = 0; mu < 4; mu++) fbc[mu][0] = fbc[mu][1] = 2;
  if (fbc_f[3] != 1) fbc[3][0] = fbc[3][1] = 2.0 * fbc_f[3];
  const size_t V = (size_t)nx * ny * nz * nt;
  void* p;
  if (posix_memalign(&p, CLS, sizeof(double) * 72 * V)) die("qws_init_: out of host memory");
  glud = (pglud_t)p;
  if (posix_memalign(&p, CLS, sizeof(float) * 72 * V)) die("qws_init_: out of host memory");
  glus = (pglus_t)p;
  if (posix_memalign(&p, CLS, sizeof(double) * 72 * V)) die("qws_init_: out of host memory");
  clvd = (pclvd_t)p;
  if (posix_memalign(&p, CLS, sizeof(float) * 72 * V)) die("qws_init_: out of host memory");
  clvs = (pclvs_t)p;
  memset(glud, 0, sizeof(double) * 72 * V);
  memset(glus, 0, sizeof(float) * 72 * V);
  memset(clvd, 0, sizeof(double) * 72 * V);
  memset(clvs, 0, sizeof(float) * 72 * V);
  int L[4] = {nx, ny, nz, nt}, NB[4] = {2, 1, 1, 1};
  if (qwsg_create(&g.lat, L, NB, fbc_f[3] == -1 ? -1 : 1) != 0)
    die(std::string("qws_init_: ") + qwsg_last_error());
  mark_dirty();
  guard("qws_init_", [&] { ensure_planes(ctx()); });
}

void qws_finalize_(void) {
  if (g.lat) {
    cudaStreamSynchronize(g.lat->c->st);
    cudaFree(g.eUd);
    cudaFree(g.eCd);
    cudaFree(g.eUs);
    cudaFree(g.eCs);
    qwsg_destroy(g.lat);
  }
  g.lat = nullptr;
  for (int i = 0; i < 3; i++) g.pd[i] = nullptr, g.ps[i] = nullptr;  // freed with the handle
  for (int i = 0; i < 4; i++) g.ed[i] = nullptr, g.es[i] = nullptr;
  g.eUd = g.eCd = nullptr;
  g.eUs = g.eCs = nullptr;
  free(glud);
  free(glus);
  free(clvd);
  free(clvs);
  glud = nullptr;
  glus = nullptr;
  clvd = nullptr;
  clvs = nullptr;
}

// ---- loaders (qws_bqcd.cc) --------------------------------------------------
}  // extern "C"

// the x position a loader writes site (x,y,z,t) to: the x-halves of the DD
// layout, or the parity slot with x/2 of the even-odd layout (qws_bqcd.cc:82-85)
static inline int slot_x(int x, int eo, bool eo_layout) { return eo_layout ? eo * nxh + x / 2 : x; }

static void load_gauge(double* u, int* volh_tot, double* in_kappa, bool eo_layout) {
  kappa = *in_kappa;
  mkappa = -kappa;
  kappa2 = kappa * kappa;
  double* gd = (double*)glud;
  float* gs = (float*)glus;
#pragma omp parallel for collapse(2)
  for (int t = 0; t < nt; t++)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int j[4] = {x, y, z, t};
          int i = xyzt2i(j), eo = eo_of(j);
          size_t ihh = (size_t)(i - 1) * 18 + (size_t)eo * (*volh_tot) * 18;
          size_t lane_d, lane_s;
          const int xs = slot_x(x, eo, eo_layout);
          size_t ed = qws_elem(xs, y, z, t, g.vlend, &lane_d);
          size_t es = qws_elem(xs, y, z, t, g.vlens, &lane_s);
          int dom = xs / nxh;
          size_t vold_ = (size_t)vold, vols_ = (size_t)vols;
          for (int mu = 0; mu < 4; mu++) {
            // link element: dom*4*vol + mu*vol + in-domain index
            size_t gd_e = ed + (size_t)dom * 3 * vold_ + mu * vold_;
            size_t gs_e = es + (size_t)dom * 3 * vols_ + mu * vols_;
            for (int c1 = 0; c1 < 3; c1++)
              for (int c2 = 0; c2 < 3; c2++)
                for (int ri = 0; ri < 2; ri++) {
                  double v = u[ri + 2 * c1 + 6 * c2 + ihh + (size_t)mu * (*volh_tot) * 36];
                  gd[(gd_e * 18 + (c2 * 3 + c1) * 2 + ri) * g.vlend + lane_d] = v;
                  gs[(gs_e * 18 + (c2 * 3 + c1) * 2 + ri) * g.vlens + lane_s] = (float)v;
                }
          }
        }
  mark_dirty();
}

// BQCD's 36 reals per chiral block -> QWS packing (qws_bqcd.cc:301-377)
static const int kClvPerm[36] = {0,  1,  20, 21, 32, 33, 2,  3,  4,  5,  6,  7,
                                 8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 19,
                                 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 34, 35};

static void load_clover(double* c, int* volh, bool eo_layout) {
  double* cd = (double*)clvd;
  float* cs = (float*)clvs;
#pragma omp parallel for collapse(2)
  for (int t = 0; t < nt; t++)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int j[4] = {x, y, z, t};
          int i = xyzt2i(j), eo = eo_of(j);
          size_t ihh = (size_t)(i - 1) * 72 + (size_t)eo * (*volh) * 72;
          size_t lane_d, lane_s;
          const int xs = slot_x(x, eo, eo_layout);
          size_t ed = qws_elem(xs, y, z, t, g.vlend, &lane_d);
          size_t es = qws_elem(xs, y, z, t, g.vlens, &lane_s);
          for (int ud = 0; ud < 2; ud++)
            for (int k = 0; k < 36; k++) {
              double v = c[kClvPerm[k] + ud * 36 + ihh];
              cd[(ed * 72 + ud * 36 + k) * g.vlend + lane_d] = v;
              cs[(es * 72 + ud * 36 + k) * g.vlens + lane_s] = (float)v;
            }
        }
  mark_dirty();
}

extern "C" {
void qws_loadg_dd_(double* u, int* volh_tot, double* in_kappa) { load_gauge(u, volh_tot, in_kappa, false); }
void qws_loadc_dd_(double* c, int* volh) { load_clover(c, volh, false); }
void qws_loadg_bqcd_(double* u, int* volh_tot, double* in_kappa) { load_gauge(u, volh_tot, in_kappa, true); }
void qws_loadc_bqcd_(double* c, int* volh) { load_clover(c, volh, true); }
}  // extern "C"

template <typename R>
static void loadf(R* out, const double* ine, const double* ino, int vlen) {
#pragma omp parallel for collapse(2)
  for (int t = 0; t < nt; t++)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int j[4] = {x, y, z, t};
          int i = xyzt2i(j), eo = eo_of(j);
          size_t ihh = (size_t)(i - 1) * 24;
          size_t lane;
          size_t e = qws_elem(x, y, z, t, vlen, &lane);
          const double* src = eo == 0 ? ine : ino;
          for (int c = 0; c < 3; c++)
            for (int s = 0; s < 4; s++)
              for (int ri = 0; ri < 2; ri++)
                out[(e * 24 + c * 8 + s * 2 + ri) * vlen + lane] = (R)src[ri + 2 * s + 8 * c + ihh];
        }
}

template <typename R>
static void storef(double* oute, double* outo, const R* in, int vlen) {
#pragma omp parallel for collapse(2)
  for (int t = 0; t < nt; t++)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int j[4] = {x, y, z, t};
          int i = xyzt2i(j), eo = eo_of(j);
          size_t ihh = (size_t)(i - 1) * 24;
          size_t lane;
          size_t e = qws_elem(x, y, z, t, vlen, &lane);
          double* dst = eo == 0 ? oute : outo;
          for (int c = 0; c < 3; c++)
            for (int s = 0; s < 4; s++)
              for (int ri = 0; ri < 2; ri++)
                dst[ri + 2 * s + 8 * c + ihh] = (double)in[(e * 24 + c * 8 + s * 2 + ri) * vlen + lane];
        }
}

// the even sites only, into / out of a half array of the even-odd layout
// (qws_bqcd.cc:384-498)
template <typename R>
static void loadf_even(R* out, const double* in, int vlen) {
#pragma omp parallel for collapse(2)
  for (int t = 0; t < nt; t++)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int j[4] = {x, y, z, t};
          if (eo_of(j) != 0) continue;
          size_t ihh = (size_t)(xyzt2i(j) - 1) * 24;
          size_t lane;
          size_t e = qws_elem(x / 2, y, z, t, vlen, &lane);
          for (int c = 0; c < 3; c++)
            for (int s = 0; s < 4; s++)
              for (int ri = 0; ri < 2; ri++)
                out[(e * 24 + c * 8 + s * 2 + ri) * vlen + lane] = (R)in[ri + 2 * s + 8 * c + ihh];
        }
}

template <typename R>
static void storef_even(double* out, const R* in, int vlen) {
#pragma omp parallel for collapse(2)
  for (int t = 0; t < nt; t++)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int j[4] = {x, y, z, t};
          if (eo_of(j) != 0) continue;
          size_t ihh = (size_t)(xyzt2i(j) - 1) * 24;
          size_t lane;
          size_t e = qws_elem(x / 2, y, z, t, vlen, &lane);
          for (int c = 0; c < 3; c++)
            for (int s = 0; s < 4; s++)
              for (int ri = 0; ri < 2; ri++)
                out[ri + 2 * s + 8 * c + ihh] = (double)in[(e * 24 + c * 8 + s * 2 + ri) * vlen + lane];
        }
}

extern "C" {

void qws_loadfd_bqcd_(scd_t* out, double* in) { loadf_even<double>((double*)out, in, g.vlend); }
void qws_loadfs_bqcd_(scs_t* out, double* in) { loadf_even<float>((float*)out, in, g.vlens); }
void qws_storefd_bqcd_(double* out, scd_t* in) { storef_even<double>(out, (const double*)in, g.vlend); }
void qws_storefs_bqcd_(double* out, scs_t* in) { storef_even<float>(out, (const float*)in, g.vlens); }

void qws_loadfd_dd_(scd_t* out, double* ine, double* ino) { loadf<double>((double*)out, ine, ino, g.vlend); }
void qws_storefd_dd_(double* oute, double* outo, scd_t* in) { storef<double>(oute, outo, (const double*)in, g.vlend); }
void qws_loadfs_dd_(scs_t* out, double* ine, double* ino) { loadf<float>((float*)out, ine, ino, g.vlens); }
void qws_storefs_dd_(double* oute, double* outo, scs_t* in) { storef<float>(oute, outo, (const float*)in, g.vlens); }

// ---- solvers ----------------------------------------------------------------
void bicgstab_dd_mix_(scd_t* x, scd_t* b, double* tol, int* conviter, int* maxiter, double* tol_s,
                      int* maxiter_s, int* nsap, int* nm) {
  guard("bicgstab_dd_mix_", [&] {
    Ctx& c = ctx();
    double t0 = wall();
    sync_fields(c);
    up<double>(c, g.pd[1], b, -1, g.vlend);
    up<double>(c, g.pd[0], x, -1, g.vlend);
    SolveStats st;
    bicgstab_dd_mix(c, g.pd[0], g.pd[1], *tol, *maxiter, *tol_s, *maxiter_s, *nsap, *nm, &st,
                    nullptr, 0);
    down<double>(c, x, g.pd[0], -1, g.vlend);
    *conviter = st.outer_iters;
    g.t_solver += wall() - t0;
    g.n_calls_dd_mix++;
  });
}

void bicgstab_precdd_s_(scs_t* x, scs_t* b, double* tol, int* conviter, int* maxiter, int* nsap,
                        int* nm) {
  guard("bicgstab_precdd_s_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    up<float>(c, g.ps[1], b, -1, g.vlens);
    int it = bicgstab_precdd_s(c, g.ps[0], g.ps[1], *tol, *maxiter, *nsap, *nm, nullptr);
    down<float>(c, x, g.ps[0], -1, g.vlens);
    *conviter = it;
  });
}

// half-precision pair: the FP16 copies are made from the resident FP32 fields
// on first use, so qws_h_init_ only has to mark the host fields as current
// (qws_h.cc:150-166 converts glus/clvs itself)
void qws_h_init_(const glus_t* g_s, const clvs_t* c_s) {
  (void)g_s;
  (void)c_s;
  mark_dirty();
}
void bqcd_qws_h_init_(void) { qws_h_init_(glus, clvs); }

void assign_mult_mSAP_s_h_(scs_t* xs, const scs_t* bs, const int* nsap, const int* nm) {
  guard("assign_mult_mSAP_s_h_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    up<float>(c, g.ps[1], bs, -1, g.vlens);
    prec_s_h(c, g.ps[0], g.ps[1], *nsap, *nm);
    down<float>(c, xs, g.ps[0], -1, g.vlens);
  });
}

// assign_mult_wd_s_ (prec_ddd_s_h.h:233-277): the FP32 D
void assign_mult_wd_s_(scs_t* x, const scs_t* b) { ddd_s_(x, (scs_t*)b); }

void bicgstab_precdd_s_h_(scs_t* x, const scs_t* b, const double* tol, int* conviter,
                          const int* maxiter, const int* nsap, const int* nm) {
  guard("bicgstab_precdd_s_h_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    up<float>(c, g.ps[1], b, -1, g.vlens);
    int it = bicgstab_precdd_s_h(c, g.ps[0], g.ps[1], *tol, *maxiter, *nsap, *nm, nullptr);
    down<float>(c, x, g.ps[0], -1, g.vlens);
    *conviter = it;
  });
}

void bicgstab_dd_mix2_hf_(scd_t* x, const scd_t* b, const double* tol, int* conviter,
                          const int* maxiter, const double* tol_s, const int* maxiter_s,
                          const int* nsap, const int* nm) {
  guard("bicgstab_dd_mix2_hf_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    up<double>(c, g.pd[1], b, -1, g.vlend);
    up<double>(c, g.pd[0], x, -1, g.vlend);
    SolveStats st;
    bicgstab_dd_mix2_hf(c, g.pd[0], g.pd[1], *tol, *maxiter, *tol_s, *maxiter_s, *nsap, *nm, 0,
                        &st);
    down<double>(c, x, g.pd[0], -1, g.vlend);
    *conviter = st.outer_iters;
  });
}

void prec_ddd_s_(scs_t* out, scs_t* in, int* nsap, int* nm) {
  guard("prec_ddd_s_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    up<float>(c, g.ps[1], in, -1, g.vlens);
    prec_ddd_s(c, g.ps[0], g.ps[1], *nsap, *nm);
    down<float>(c, out, g.ps[0], -1, g.vlens);
  });
}

void prec_s_(scs_t* out, scs_t* in, int* nsap, int* nm) {
  guard("prec_s_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    up<float>(c, g.ps[1], in, -1, g.vlens);
    prec_s(c, g.ps[0], g.ps[1], *nsap, *nm);
    down<float>(c, out, g.ps[0], -1, g.vlens);
  });
}

void jinv_ddd_in_s_(scs_t* x, scs_t* b, int* DEO, int* maxiter) {
  guard("jinv_ddd_in_s_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    up<float>(c, g.ps[1], b, *DEO, g.vlens);
    jinv_s(c, g.ps[0], g.ps[1], *DEO, *maxiter);
    down<float>(c, x, g.ps[0], *DEO, g.vlens);
  });
}

// ---- DD operator ------------------------------------------------------------
void ddd_d_(scd_t* out, scd_t* in) {
  guard("ddd_d_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    up<double>(c, g.pd[1], in, -1, g.vlend);
    dslash_full_d(c, g.pd[0], g.pd[1]);
    down<double>(c, out, g.pd[0], -1, g.vlend);
  });
}

void ddd_s_(scs_t* out, scs_t* in) {
  guard("ddd_s_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    up<float>(c, g.ps[1], in, -1, g.vlens);
    dslash_full_s(c, g.ps[0], g.ps[1]);
    down<float>(c, out, g.ps[0], -1, g.vlens);
  });
}

// ddd_eo_s_ (qws.cc:634-639): D on the half of the full arrays of one domain
void ddd_eo_s_(scs_t* out, scs_t* in, int* domain) {
  guard("ddd_eo_s_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    const int d = *domain;
    up<float>(c, g.ps[1], in, -1, g.vlens);
    dslash_inner<float>(c, g.ps[0], g.ps[1], d, -1);
    dslash_outer<float>(c, g.ps[0], g.ps[1], d, -1, -c.kappa, -1);
    // the other half of `out` is left as the caller had it
    float* half = (float*)out + (size_t)d * c.G.Vh * 24;
    down<float>(c, half, g.ps[0], d, g.vlens);
  });
}

void ddd_in_d_(scd_t* out, scd_t* in, int* DEO) {
  guard("ddd_in_d_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    up<double>(c, g.pd[1], in, *DEO, g.vlend);
    dslash_inner<double>(c, g.pd[0], g.pd[1], *DEO, -1);
    down<double>(c, out, g.pd[0], *DEO, g.vlend);
  });
}

void ddd_in_s_(scs_t* out, scs_t* in, int* DEO) {
  guard("ddd_in_s_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    up<float>(c, g.ps[1], in, *DEO, g.vlens);
    dslash_inner<float>(c, g.ps[0], g.ps[1], *DEO, -1);
    down<float>(c, out, g.ps[0], *DEO, g.vlens);
  });
}

// pre: capture the faces = keep a device copy of the whole field
void ddd_out_pre_d_(scd_t* in, int* DEO) {
  (void)DEO;
  guard("ddd_out_pre_d_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    up<double>(c, g.pd[2], in, -1, g.vlend);
  });
}

void ddd_out_pos_d_(scd_t* out, scd_t* in, int* DEO) {
  (void)in;
  guard("ddd_out_pos_d_", [&] {
    Ctx& c = ctx();
    up<double>(c, g.pd[0], out, *DEO, g.vlend);
    dslash_outer<double>(c, g.pd[0], g.pd[2], *DEO, -1, -c.kappa, -1);
    down<double>(c, out, g.pd[0], *DEO, g.vlend);
  });
}

void ddd_out_pre_s_(scs_t* in, int* DEO) {
  (void)DEO;
  guard("ddd_out_pre_s_", [&] {
    Ctx& c = ctx();
    sync_fields(c);
    up<float>(c, g.ps[2], in, -1, g.vlens);
  });
}

void ddd_out_pos_s_(scs_t* out, scs_t* in, int* DEO, float factor) {
  (void)in;
  guard("ddd_out_pos_s_", [&] {
    Ctx& c = ctx();
    up<float>(c, g.ps[0], out, *DEO, g.vlens);
    dslash_outer<float>(c, g.ps[0], g.ps[2], *DEO, -1, factor, -1);
    down<float>(c, out, g.ps[0], *DEO, g.vlens);
  });
}

void ddd_out_pre_s_no_timer_(scs_t* in, int* DEO) { ddd_out_pre_s_(in, DEO); }
void ddd_out_pos_s_no_timer_(scs_t* out, scs_t* in, int* DEO, float factor) {
  ddd_out_pos_s_(out, in, DEO, factor);
}

}  // extern "C"

// ---- even-odd (site parity) family (qws.cc:390-605, deo_*.cc) --------------
// Arguments are one-parity half arrays (vol elements, x/2 compressed):
// `out` of parity pe, `in` of parity po = 1 - pe, `in0` of parity pe.
namespace {

struct EoOp {
  int which, dag, clov, mode;  // hop set (1 in, 2 out, 3 all), adjoint, A^-1, store mode
};
constexpr EoOp kIn{1, 0, 0, 0}, kDeeIn{1, 0, 1, 0}, kDagIn{1, 1, 0, 0}, kDeeDagIn{1, 1, 1, 0},
    kOmDeeIn{1, 0, 1, 2}, kOmDagIn{1, 1, 0, 2}, kPos{2, 0, 0, 1}, kDagPos{2, 1, 0, 1},
    kDeePos{2, 0, 1, 1}, kDeeDagPos{2, 1, 1, 1}, kAll{3, 0, 0, 0}, kDeeAll{3, 0, 1, 0},
    kDagAll{3, 1, 0, 0}, kDeeDagAll{3, 1, 1, 0}, kOmDeeAll{3, 0, 1, 2}, kOmDagAll{3, 1, 0, 2};

void check_parities(const char* name, const int* pe, const int* po) {
  if (!((*pe == 0 && *po == 1) || (*pe == 1 && *po == 0)))
    die(std::string(name) + ": parities must be (0,1) or (1,0)");
}

template <typename R>
int eo_vlen() {
  return sizeof(R) == 8 ? g.vlend : g.vlens;
}
template <typename R>
R** eo_planes();
template <>
double** eo_planes<double>() {
  return g.ed;
}
template <>
float** eo_planes<float>() {
  return g.es;
}

// out = op(in); pos ops (OUT hops, mode 1) read the snapshot taken by the pre
template <typename R>
void eo_apply(const char* name, const int* pe, const int* po, void* out, const void* in,
              const void* in0, EoOp op, double factor) {
  check_parities(name, pe, po);
  guard(name, [&] {
    Ctx& c = ctx();
    sync_eo(c);
    R** P = eo_planes<R>();
    const int vl = eo_vlen<R>();
    const R* src = P[3];
    if (op.which != 2) {
      up_eo<R>(c, P[1], in, *po, vl);
      src = P[1];
    }
    if (op.mode == 1) up_eo<R>(c, P[0], out, *pe, vl);
    if (op.mode == 2) up_eo<R>(c, P[2], in0, *pe, vl);
    deo<R>(c, P[0], src, *pe, op.which, op.dag, op.clov, op.mode, factor,
           op.mode == 2 ? P[2] : nullptr);
    down_eo<R>(c, out, P[0], *pe, vl);
  });
}

// deo_out_pre: keep the field whose faces the following pos reads
template <typename R>
void eo_pre(const char* name, const int* pe, const int* po, const void* in) {
  check_parities(name, pe, po);
  guard(name, [&] {
    Ctx& c = ctx();
    sync_eo(c);
    up_eo<R>(c, eo_planes<R>()[3], in, *po, eo_vlen<R>());
  });
}

template <typename R>
void eo_clover(const char* name, const int* pe, void* out, const void* in) {
  if (*pe != 0 && *pe != 1) die(std::string(name) + ": parity must be 0 or 1");
  guard(name, [&] {
    Ctx& c = ctx();
    sync_eo(c);
    R** P = eo_planes<R>();
    up_eo<R>(c, P[1], in, *pe, eo_vlen<R>());
    clv<R>(c, P[0], P[1], *pe);
    down_eo<R>(c, out, P[0], *pe, eo_vlen<R>());
  });
}

// mtilde family on parity-pce half arrays
template <typename R, typename F>
void eo_mtilde(const char* name, void* out, const void* in, F&& f) {
  guard(name, [&] {
    Ctx& c = ctx();
    sync_eo(c);
    R** P = eo_planes<R>();
    up_eo<R>(c, P[1], in, g.pce, eo_vlen<R>());
    f(c, P[0], P[1]);
    down_eo<R>(c, out, P[0], g.pce, eo_vlen<R>());
  });
}

}  // namespace

extern "C" {

void deo_in_vm_(int* pe, int* po, scd_t* out, scd_t* in) {
  eo_apply<double>("deo_in_vm_", pe, po, out, in, nullptr, kIn, 0);
}
void dee_deo_in_vm_(int* pe, int* po, scd_t* out, scd_t* in) {
  eo_apply<double>("dee_deo_in_vm_", pe, po, out, in, nullptr, kDeeIn, 0);
}
void deo_dag_in_vm_(int* pe, int* po, scd_t* out, scd_t* in) {
  eo_apply<double>("deo_dag_in_vm_", pe, po, out, in, nullptr, kDagIn, 0);
}
void dee_deo_dag_in_vm_(int* pe, int* po, scd_t* out, scd_t* in) {
  eo_apply<double>("dee_deo_dag_in_vm_", pe, po, out, in, nullptr, kDeeDagIn, 0);
}
void one_minus_dee_deo_in_vm_(int* pe, int* po, scd_t* out, scd_t* in, scd_t* in0, double factor) {
  eo_apply<double>("one_minus_dee_deo_in_vm_", pe, po, out, in, in0, kOmDeeIn, factor);
}
void one_minus_deo_dag_in_vm_(int* pe, int* po, scd_t* out, scd_t* in, scd_t* in0, double factor) {
  eo_apply<double>("one_minus_deo_dag_in_vm_", pe, po, out, in, in0, kOmDagIn, factor);
}
void deo_out_pre_vm_(int* pe, int* po, scd_t* out, scd_t* in) {
  (void)out;
  eo_pre<double>("deo_out_pre_vm_", pe, po, in);
}
void deo_dag_out_pre_vm_(int* pe, int* po, scd_t* out, scd_t* in) {
  (void)out;
  eo_pre<double>("deo_dag_out_pre_vm_", pe, po, in);
}
void deo_out_pos_vm_(int* pe, int* po, scd_t* out, scd_t* in, double factor) {
  eo_apply<double>("deo_out_pos_vm_", pe, po, out, in, nullptr, kPos, factor);
}
void deo_dag_out_pos_vm_(int* pe, int* po, scd_t* out, scd_t* in, double factor) {
  eo_apply<double>("deo_dag_out_pos_vm_", pe, po, out, in, nullptr, kDagPos, factor);
}
void dee_deo_out_pos_vm_(int* pe, int* po, scd_t* out, scd_t* in, double factor) {
  eo_apply<double>("dee_deo_out_pos_vm_", pe, po, out, in, nullptr, kDeePos, factor);
}
void dee_deo_dag_out_pos_vm_(int* pe, int* po, scd_t* out, scd_t* in, double factor) {
  eo_apply<double>("dee_deo_dag_out_pos_vm_", pe, po, out, in, nullptr, kDeeDagPos, factor);
}
void clvd_vm_(int* pe, scd_t* inout) { eo_clover<double>("clvd_vm_", pe, inout, inout); }
void clvd_vm2_(int* pe, scd_t* out, scd_t* in) { eo_clover<double>("clvd_vm2_", pe, out, in); }
void deo_vm_(int* pe, int* po, scd_t* out, scd_t* in) {
  eo_apply<double>("deo_vm_", pe, po, out, in, nullptr, kAll, 0);
}
void dee_deo_vm_(int* pe, int* po, scd_t* out, scd_t* in) {
  eo_apply<double>("dee_deo_vm_", pe, po, out, in, nullptr, kDeeAll, 0);
}
void one_minus_dee_deo_vm_(int* pe, int* po, scd_t* out, scd_t* in, scd_t* in0) {
  eo_apply<double>("one_minus_dee_deo_vm_", pe, po, out, in, in0, kOmDeeAll, -kappa2);
}
void deo_dag_vm_(int* pe, int* po, scd_t* out, scd_t* in) {
  eo_apply<double>("deo_dag_vm_", pe, po, out, in, nullptr, kDagAll, 0);
}
void dee_deo_dag_vm_(int* pe, int* po, scd_t* out, scd_t* in) {
  eo_apply<double>("dee_deo_dag_vm_", pe, po, out, in, nullptr, kDeeDagAll, 0);
}
void one_minus_deo_dag_vm_(int* pe, int* po, scd_t* out, scd_t* in, scd_t* in0) {
  eo_apply<double>("one_minus_deo_dag_vm_", pe, po, out, in, in0, kOmDagAll, -kappa2);
}
void mtilde_vm_(scd_t* out, scd_t* in) {
  eo_mtilde<double>("mtilde_vm_", out, in,
                    [](Ctx& c, double* o, const double* i) { mtilde_d(c, o, i); });
}
void mtilde_dag_vm_(scd_t* out, scd_t* in) {
  eo_mtilde<double>("mtilde_dag_vm_", out, in,
                    [](Ctx& c, double* o, const double* i) { mtilde_dag_d(c, o, i); });
}
void mtdagmt_vm_(scd_t* out, scd_t* in) {
  eo_mtilde<double>("mtdagmt_vm_", out, in, [](Ctx& c, double* o, const double* i) {
    double* t = g.ed[2];
    mtilde_d(c, t, i);
    mtilde_dag_d(c, o, t);
  });
}
// bicgstab.cc:68-333: x (initial guess in, solution out) and b are parity-pce half arrays
void bicgstab_vm_(scd_t* x, scd_t* b, int* conviter, int* maxiter) {
  guard("bicgstab_vm_", [&] {
    Ctx& c = ctx();
    sync_eo(c);
    double** P = g.ed;
    up_eo<double>(c, P[0], x, g.pce, g.vlend);
    up_eo<double>(c, P[1], b, g.pce, g.vlend);
    *conviter = bicgstab_vm(c, P[0], P[1], *maxiter);
    down_eo<double>(c, x, P[0], g.pce, g.vlend);
  });
}

// cg.cc:65-172: x (initial guess in, solution out) and b are parity-pce half arrays
void cg_vm_(scd_t* x, scd_t* b, int* conviter, int* maxiter) {
  guard("cg_vm_", [&] {
    Ctx& c = ctx();
    sync_eo(c);
    double** P = g.ed;
    up_eo<double>(c, P[0], x, g.pce, g.vlend);
    up_eo<double>(c, P[1], b, g.pce, g.vlend);
    const int it = cg_vm(c, P[0], P[1], *maxiter);
    if (conviter) *conviter = it;
    down_eo<double>(c, x, P[0], g.pce, g.vlend);
  });
}
// mcg.cc:65-219: *n solutions, each a parity-pce half array, back to back in xx
void mcg_vm_(scd_t* xx, scd_t* b, int* n, double* sigma, int* maxiter) {
  guard("mcg_vm_", [&] {
    Ctx& c = ctx();
    sync_eo(c);
    if (*n < 1 || *n > Ctx::kMaxRhs) throw Error(1, "mcg_vm_: number of shifts must be 1..32");
    double** P = g.ed;
    up_eo<double>(c, P[1], b, g.pce, g.vlend);
    double* X = nullptr;
    QWSG_CUDA(cudaMalloc(&X, sizeof(double) * c.spinor_elems() * *n));
    try {
      mcg_vm(c, X, P[1], *n, sigma, *maxiter);
      const size_t half = (size_t)c.G.Vh * 24;  // reals of one half array
      for (int k = 0; k < *n; k++)
        down_eo<double>(c, (double*)xx + k * half, X + k * c.spinor_elems(), g.pce, g.vlend);
      QWSG_CUDA(cudaStreamSynchronize(c.st));
    } catch (...) {
      cudaStreamSynchronize(c.st);
      cudaFree(X);
      throw;
    }
    QWSG_CUDA(cudaFree(X));
  });
}

void deo_in_s_(int* pe, int* po, scs_t* out, scs_t* in) {
  eo_apply<float>("deo_in_s_", pe, po, out, in, nullptr, kIn, 0);
}
void dee_deo_in_s_(int* pe, int* po, scs_t* out, scs_t* in) {
  eo_apply<float>("dee_deo_in_s_", pe, po, out, in, nullptr, kDeeIn, 0);
}
void one_minus_dee_deo_in_s_(int* pe, int* po, scs_t* out, scs_t* in, scs_t* in0, float factor) {
  eo_apply<float>("one_minus_dee_deo_in_s_", pe, po, out, in, in0, kOmDeeIn, factor);
}
// deo_out_{pre,pos}_s_ take const pointers in the reference (qws.cc:577-578); pos writes out
void deo_out_pre_s_(const int* pe, const int* po, const scs_t* out, const scs_t* in) {
  (void)out;
  eo_pre<float>("deo_out_pre_s_", pe, po, in);
}
void deo_out_pos_s_(const int* pe, const int* po, const scs_t* out, const scs_t* in, float factor) {
  eo_apply<float>("deo_out_pos_s_", pe, po, (void*)out, in, nullptr, kPos, factor);
}
void dee_deo_out_pos_s_(int* pe, int* po, scs_t* out, scs_t* in, float factor) {
  eo_apply<float>("dee_deo_out_pos_s_", pe, po, out, in, nullptr, kDeePos, factor);
}
void clv_s_(int* pe, scs_t* inout) { eo_clover<float>("clv_s_", pe, inout, inout); }
void deo_s_(int* pe, int* po, scs_t* out, scs_t* in) {
  eo_apply<float>("deo_s_", pe, po, out, in, nullptr, kAll, 0);
}
void dee_deo_s_(int* pe, int* po, scs_t* out, scs_t* in) {
  eo_apply<float>("dee_deo_s_", pe, po, out, in, nullptr, kDeeAll, 0);
}
void one_minus_dee_deo_s_(int* pe, int* po, scs_t* out, scs_t* in, scs_t* in0) {
  eo_apply<float>("one_minus_dee_deo_s_", pe, po, out, in, in0, kOmDeeAll,
                  (double)(-(float)kappa2));
}
void mtilde_s_(scs_t* out, scs_t* in) {
  eo_mtilde<float>("mtilde_s_", out, in,
                   [](Ctx& c, float* o, const float* i) { mtilde_s(c, o, i); });
}

// ---- converters (reordering.cc) ---------------------------------------------
void fermi_reorder_s2d_dd_(scd_t* out, const scs_t* in) {
  guard("fermi_reorder_s2d_dd_", [&] {
    Ctx& c = ctx();
    up<float>(c, g.ps[0], in, -1, g.vlens);
    blas_s2d(c.G, g.pd[0], g.ps[0], 1.0, c.st);
    down<double>(c, out, g.pd[0], -1, g.vlend);
  });
}

void fermi_reorder_d2s_dd_(scs_t* out, const scd_t* in) {
  guard("fermi_reorder_d2s_dd_", [&] {
    Ctx& c = ctx();
    up<double>(c, g.pd[0], in, -1, g.vlend);
    blas_d2s(c.G, g.ps[0], g.pd[0], 1.0, c.st);
    down<float>(c, out, g.ps[0], -1, g.vlens);
  });
}

void fermi_reorder_s2d_dd_renorm_(scd_t* out, const scs_t* in, const double* dnorm) {
  guard("fermi_reorder_s2d_dd_renorm_", [&] {
    Ctx& c = ctx();
    up<float>(c, g.ps[0], in, -1, g.vlens);
    blas_s2d(c.G, g.pd[0], g.ps[0], *dnorm, c.st);
    down<double>(c, out, g.pd[0], -1, g.vlend);
  });
}

void fermi_reorder_d2s_dd_renorm_(scs_t* out, const scd_t* in, double* dnorm) {
  guard("fermi_reorder_d2s_dd_renorm_", [&] {
    Ctx& c = ctx();
    up<double>(c, g.pd[0], in, -1, g.vlend);
    blas_norm2<double>(c.G, g.pd[0], c.d_res, c.rb, c.st);
    const double n = std::sqrt(c.fetch(1)[0]);
    *dnorm = n;
    blas_d2s(c.G, g.ps[0], g.pd[0], 1.0 / n, c.st);
    down<float>(c, out, g.ps[0], -1, g.vlens);
  });
}

// ---- helpers ----------------------------------------------------------------
void print_scdnorm2(const char* a, scd_t* in, int size) {
  const double* p = (const double*)in;
  const size_t n = (size_t)size * 24 * g.vlend;
  double r = 0;
#pragma omp parallel for reduction(+ : r)
  for (size_t i = 0; i < n; i++) r += p[i] * p[i];
  printf("%30s : %24.14e\n", a, r);
  fflush(stdout);
}

void print_scsnorm2(const char* a, scs_t* in, int size) {
  const float* p = (const float*)in;
  const size_t n = (size_t)size * 24 * g.vlens;
  double r = 0;
#pragma omp parallel for reduction(+ : r)
  for (size_t i = 0; i < n; i++) r += (double)p[i] * p[i];
  printf("%30s : %24.14e\n", a, (double)(float)r);
  fflush(stdout);
}

void zero_scd_field(scd_t* inout, int size) { memset(inout, 0, sizeof(double) * 24 * g.vlend * (size_t)size); }
void zero_scs_field(scs_t* inout, int size) { memset(inout, 0, sizeof(float) * 24 * g.vlens * (size_t)size); }

double get_clock(void) { return wall(); }

// region table in the spirit of timing.c:81-185 (call counts of this library)
void print_timing_(void) {
  if (!g.lat) return;
  Ctx& c = *g.lat->c;
  printf("    rank\tfunc_id                         \t   calls\n");
  printf("       0\t%-32s\t%8ld\n", "bicgstab_dd_mix_", g.n_calls_dd_mix);
  printf("       0\t%-32s\t%8ld\n", "bicgstab_precdd_s_iter_", c.n_inner_iter);
  printf("       0\t%-32s\t%8ld\n", "prec_ddd_s_", c.n_prec_ddd);
  printf("       0\t%-32s\t%8ld\n", "prec_s_", c.n_prec_s);
  printf("       0\t%-32s\t%8ld\n", "jinv_ddd_in_s_", c.n_jinv);
  printf("       0\t%-32s\t%8ld\n", "ddd_d_", c.n_dslash_d);
  fflush(stdout);
}

}  // extern "C"
