// Host orchestration of the DD solver on the GPU: SAP preconditioner and the
// BiCGStab loops.  Follows the reference's algorithms step by step
// (qws.cc:776-975, static_solver.cc:65-140, bicgstab_precdd_s.cc:85-559,
// bicgstab_dd_mix.cc:76-388, and the half-precision pair
// bicgstab_precdd_s_h.cc:83-369 / bicgstab_dd_mix2_hf.cc:88-373) with its
// halo/aliasing bookkeeping replaced by fused kernels over the resident
// lattice.  The SAP sweep is written once for every storage format (FP32,
// FP16 with per-site scales).
#include <algorithm>
#include <initializer_list>
#include <cmath>
#include <cstring>

#include "ctx.h"

namespace qwsg {

namespace {

template <typename T>
HopArgs<T> hop_args(const Geom& G, const typename Store<T>::type* U,
                    const typename Store<T>::type* C) {
  HopArgs<T> a{};
  a.G = G;
  a.U = U;
  a.C = C;
  a.dom = -1;
  a.zero_col = -1;
  return a;
}

// the resident fields of the handle; FP32 launches read the 12-real links
// when they are on
template <typename T>
HopArgs<T> hop_args_c(Ctx& c);
// (with per-RHS kappa: the handle's clover planes and kappa tables)
template <>
HopArgs<float> hop_args_c<float>(Ctx& c) {
  c.ensure_links12();
  auto a = hop_args<float>(c.G, c.Us, c.Cs);
  a.U12 = c.links12_on ? c.Us12 : nullptr;
  if (!c.rhs_kappas.empty()) {
    a.Cr = c.Csr;
    a.kap = c.kap_s;
  }
  return a;
}
template <>
HopArgs<double> hop_args_c<double>(Ctx& c) {
  auto a = hop_args<double>(c.G, c.Ud, c.Cd);
  if (!c.rhs_kappas.empty()) {
    a.Cr = c.Cdr;
    a.kap = c.kap_d;
  }
  return a;
}
template <>
HopArgs<H16> hop_args_c<H16>(Ctx& c) {
  auto a = hop_args<H16>(c.G, c.Uh, c.Ch);
  if (!c.rhs_kappas.empty()) {
    a.Cr = c.Chr;
    a.kap = c.kap_s;
  }
  return a;
}

// algorithmic bytes moved per handled site: each spinor stream once per
// right-hand side, links and clover once per site (48 B less per link
// direction pair for 12-real FP32 links)
template <typename T>
double hop_bytes(int sel, int epi, int nr, bool links12 = false) {
  const double sp = Bytes<T>::spinor * nr,
               lc = (links12 ? Bytes<T>::links * 2 / 3 : Bytes<T>::links) + Bytes<T>::clover;
  if (epi == EPI_JINV) return 3 * sp + lc;  // src, b, out
  if (epi == EPI_SAPE) return 4 * sp + lc;  // a, in, s (r+w)
  // out (r+w), one face neighbour and its one link (a face site has 1.1
  // face hops on average at the reference partition), clover
  if (epi == EPI_ADD)
    return 3 * sp + (links12 ? Bytes<T>::links * 2 / 3 : Bytes<T>::links) / 4 + Bytes<T>::clover;
  (void)sel;
  return 2 * sp + lc;                       // in, out
}

template <typename T>
int kind_of(int sel, int epi) {
  const bool d = sizeof(typename Store<T>::type) == 8;
  const bool h = sizeof(typename Store<T>::type) == 2;
  if (sel == HOP_ALL) return d ? K_D_F64 : K_D_F32;
  if (sel == HOP_OUTER) return h ? K_OUT_F16 : d ? K_OUT_F64 : K_OUT_F32;
  if (epi == EPI_JINV) return h ? K_JINV_F16 : K_JINV_F32;
  if (epi == EPI_SAPE) return h ? K_SAPE_F16 : K_SAPE_F32;
  return h ? K_DIN_F16 : d ? K_DIN_F64 : K_DIN_F32;
}

// sites of one colour that touch a block face
long face_sites_per_colour(const Geom& G) {
  long inner = 1;
  for (int mu = 0; mu < 4; mu++) inner *= (G.B[mu] > 2 ? G.B[mu] - 2 : 0);
  long nblk_c = (long)G.NB[0] * G.NB[1] * G.NB[2] * G.NB[3] / 2;
  return nblk_c * (G.Vb - inner);
}

template <typename T>
void run_hop(Ctx& c, int sel, int epi, const HopArgs<T>& a) {
  if (!c.timing) {
    launch_hop<T>(sel, epi, a, c.st);
    return;
  }
  cudaEvent_t e0 = c.next_event(), e1 = c.next_event();
  QWSG_CUDA(cudaEventRecord(e0, c.st));
  launch_hop<T>(sel, epi, a, c.st);
  QWSG_CUDA(cudaEventRecord(e1, c.st));
  long sites = a.nsites;
  if (sel == HOP_OUTER && !a.list) sites = face_sites_per_colour(c.G) * (a.nsites == c.G.V ? 2 : 1);
  if (a.dom >= 0) sites /= 2;
  c.recs.push_back({kind_of<T>(sel, epi), e0, e1,
                    (double)sites * hop_bytes<T>(sel, epi, c.G.nr, a.U12 != nullptr)});
}

void site_range(const Ctx& c, int col, int& site0, int& n) {
  if (col >= 0) {
    site0 = col * c.G.Vh;
    n = c.G.Vh;
  } else {
    site0 = 0;
    n = c.G.V;
  }
}

}  // namespace

const char* kernel_kind_name(int k) {
  static const char* n[K_NKIND] = {"dslash_full_f64", "dslash_full_f32", "dslash_block_f64",
                                   "dslash_block_f32", "jinv_step_f32", "sap_update_f32",
                                   "dslash_face_f64", "dslash_face_f32", "jinv_step_f16",
                                   "sap_update_f16", "dslash_face_f16", "dslash_block_f16"};
  return (k >= 0 && k < K_NKIND) ? n[k] : "?";
}

cudaEvent_t Ctx::next_event() {
  if (ev_next == ev_pool.size()) {
    cudaEvent_t e;
    QWSG_CUDA(cudaEventCreate(&e));
    ev_pool.push_back(e);
  }
  return ev_pool[ev_next++];
}

void kernel_stats(Ctx& c, long* launches, double* ms, double* bytes) {
  QWSG_CUDA(cudaStreamSynchronize(c.st));
  for (const auto& r : c.recs) {
    float t = 0;
    QWSG_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
    launches[r.kind] += 1;
    ms[r.kind] += t;
    bytes[r.kind] += r.bytes;
  }
  c.recs.clear();
  c.ev_next = 0;
}

Ctx::Ctx(const int L[4], const int NB[4], int tbc, int nrhs) {
  if (nrhs < 1 || nrhs > kMaxRhs || (nrhs & (nrhs - 1)))
    throw Error(1, "number of right-hand sides must be a power of two in 1..32");
  G.nr = nrhs;
  G.hop_threads = 128;
  G.lgnr = 0;
  while ((1 << G.lgnr) < nrhs) G.lgnr++;
  for (int mu = 0; mu < 4; mu++) {
    if (L[mu] <= 0 || NB[mu] <= 0 || L[mu] % NB[mu] != 0)
      throw Error(1, "lattice extent not divisible by the block grid");
    G.L[mu] = L[mu];
    G.NB[mu] = NB[mu];
    G.B[mu] = L[mu] / NB[mu];
  }
  if (NB[0] % 2 != 0) throw Error(1, "block grid NB[0] must be even (two x-halves per rank)");
  for (int mu = 1; mu < 4; mu++)
    if (NB[mu] != 1 && NB[mu] % 2 != 0)
      throw Error(1, "block grid NB[1..3] must be 1 or even (red-black block colouring)");
  long V = (long)L[0] * L[1] * L[2] * L[3];
  if (V >= (1L << 30)) throw Error(1, "lattice too large for 32-bit site indices");
  if (((long)(V + 127) / 128 * 128) * nrhs * 12 >= (1L << 31))
    throw Error(1, "lattice x right-hand sides too large for 32-bit plane offsets");
  G.tbc = tbc;
  geom_layout(G);  // V, Vh, Vb, pad, the in-block order, the divisions
  QWSG_CUDA(cudaGetDevice(&device));
  QWSG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  own_stream = true;
  rb.nblk = 148 * 8;
  QWSG_CUDA(cudaMalloc(&rb.partial, sizeof(double) * 4 * kMaxRhs * rb.nblk));
  QWSG_CUDA(cudaMalloc(&rb.counter, sizeof(unsigned) * 4));
  QWSG_CUDA(cudaMemset(rb.counter, 0, sizeof(unsigned) * 4));
  QWSG_CUDA(cudaMalloc(&d_res, sizeof(double) * 4 * kMaxRhs));
  QWSG_CUDA(cudaMallocHost(&h_res, sizeof(double) * 4 * kMaxRhs));
  QWSG_CUDA(cudaMalloc(&d_coef, sizeof(double) * 4 * kMaxRhs * kCoefSlots));
  QWSG_CUDA(cudaMallocHost(&h_coef, sizeof(double) * 4 * kMaxRhs * kCoefSlots));
}

// Each slot is used once per kCoefSlots calls; the batched solvers read a
// reduction result (a stream synchronisation) between consecutive uses of
// one slot, so a slot is never rewritten while its copy is pending.
const double* Ctx::put_coefs(const double* v) { return put_coefs(v, 4 * G.nr); }

const double* Ctx::put_coefs(const double* v, int n) {
  const int slot = 4 * kMaxRhs;
  if (n < 0 || n > slot) throw Error(1, "coefficient table too large");
  double* h = h_coef + (size_t)coef_next * slot;
  double* d = d_coef + (size_t)coef_next * slot;
  coef_next = (coef_next + 1) % kCoefSlots;
  std::memcpy(h, v, sizeof(double) * n);
  QWSG_CUDA(cudaMemcpyAsync(d, h, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  return d;
}

Ctx::~Ctx() {
  if (st) cudaStreamSynchronize(st);
  for (void* p : owned) cudaFree(p);
  if (stage) cudaFree(stage);
  for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
  clear_graphs();
  if (owns_fields) {
    cudaFree(Ud);
    cudaFree(Cd);
    cudaFree(Us);
    cudaFree(Cs);
    cudaFree(Uh);
    cudaFree(Ch);
  }
  cudaFree(face_list[0]);
  cudaFree(face_list[1]);
  cudaFree(d_coef);
  cudaFreeHost(h_coef);
  if (parent_ev) cudaEventDestroy(parent_ev);
  cudaFree(rb.partial);
  cudaFree(rb.counter);
  cudaFree(d_res);
  cudaFreeHost(h_res);
  if (h_isc) cudaFreeHost(h_isc);
  if (own_stream && st) cudaStreamDestroy(st);
}

template <typename R>
R* Ctx::alloc_spinor() {
  R* p = nullptr;
  QWSG_CUDA(cudaMalloc(&p, sizeof(R) * spinor_elems()));
  QWSG_CUDA(cudaMemsetAsync(p, 0, sizeof(R) * spinor_elems(), st));
  owned.push_back(p);
  return p;
}
template float* Ctx::alloc_spinor<float>();
template double* Ctx::alloc_spinor<double>();

// FP16 spinor: three 16-byte planes + one float plane of per-site scales (IO<H16>)
__half* Ctx::alloc_spinor_h() {
  void* p = nullptr;
  const size_t bytes = (size_t)(6 * 8 + 4) * spad(G);
  QWSG_CUDA(cudaMalloc(&p, bytes));
  QWSG_CUDA(cudaMemsetAsync(p, 0, bytes, st));
  owned.push_back(p);
  return (__half*)p;
}

// Each buffer is allocated on its own when it is missing: an allocation
// that fails (out of device memory) throws with that buffer and the ones
// after it still null, and the next call allocates exactly those, so no
// launch ever sees a buffer of a set that is missing.
template <typename R>
static void alloc_missing(Ctx& c, std::initializer_list<R**> ps) {
  for (R** p : ps)
    if (!*p) *p = c.alloc_spinor<R>();
}

void Ctx::ensure_sap() { alloc_missing<float>(*this, {&sap_s, &sap_a, &sap_t}); }
// (the FP32 SAP buffers are allocated by the FP32 SAP itself: the
// precision form's inner solve does not need them)
void Ctx::ensure_inner() { alloc_missing<float>(*this, {&in_q, &in_r, &in_p, &in_t, &in_r0}); }
void Ctx::ensure_outer() {
  ensure_inner();
  alloc_missing<double>(*this, {&out_q, &out_r, &out_p, &out_t, &out_u, &out_r0});
  alloc_missing<float>(*this, {&ai_b, &ai_t, &ai_x});
}
void Ctx::ensure_hp() {
  ensure_inner();
  ensure_fields_h();
  for (__half** p : {&h_s, &h_a, &h_t, &h_b})
    if (!*p) *p = alloc_spinor_h();
  alloc_missing<float>(*this, {&in_w});
  if (!d_isc) {
    void* q = nullptr;
    QWSG_CUDA(cudaMalloc(&q, sizeof(InnerScalars)));
    owned.push_back(q);
    d_isc = static_cast<InnerScalars*>(q);
  }
  if (!h_isc) QWSG_CUDA(cudaMallocHost(&h_isc, sizeof(InnerScalars)));
}
void Ctx::ensure_fields_d() {
  for (double** p : {&Ud, &Cd})
    if (!*p) {
      QWSG_CUDA(cudaMalloc(p, sizeof(double) * 72 * (size_t)G.pad));
      QWSG_CUDA(cudaMemsetAsync(*p, 0, sizeof(double) * 72 * (size_t)G.pad, st));
    }
}
void Ctx::ensure_fields_s() {
  for (float** p : {&Us, &Cs})
    if (!*p) {
      QWSG_CUDA(cudaMalloc(p, sizeof(float) * 72 * (size_t)G.pad));
      QWSG_CUDA(cudaMemsetAsync(*p, 0, sizeof(float) * 72 * (size_t)G.pad, st));
    }
  fields_h_valid = false;  // the FP16 copies follow the FP32 fields
  links12_valid = false;   // so does the 12-real link copy
}

// The FP32 links are checked once per load: if every link is SU(3) to 1e-5
// (|U U^+ - 1| and |det U - 1|), the Dirac kernels read the 12-real copy and
// rebuild the third row (a third fewer link bytes).  Fields that are not
// SU(3), e.g. the reference's own test fields, keep the 18-real links.
void Ctx::ensure_links12() {
  if (parent) {
    parent->ensure_links12();
    Us12 = parent->Us12;
    if (links12_on != parent->links12_on) {
      QWSG_CUDA(cudaStreamSynchronize(st));
      clear_graphs();
    }
    links12_on = parent->links12_on;
    links12_valid = true;
    return;
  }
  if (links12_valid || !Us) return;
  bool on = false;
  if (link_compress) {
    unsigned* dev = rb.counter + 2;
    QWSG_CUDA(cudaMemsetAsync(dev, 0, sizeof(unsigned), st));
    links_su3_deviation(G, Us, dev, st);
    check_launch("links_su3_deviation");
    unsigned h = 0;
    QWSG_CUDA(cudaMemcpyAsync(&h, dev, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    QWSG_CUDA(cudaStreamSynchronize(st));
    float worst;
    std::memcpy(&worst, &h, sizeof(float));
    on = worst < 1e-5f;
    if (on) {
      if (!Us12) {
        QWSG_CUDA(cudaMalloc(&Us12, sizeof(float) * 48 * (size_t)G.pad));
        owned.push_back(Us12);
      }
      links_compress12(G, Us12, Us, st);
      check_launch("links_compress12");
    }
  }
  if (on != links12_on) {  // captured launches carry the link form
    QWSG_CUDA(cudaStreamSynchronize(st));
    clear_graphs();
  }
  links12_on = on;
  links12_valid = true;
}
// FP16 copies of the FP32 gauge and clover planes (made on first use after
// every load)
void Ctx::sync_from_parent(bool half) {
  if (!parent) return;
  if (!parent->Ud || !parent->Us) throw Error(4, "gauge/clover fields not loaded");
  if (half) parent->ensure_fields_h();
  Ud = parent->Ud;
  Cd = parent->Cd;
  Us = parent->Us;
  Cs = parent->Cs;
  Uh = parent->Uh;
  Ch = parent->Ch;
  fields_h_valid = parent->fields_h_valid;
  links12_valid = false;  // taken from the parent at the next FP32 launch
  kappa = parent->kappa;
  // the parent's field uploads and conversions are on its stream
  if (parent->st != st) {
    if (!parent_ev) QWSG_CUDA(cudaEventCreateWithFlags(&parent_ev, cudaEventDisableTiming));
    QWSG_CUDA(cudaEventRecord(parent_ev, parent->st));
    QWSG_CUDA(cudaStreamWaitEvent(st, parent_ev, 0));
  }
}

void Ctx::ensure_fields_h() {
  if (parent) {
    sync_from_parent(true);
    return;
  }
  if (!Us) throw Error(4, "gauge/clover fields not loaded");
  for (__half** p : {&Uh, &Ch})
    if (!*p) {
      QWSG_CUDA(cudaMalloc(p, sizeof(__half) * 72 * (size_t)G.pad));
      fields_h_valid = false;
    }
  if (!fields_h_valid) {
    fields_s2h(G, Uh, Us, Ch, Cs, st);
    check_launch("fields_s2h");
    fields_h_valid = true;
  }
}

const InnerScalars* Ctx::fetch_inner() {
  if (gm) {
    group_park(*gm, d_isc, h_isc, sizeof(InnerScalars));
    return h_isc;
  }
  QWSG_CUDA(cudaMemcpyAsync(h_isc, d_isc, sizeof(InnerScalars), cudaMemcpyDeviceToHost, st));
  QWSG_CUDA(cudaStreamSynchronize(st));
  return h_isc;
}

const double* Ctx::fetch(int n) {
  if (gm) {
    group_park(*gm, d_res, h_res, sizeof(double) * n);
    return h_res;
  }
  QWSG_CUDA(cudaMemcpyAsync(h_res, d_res, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  QWSG_CUDA(cudaStreamSynchronize(st));
  return h_res;
}

void Ctx::check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw Error(3, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// operators
// ---------------------------------------------------------------------------
void dslash_full_d(Ctx& c, double* out, const double* in) {
  Region region_("ddd_d");
  auto a = hop_args_c<double>(c);
  a.src = in;
  a.out = out;
  a.coef = -c.kappa;
  a.site0 = 0;
  a.nsites = c.G.V;
  run_hop<double>(c, HOP_ALL, EPI_D, a);
  c.n_dslash_d++;
  c.check_launch("dslash_full_d");
}

void dslash_full_s(Ctx& c, float* out, const float* in) {
  Region region_("ddd_s");
  auto a = hop_args_c<float>(c);
  a.src = in;
  a.out = out;
  a.coef = -(float)c.kappa;
  a.site0 = 0;
  a.nsites = c.G.V;
  run_hop<float>(c, HOP_ALL, EPI_D, a);
  c.check_launch("dslash_full_s");
}

template <typename R>
void dslash_inner(Ctx& c, R* out, const R* in, int col, int dom) {
  auto a = hop_args_c<R>(c);
  a.src = in;
  a.out = out;
  a.coef = (R)(-c.kappa);
  site_range(c, col, a.site0, a.nsites);
  a.dom = dom;
  run_hop<R>(c, HOP_INNER, EPI_D, a);
  c.check_launch("dslash_inner");
}
template void dslash_inner<float>(Ctx&, float*, const float*, int, int);
template void dslash_inner<double>(Ctx&, double*, const double*, int, int);

// out += factor A^-1 H_face in on the face sites of one colour (or one domain
// of the reference partition NB = (2,1,1,1), where a domain is a colour)
template <typename T>
static void outer_t(Ctx& c, typename Store<T>::type* out, const typename Store<T>::type* in,
                    int col, int dom, double factor, int zero_col) {
  auto a = hop_args_c<T>(c);
  a.src = in;
  a.out = out;
  a.coef = (typename Arith<T>::R)factor;
  site_range(c, col, a.site0, a.nsites);
  a.dom = dom;
  a.zero_col = zero_col;
  const bool ref_partition = c.G.NB[0] == 2 && c.G.NB[1] == 1 && c.G.NB[2] == 1 && c.G.NB[3] == 1;
  const int lc = col >= 0 ? col : (dom >= 0 && ref_partition ? dom : -1);
  if (lc >= 0) {
    c.ensure_face_lists();
    a.list = c.face_list[lc];
    a.nsites = c.n_face[lc];
    a.dom = -1;
  }
  run_hop<T>(c, HOP_OUTER, EPI_ADD, a);
  c.check_launch("dslash_outer");
}

template <typename R>
void dslash_outer(Ctx& c, R* out, const R* in, int col, int dom, double factor, int zero_col) {
  outer_t<R>(c, out, in, col, dom, factor, zero_col);
}
template void dslash_outer<float>(Ctx&, float*, const float*, int, int, double, int);
template void dslash_outer<double>(Ctx&, double*, const double*, int, int, double, int);

// face-site lists, built once on the host from the block geometry
void Ctx::ensure_face_lists() {
  if (face_list[0] && face_list[1]) return;
  std::vector<int> lst[2];
  for (int g = 0; g < G.V; g++)
    if (on_block_face(G, g)) lst[g >= G.Vh].push_back(g);
  for (int c2 = 0; c2 < 2; c2++) {
    if (face_list[c2]) continue;  // made by an earlier call that failed on the other
    int* d = nullptr;
    QWSG_CUDA(cudaMalloc(&d, sizeof(int) * (lst[c2].size() + 1)));
    cudaError_t e = cudaMemcpy(d, lst[c2].data(), sizeof(int) * lst[c2].size(),
                               cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(d);
      QWSG_CUDA(e);
    }
    n_face[c2] = (int)lst[c2].size();
    face_list[c2] = d;
  }
}

// jinv_ddd_in_s_: nm Richardson steps x <- b + kappa A^-1 H_blk x from x = b
// (static_solver.cc:65-140; at least one step, as the reference's first
// step is unconditional).  Ping-pongs between x and tmp so the last step
// lands in x.
template <typename T>
static void jinv_t(Ctx& c, typename Store<T>::type* x, const typename Store<T>::type* b, int col,
                   int nm, typename Store<T>::type* tmp) {
  Region region_("jinv_ddd_in_s");
  const int steps = nm < 1 ? 1 : nm;
  auto a = hop_args_c<T>(c);
  a.aux = b;
  a.coef = (typename Arith<T>::R)c.kappa;
  site_range(c, col, a.site0, a.nsites);
  const typename Store<T>::type* src = b;
  for (int k = 1; k <= steps; k++) {
    typename Store<T>::type* dst = ((steps - k) % 2 == 0) ? x : tmp;
    a.src = src;
    a.out = dst;
    run_hop<T>(c, HOP_INNER, EPI_JINV, a);
    src = dst;
  }
  c.n_jinv++;
  c.check_launch("jinv");
}

void jinv_s(Ctx& c, float* x, const float* b, int col, int nm) {
  c.ensure_sap();
  jinv_t<float>(c, x, b, col, nm, c.sap_t);
}

// The alternating SAP sweeps of prec_ddd_s_/prec_s_ (qws.cc:802-841) and of
// the half-precision assign_mult_mSAP_s_h_ (prec_ddd_s_h.h:133-170).
// With a_c the block solution of colour c and s the running right-hand side:
//   a_e = J_e(s_e);  s_e += in_e - D_blk,e a_e;  s_o += kappa A^-1 H_face a
// for (e,o) = (E,O) then (O,E).  The reference's first sweep reads the odd
// colour's block solution as zero (qws.cc:806-808); zero_col expresses that.
template <typename T>
static void sap_sweeps_t(Ctx& c, typename Store<T>::type* s, typename Store<T>::type* a,
                         typename Store<T>::type* tmp, const typename Store<T>::type* in,
                         int nsweep, int nm) {
  const double k = c.kappa;
  for (int isap = 0; isap < nsweep; isap++) {
    for (int e = 0; e < 2; e++) {
      const int o = 1 - e;
      jinv_t<T>(c, a, s, e, nm, tmp);
      auto h = hop_args_c<T>(c);
      h.src = a;
      h.aux = in;
      h.out = s;
      h.coef = (typename Arith<T>::R)(-k);
      site_range(c, e, h.site0, h.nsites);
      run_hop<T>(c, HOP_INNER, EPI_SAPE, h);
      outer_t<T>(c, s, a, o, -1, k, (isap == 0 && e == 0) ? 1 : -1);
    }
  }
}

// the final stage of prec_s_ / assign_mult_mSAP_s_h_ (qws.cc:966-973,
// prec_ddd_s_h.h:173-186): out_E = J_E(s_E), s_O += kappa A^-1 H_face (out_E, 0),
// out_O = J_O(s_O)
template <typename T>
static void sap_final_t(Ctx& c, typename Store<T>::type* out, typename Store<T>::type* s,
                        typename Store<T>::type* tmp, int nm) {
  jinv_t<T>(c, out, s, 0, nm, tmp);
  outer_t<T>(c, s, out, 1, -1, c.kappa, 1);
  jinv_t<T>(c, out, s, 1, nm, tmp);
}

void Ctx::clear_graphs() {
  for (auto& e : graphs) cudaGraphExecDestroy(e.exec);
  graphs.clear();
}

// Run `body` (launches only) through a cached CUDA graph.  Everything the
// body allocates or builds must exist before the first capture.
template <typename F>
static void graphed(Ctx& c, Ctx::GraphKey k, F&& body) {
  k.gen = c.graph_gen;
  // the link form is settled before a capture (its check reads back a result)
  // and a change of form drops the graphs captured with the other one
  c.ensure_links12();
  // (a group solve records the launches one by one to merge them)
  if (c.timing || !c.use_graphs || c.st == nullptr || c.st == cudaStreamLegacy ||
      c.st == cudaStreamPerThread || g_group_rec) {
    body();
    return;
  }
  // inside a capture that is already running (a solver step that contains
  // this sequence): the launches become part of that graph
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  QWSG_CUDA(cudaStreamIsCapturing(c.st, &cs));
  if (cs == cudaStreamCaptureStatusActive) {
    body();
    return;
  }
  for (auto& e : c.graphs)
    if (e.key == k) {
      QWSG_CUDA(cudaGraphLaunch(e.exec, c.st));
      c.n_jinv += e.d_jinv;
      c.n_prec_ddd += e.d_prec_ddd;
      c.n_prec_s += e.d_prec_s;
      c.n_prec_s_h += e.d_prec_s_h;
      g_kernel_launches.fetch_add(e.d_launches, std::memory_order_relaxed);
      c.n_graph_launches++;
      return;
    }
  const long j0 = c.n_jinv, p0 = c.n_prec_ddd, s0 = c.n_prec_s, h0 = c.n_prec_s_h;
  const long l0 = g_kernel_launches.load();
  QWSG_CUDA(cudaStreamBeginCapture(c.st, cudaStreamCaptureModeThreadLocal));
  try {
    body();
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(c.st, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  cudaGraph_t g = nullptr;
  QWSG_CUDA(cudaStreamEndCapture(c.st, &g));
  // the same step with other scalar arguments (kappa, tolerance) or other
  // fields (graph_gen): the launch sequence is the same, so update the
  // instantiated graph in place -- far cheaper than instantiating one (a
  // service sees a new kappa in nearly every request); launches already
  // enqueued keep their arguments
  for (size_t i = 0; i < c.graphs.size(); i++) {
    auto& en = c.graphs[i];
    if (en.key.op == k.op && en.key.a == k.a && en.key.b == k.b && en.key.nsap == k.nsap &&
        en.key.nm == k.nm) {
      cudaGraphExecUpdateResultInfo info{};
      if (cudaGraphExecUpdate(en.exec, g, &info) == cudaSuccess) {
        cudaGraphDestroy(g);
        en.key = k;
        QWSG_CUDA(cudaGraphLaunch(en.exec, c.st));
        c.n_graph_launches++;
        return;
      }
      // not updatable: drop that graph (after its pending launches) and
      // instantiate a new one below
      (void)cudaGetLastError();
      QWSG_CUDA(cudaStreamSynchronize(c.st));
      cudaGraphExecDestroy(en.exec);
      c.graphs.erase(c.graphs.begin() + i);
      break;
    }
  }
  cudaGraphExec_t exec = nullptr;
  cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  QWSG_CUDA(e);
  if (c.graphs.size() >= 16) {  // a bounded cache: drop the oldest
    // (after the stream has finished any launch of it)
    QWSG_CUDA(cudaStreamSynchronize(c.st));
    cudaGraphExecDestroy(c.graphs.front().exec);
    c.graphs.erase(c.graphs.begin());
  }
  c.graphs.push_back({k, exec, c.n_jinv - j0, c.n_prec_ddd - p0, c.n_prec_s - s0,
                      c.n_prec_s_h - h0, g_kernel_launches.load() - l0});
  QWSG_CUDA(cudaGraphLaunch(exec, c.st));
  c.n_graph_launches++;
}

// prec_ddd_s_ (qws.cc:776-926): out = D M_SAP in.  Both of the reference's
// final-stage branches compute a_E = J_E(s_E), a_O = J_O(s_O - D_face,O (a_E, 0)),
// out = D (a_E, a_O); here the last product is one full-lattice D.
void prec_ddd_s(Ctx& c, float* out, const float* in, int nsap, int nm) {
  Region region_("prec_ddd_s");
  if (nsap > 10 || nm > 10) throw Error(2, "prec_ddd_s_: nsap and nm must be <= 10 (qws.cc:798-799)");
  c.ensure_sap();
  c.ensure_face_lists();
  float *s = c.sap_s, *a = c.sap_a;
  graphed(c, {0, out, in, nsap, nm, c.kappa}, [&] {
    blas_copy<float>(c.G, s, in, 0, c.G.V, c.st);
    sap_sweeps_t<float>(c, s, a, c.sap_t, in, nsap, nm);
    sap_final_t<float>(c, a, s, c.sap_t, nm);
    dslash_full_s(c, out, a);
    c.n_prec_ddd++;
  });
}

// prec_s_ (qws.cc:929-975): out = M_SAP in.
void prec_s(Ctx& c, float* out, const float* in, int nsap, int nm) {
  Region region_("prec_s");
  c.ensure_sap();
  c.ensure_face_lists();
  float *s = c.sap_s, *a = c.sap_a;
  graphed(c, {1, out, in, nsap, nm, c.kappa}, [&] {
    blas_copy<float>(c.G, s, in, 0, c.G.V, c.st);
    sap_sweeps_t<float>(c, s, a, c.sap_t, in, nsap, nm);
    sap_final_t<float>(c, out, s, c.sap_t, nm);
    c.n_prec_s++;
  });
}

// assign_mult_mSAP_s_h_ (prec_ddd_s_h.h:63-231) with FP16 storage: the input
// is stored with per-site scales instead of the reference's one global
// scale (assign_q_s2h, qws_h.cc:175-207), arithmetic is FP32, and the sweep
// count is the reference's half-precision one (isap = 1 .. nsap-1).
// the launches alone (buffers, face lists and fields already in place), for
// callers that capture them inside a larger step
static void prec_s_h_seq(Ctx& c, float* out, const float* in, int nsap, int nm) {
  Region region_("assign_mult_mSAP_s_h");
  graphed(c, {2, out, in, nsap, nm, c.kappa}, [&] {
    spinor_s2h(c.G, c.h_b, in, c.st);
    spinor_h2h(c.G, c.h_s, c.h_b, c.st);
    sap_sweeps_t<H16>(c, c.h_s, c.h_a, c.h_t, c.h_b, nsap - 1, nm);
    sap_final_t<H16>(c, c.h_a, c.h_s, c.h_t, nm);
    spinor_h2s(c.G, out, c.h_a, c.st);
    c.n_prec_s_h++;
  });
}

void prec_s_h(Ctx& c, float* out, const float* in, int nsap, int nm) {
  if (nsap > 10 || nm > 10)
    throw Error(2, "assign_mult_mSAP_s_h_: nsap and nm must be <= 10 (prec_ddd_s_h.h:100-101)");
  c.ensure_hp();
  c.ensure_face_lists();
  prec_s_h_seq(c, out, in, nsap, nm);
  c.check_launch("prec_s_h");
}

// One kernel of the SAP on its own (ctx.h).  The reference's counterparts:
// ddd_in_s_/ddd_in_h_ (ddd_in_s.cc:376, ddd_in_h.h:54), jinv_ddd_in_s_/_h_
// (static_solver.cc:141, jinv_ddd_in_h.h:53-118), ddd_out_pre+pos_s_/_h_
// (ddd_out_s.cc:639,661, ddd_out_h.h:57,283) and the update loop of a SAP
// half-sweep (qws.cc:815-818, prec_ddd_s_h.h:143-150).  The FP16 forms use
// the SAP's own FP16 work planes, which no other call holds between calls.
template <typename T>
static void sap_kernel_t(Ctx& c, typename Store<T>::type* out, const typename Store<T>::type* in,
                         const typename Store<T>::type* aux, int op, int col, int nm,
                         double factor, typename Store<T>::type* tmp) {
  using R = typename Arith<T>::R;
  if (op == 1) {
    jinv_t<T>(c, out, in, col, nm, tmp);
    return;
  }
  if (op == 2) {
    outer_t<T>(c, out, in, col, -1, factor, -1);
    return;
  }
  auto a = hop_args_c<T>(c);
  a.src = in;
  a.aux = aux;
  a.out = out;
  a.coef = (R)(-c.kappa);
  site_range(c, col, a.site0, a.nsites);
  run_hop<T>(c, HOP_INNER, op == 0 ? EPI_D : EPI_SAPE, a);
}

void sap_kernel(Ctx& c, float* out, const float* in, const float* aux, int op, int col, int nm,
                double factor, bool half) {
  if (op < 0 || op > 3) throw Error(1, "sap_kernel: op must be 0..3");
  if (col != 0 && col != 1) throw Error(1, "colour must be 0 or 1");
  if (op == 3 && !aux) throw Error(1, "sap_kernel: the SAP update needs its right-hand side");
  c.ensure_face_lists();
  if (!half) {
    c.ensure_sap();
    sap_kernel_t<float>(c, out, in, aux, op, col, nm, factor, c.sap_t);
  } else {
    c.ensure_hp();
    spinor_s2h(c.G, c.h_b, in, c.st);
    spinor_s2h(c.G, c.h_s, out, c.st);
    if (aux) spinor_s2h(c.G, c.h_a, aux, c.st);
    sap_kernel_t<H16>(c, c.h_s, c.h_b, aux ? c.h_a : nullptr, op, col, nm, factor, c.h_t);
    spinor_h2s(c.G, out, c.h_s, c.st);
  }
  c.check_launch("sap_kernel");
}

// bicgstab_precdd_s_ (bicgstab_precdd_s.cc:85-559).  Returns the number of
// iterations run (a half iteration that converged counts as one).
int bicgstab_precdd_s(Ctx& c, float* x, const float* b, double tol, int maxiter, int nsap, int nm,
                      double* final_rel) {
  Region region_("bicgstab_precdd_s");
  c.ensure_inner();
  const Geom& G = c.G;
  float *q = c.in_q, *r = c.in_r, *p = c.in_p, *t = c.in_t, *r0 = c.in_r0;
  blas_zero<float>(G, x, 0, G.V, c.st);
  blas_bicg_init<float>(G, b, nullptr, r, p, r0, c.d_res, c.rb, c.st);
  const double* h = c.fetch(2);
  const float bnorm = (float)h[0];
  if (bnorm == 0) {  // b = 0: x = 0 (zeroed above)
    if (final_rel) *final_rel = 0;
    return 0;
  }
  std::complex<float> rho0(bnorm, 0), rho, beta, omega, alpha, ctmp;
  float rnorm = bnorm;
  int done = maxiter;
  for (int iter = 0; iter < maxiter; iter++) {
    c.n_inner_iter++;
    prec_ddd_s(c, q, p, nsap, nm);
    blas_cdot<float>(G, r0, q, c.d_res, c.rb, c.st);
    h = c.fetch(2);
    ctmp = std::complex<float>((float)h[0], (float)h[1]);
    alpha = rho0 / ctmp;
    if (std::abs(ctmp) == 0) alpha = 0;
    blas_bicg_update<float>(G, x, r, p, q, alpha.real(), alpha.imag(), nullptr, c.d_res, c.rb,
                            c.st);
    rnorm = (float)c.fetch(1)[0];
    if (!std::isfinite(rnorm)) throw Error(3, "solver: non-finite residual norm");
    if (std::sqrt(rnorm / bnorm) < tol) {
      done = iter + 1;
      break;
    }
    prec_ddd_s(c, t, r, nsap, nm);
    blas_norm_cdot<float>(G, t, r, c.d_res, c.rb, c.st);
    h = c.fetch(3);
    const float redu0 = (float)h[0], redu1 = (float)h[1], redu2 = (float)h[2];
    omega = std::complex<float>(redu1 / redu0, redu2 / redu0);
    if (redu0 == 0) omega = 0;
    blas_bicg_update<float>(G, x, r, r, t, omega.real(), omega.imag(), r0, c.d_res, c.rb, c.st);
    h = c.fetch(3);
    rnorm = (float)h[0];
    if (!std::isfinite(rnorm)) throw Error(3, "solver: non-finite residual norm");
    rho = std::complex<float>((float)h[1], (float)h[2]);
    if (std::sqrt(rnorm / bnorm) < tol) {
      done = iter + 1;
      break;
    }
    beta = alpha * rho / (rho0 * omega);
    rho0 = rho;
    if (std::abs(omega) == 0 || std::abs(rho0) == 0) beta = 0;
    blas_bicg_p<float>(G, p, r, q, beta.real(), beta.imag(), omega.real(), omega.imag(), c.st);
  }
  if (final_rel) *final_rel = std::sqrt((double)rnorm / (double)bnorm);
  c.check_launch("bicgstab_precdd_s");
  return done;
}

// bicgstab_precdd_s_h_ (bicgstab_precdd_s_h.cc:83-369): flexible BiCGStab,
// w = M p, q = D w, x += alpha w (and likewise for the omega step), with the
// FP16-storage SAP as M and the FP32 D (assign_mult_wd_s_, prec_ddd_s_h.h:233).
// The scalars live on the device (InnerScalars, inner_scalars): each half
// iteration -- SAP, D, the reduction, the scalar update, the vector update
// and its norms -- is one CUDA graph replay, after which the host reads
// back one small record (convergence, a non-finite residual) instead of
// every reduction.  The arithmetic and its order are the host loop's.
int bicgstab_precdd_s_h(Ctx& c, float* x, const float* b, double tol, int maxiter, int nsap,
                        int nm, double* final_rel) {
  Region region_("bicgstab_precdd_s_h");
  if (nsap > 10 || nm > 10)
    throw Error(2, "assign_mult_mSAP_s_h_: nsap and nm must be <= 10 (prec_ddd_s_h.h:100-101)");
  c.ensure_hp();
  c.ensure_face_lists();  // built before any capture
  c.ensure_links12();
  const Geom& G = c.G;
  float *q = c.in_q, *r = c.in_r, *p = c.in_p, *t = c.in_t, *r0 = c.in_r0, *w = c.in_w;
  InnerScalars* S = c.d_isc;
  blas_zero<float>(G, x, 0, G.V, c.st);
  blas_bicg_init<float>(G, b, nullptr, r, p, r0, c.d_res, c.rb, c.st);
  inner_scalars(S, c.d_res, 0, tol, c.st);
  const InnerScalars* h = c.fetch_inner();
  if (h->done) {  // b = 0: x = 0 (zeroed above)
    if (final_rel) *final_rel = 0;
    return 0;
  }
  for (int iter = 0; iter < maxiter; iter++) {
    c.n_inner_iter++;
    graphed(c, {5, x, r0, nsap, nm, c.kappa, tol}, [&] {
      prec_s_h_seq(c, w, p, nsap, nm);
      dslash_full_s(c, q, w);
      blas_cdot<float>(G, r0, q, c.d_res, c.rb, c.st);
      inner_scalars(S, c.d_res, 1, tol, c.st);
      blas_bicg_update<float>(G, x, r, w, q, 0, 0, nullptr, c.d_res, c.rb, c.st,
                              inner_coefs(S, 0));
      inner_scalars(S, c.d_res, 2, tol, c.st);
    });
    h = c.fetch_inner();
    if (h->bad) throw Error(3, "solver: non-finite residual norm");
    if (h->done) break;
    graphed(c, {6, x, r0, nsap, nm, c.kappa, tol}, [&] {
      prec_s_h_seq(c, w, r, nsap, nm);
      dslash_full_s(c, t, w);
      blas_norm_cdot<float>(G, t, r, c.d_res, c.rb, c.st);
      inner_scalars(S, c.d_res, 3, tol, c.st);
      blas_bicg_update<float>(G, x, r, w, t, 0, 0, r0, c.d_res, c.rb, c.st, inner_coefs(S, 4));
      inner_scalars(S, c.d_res, 4, tol, c.st);
      blas_bicg_p<float>(G, p, r, q, 0, 0, 0, 0, c.st, inner_coefs(S, 8));
    });
    h = c.fetch_inner();
    if (h->bad) throw Error(3, "solver: non-finite residual norm");
    if (h->done) break;
  }
  if (final_rel) *final_rel = std::sqrt((double)h->rnorm / (double)h->bnorm);
  c.check_launch("bicgstab_precdd_s_h");
  return h->done ? h->iters : maxiter;
}

// approx_inv_dirac_op (bicgstab_dd_mix.cc:76-102) with the renormalising
// FP64<->FP32 converters (reordering.cc:108-204); the half-precision variant
// (approx_inv_dirac_op_hf, bicgstab_dd_mix2_hf.cc:88-107) has no trailing
// prec_s_ because its inner solve is flexible.
static int approx_inv(Ctx& c, double* x, const double* b, double tol_s, int maxiter_s, int nsap,
                      int nm, bool hf) {
  Region region_("approx_inv_dirac_op");
  blas_norm2<double>(c.G, b, c.d_res, c.rb, c.st);
  const double bn = std::sqrt(c.fetch(1)[0]);
  blas_d2s(c.G, c.ai_b, b, 1.0 / bn, c.st);
  int it;
  if (hf) {
    it = bicgstab_precdd_s_h(c, c.ai_x, c.ai_b, tol_s, maxiter_s, nsap, nm, nullptr);
  } else {
    it = bicgstab_precdd_s(c, c.ai_t, c.ai_b, tol_s, maxiter_s, nsap, nm, nullptr);
    prec_s(c, c.ai_x, c.ai_t, nsap, nm);
  }
  blas_s2d(c.G, x, c.ai_x, bn, c.st);
  return it;
}

// The flexible FP64 BiCGStab of bicgstab_dd_mix_ (bicgstab_dd_mix.cc:105-388)
// and bicgstab_dd_mix2_hf_ (bicgstab_dd_mix2_hf.cc:110-373): two
// preconditioned inner solves + two D per iteration.  iter runs
// [iter_begin, iter_end); returns the reference's conviter.
static int outer_loop(Ctx& c, double* x, const double* b, double tol, int iter_begin, int iter_end,
                      double tol_s, int maxiter_s, int nsap, int nm, bool hf, long* inner_out,
                      double* rel_out, double* hist, int hist_len) {
  const Geom& G = c.G;
  double *q = c.out_q, *r = c.out_r, *p = c.out_p, *t = c.out_t, *u = c.out_u, *r0 = c.out_r0;
  dslash_full_d(c, q, x);
  blas_bicg_init<double>(G, b, q, r, p, r0, c.d_res, c.rb, c.st);
  const double* h = c.fetch(2);
  const double bnorm = h[0];
  if (bnorm == 0) {  // b = 0: x = 0 (the reference would divide 0 by 0)
    blas_zero<double>(G, x, 0, G.V, c.st);
    *rel_out = 0;
    return iter_begin;
  }
  std::complex<double> rho0(h[1], 0), rho, beta, omega, alpha, ctmp;
  double rnorm = h[1];
  long inner = 0;
  int iter, nh = 0, conv = iter_end;
  for (iter = iter_begin; iter < iter_end; iter++) {
    inner += approx_inv(c, u, p, tol_s, maxiter_s, nsap, nm, hf);
    dslash_full_d(c, q, u);
    blas_cdot<double>(G, r0, q, c.d_res, c.rb, c.st);
    h = c.fetch(2);
    ctmp = std::complex<double>(h[0], h[1]);
    if (iter == c.breakdown_at && iter > 0) ctmp = 0;  // injected on the host (tests)
    alpha = rho0 / ctmp;
    if (std::abs(ctmp) == 0) alpha = 0;
    blas_bicg_update<double>(G, x, r, u, q, alpha.real(), alpha.imag(), nullptr, c.d_res, c.rb,
                             c.st);
    rnorm = c.fetch(1)[0];
    if (!std::isfinite(rnorm)) throw Error(3, "solver: non-finite residual norm");
    if (hist && nh < hist_len) hist[nh++] = std::sqrt(rnorm / bnorm);
    if (std::sqrt(rnorm / bnorm) < tol) {
      conv = iter;
      break;
    }
    inner += approx_inv(c, u, r, tol_s, maxiter_s, nsap, nm, hf);
    dslash_full_d(c, t, u);
    blas_norm_cdot<double>(G, t, r, c.d_res, c.rb, c.st);
    h = c.fetch(3);
    omega = std::complex<double>(h[1] / h[0], h[2] / h[0]);
    if (h[0] == 0) omega = 0;
    blas_bicg_update<double>(G, x, r, u, t, omega.real(), omega.imag(), r0, c.d_res, c.rb, c.st);
    h = c.fetch(3);
    rnorm = h[0];
    if (!std::isfinite(rnorm)) throw Error(3, "solver: non-finite residual norm");
    rho = std::complex<double>(h[1], h[2]);
    if (hist && nh < hist_len) hist[nh++] = std::sqrt(rnorm / bnorm);
    if (std::sqrt(rnorm / bnorm) < tol) {
      conv = iter;
      break;
    }
    beta = alpha * rho / (rho0 * omega);
    rho0 = rho;
    if (std::abs(omega) == 0 || std::abs(rho0) == 0) beta = 0;
    blas_bicg_p<double>(G, p, r, q, beta.real(), beta.imag(), omega.real(), omega.imag(), c.st);
  }
  *inner_out += inner;
  *rel_out = std::sqrt(rnorm / bnorm);
  return conv;
}

void bicgstab_dd_mix(Ctx& c, double* x, const double* b, double tol, int maxiter, double tol_s,
                     int maxiter_s, int nsap, int nm, SolveStats* stats, double* hist,
                     int hist_len) {
  Region region_("bicgstab_dd_mix");
  c.ensure_outer();
  long inner = 0;
  double rel = 0;
  int conv = outer_loop(c, x, b, tol, 1, maxiter, tol_s, maxiter_s, nsap, nm, false, &inner, &rel,
                        hist, hist_len);
  if (stats) {
    stats->outer_iters = conv;
    stats->inner_iters = inner;
    stats->rel_resid_recursive = rel;
  }
  c.check_launch("bicgstab_dd_mix");
}

// |b - D x| / |b| in FP64 (the true residual main.cc:286-311 prints).
double true_residual(Ctx& c, const double* x, const double* b) {
  c.ensure_outer();
  dslash_full_d(c, c.out_t, x);
  blas_bicg_init<double>(c.G, b, c.out_t, c.out_q, c.out_p, c.out_r0, c.d_res, c.rb, c.st);
  const double* h = c.fetch(2);
  if (h[0] == 0) return h[1] == 0 ? 0.0 : INFINITY;  // b = 0: exact only for D x = 0
  return std::sqrt(h[1] / h[0]);
}

// bicgstab_dd_mix2_hf_: iter = 0 .. maxiter-1, conviter = the 0-based
// iteration of convergence.  With reliable > 0, the loop is restarted from
// the recomputed FP64 true residual (at most `reliable` times) until
// |b - D x| / |b| < tol: the recursive residual of the flexible outer loop can
// drift from the true one when the inner solve is low precision.
void bicgstab_dd_mix2_hf(Ctx& c, double* x, const double* b, double tol, int maxiter,
                         double tol_s, int maxiter_s, int nsap, int nm, int reliable,
                         SolveStats* stats) {
  Region region_("bicgstab_dd_mix2_hf");
  c.ensure_outer();
  c.ensure_hp();
  long inner = 0;
  double rel = 0, truerel = -1;
  int conv = 0, total = 0;
  for (int pass = 0; pass <= reliable; pass++) {
    conv = outer_loop(c, x, b, tol, 0, maxiter, tol_s, maxiter_s, nsap, nm, true, &inner, &rel,
                      nullptr, 0);
    total += (conv < maxiter ? conv + 1 : maxiter);
    if (reliable <= 0) break;
    truerel = true_residual(c, x, b);
    if (truerel < tol) break;
  }
  if (stats) {
    stats->outer_iters = reliable > 0 ? total : conv;
    stats->inner_iters = inner;
    stats->rel_resid_recursive = rel;
    stats->rel_resid_true = truerel;
  }
  c.check_launch("bicgstab_dd_mix2_hf");
}

}  // namespace qwsg
