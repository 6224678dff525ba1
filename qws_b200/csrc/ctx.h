// Solver context: geometry, resident fields and work buffers on one GPU.
#pragma once
#include <cuda_runtime.h>

#include <complex>
#include <stdexcept>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "kernels.h"

namespace qwsg {

// A named range for profilers (NVTX: ncu --nvtx, Nsight Systems), named
// after the reference's routine and timing region it stands for; it costs
// nothing measurable when no tool is attached.
struct Region {
  explicit Region(const char* name) { nvtxRangePushA(name); }
  ~Region() { nvtxRangePop(); }
  Region(const Region&) = delete;
  Region& operator=(const Region&) = delete;
};

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define QWSG_CUDA(call)                                                                     \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      throw ::qwsg::Error(3, std::string(#call) + ": " + cudaGetErrorString(e_));           \
  } while (0)

struct GroupMember;

struct SolveStats {
  int outer_iters = 0;
  long inner_iters = 0;
  double rel_resid_recursive = 0;  // sqrt(|r|^2/|b|^2) at exit
  double rel_resid_true = -1;      // |b - D x| / |b| (when requested)
};

struct Ctx {
  Geom G{};
  double kappa = 0;
  cudaStream_t st = nullptr;
  bool own_stream = false;
  // a multi-RHS context borrows the gauge/clover planes of its parent
  // lattice (same fields, same geometry) and owns only its spinor buffers
  bool owns_fields = true;
  Ctx* parent = nullptr;
  // refresh the borrowed field pointers and kappa from the parent (the FP16
  // copies too when `half`), before every batched call
  void sync_from_parent(bool half);
  cudaEvent_t parent_ev = nullptr;
  int device = 0;

  // resident fields (device planes)
  double* Ud = nullptr;
  double* Cd = nullptr;
  float* Us = nullptr;
  // FP32 links in 12-real form, used by the FP32 Dirac kernels when the
  // links are SU(3) to FP32 accuracy (link_compress: 1 = automatic, 0 = off)
  float* Us12 = nullptr;
  bool links12_valid = false;  // the check / copy reflects the current Us
  bool links12_on = false;
  int link_compress = 1;
  void ensure_links12();
  float* Cs = nullptr;

  // reductions
  RedBuf rb{};
  double* d_res = nullptr;
  double* h_res = nullptr;  // pinned
  // device-side scalars of the single-RHS flexible inner solve, and their
  // pinned host copy (ensure_hp)
  InnerScalars* d_isc = nullptr;
  InnerScalars* h_isc = nullptr;
  const InnerScalars* fetch_inner();

  // work buffers, allocated on first use
  float* sap_s = nullptr;
  float* sap_a = nullptr;
  float* sap_t = nullptr;
  float* in_q = nullptr;
  float* in_r = nullptr;
  float* in_p = nullptr;
  float* in_t = nullptr;
  float* in_r0 = nullptr;
  float* ai_b = nullptr;
  float* ai_t = nullptr;
  float* ai_x = nullptr;
  double* out_q = nullptr;
  double* out_r = nullptr;
  double* out_p = nullptr;
  double* out_t = nullptr;
  double* out_u = nullptr;
  double* out_r0 = nullptr;
  std::vector<void*> owned;
  void* stage = nullptr;  // host<->device conversion staging
  size_t stage_bytes = 0;
  // sites of each colour that touch a SAP-block face (DD order, ascending)
  int* face_list[2] = {nullptr, nullptr};
  int n_face[2] = {0, 0};
  void ensure_face_lists();

  // per-kernel CUDA-event timing (kind = kernel_kind(), see solver.cu)
  struct KRec {
    int kind;
    cudaEvent_t a, b;
    double bytes;
  };
  bool timing = false;
  std::vector<KRec> recs;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_next = 0;
  cudaEvent_t next_event();

  // counters (calls of each reference-named region)
  long n_prec_ddd = 0, n_prec_s = 0, n_jinv = 0, n_dslash_d = 0, n_inner_iter = 0;

  // nrhs: right-hand sides per spinor field (power of two, 1..32)
  Ctx(const int L[4], const int NB[4], int tbc, int nrhs = 1);
  ~Ctx();

  size_t spinor_elems() const { return (size_t)24 * spad(G); }
  static constexpr int kMaxRhs = 32;
  // per-RHS statistics of the last multi-RHS solve
  std::vector<SolveStats> last_stats;
  std::vector<int> last_iters;
  template <typename R>
  R* alloc_spinor();
  void ensure_sap();
  void ensure_inner();
  void ensure_outer();
  void ensure_fields_d();
  void ensure_fields_s();
  // synchronous read of n reduction results
  // the first n reduction results (res[4*rhs + k]: use 4*nr for all RHS)
  const double* fetch(int n);
  // per-RHS scalar table (4 doubles per RHS) for the batched BLAS updates:
  // copied from host `v` to a device slot; returns the device pointer
  const double* put_coefs(const double* v);
  // the same for n doubles (n <= 4 * kMaxRhs)
  const double* put_coefs(const double* v, int n);
  double* d_coef = nullptr;  // kCoefSlots x 4*kMaxRhs
  double* h_coef = nullptr;  // pinned staging of the same size
  int coef_next = 0;
  static constexpr int kCoefSlots = 64;
  void check_launch(const char* what);

  // FP16-storage SAP (precision form): fields converted from the FP32 ones,
  // work spinors with per-site scales, and the flexible inner solver's w
  __half* Uh = nullptr;
  __half* Ch = nullptr;
  // per-RHS kappa on a multi-RHS handle (set_rhs_kappas): clover planes per
  // (site, RHS) entry in FP64/FP32/FP16 and the kappas; empty: the parent's
  std::vector<double> rhs_kappas;
  // per-RHS stopping tolerance of the FP64 outer solvers (qwsg_batch_set_tols);
  // empty: the tolerance argument of the call for every RHS
  std::vector<double> rhs_tols;
  // fault injection on the host (qwsg_inject_breakdown): the FP64 outer loop
  // takes <r0, q> as zero at this outer iteration (0: never)
  int breakdown_at = 0;
  double* Cdr = nullptr;
  float* Csr = nullptr;
  __half* Chr = nullptr;
  double* kap_d = nullptr;
  float* kap_s = nullptr;
  bool fields_h_valid = false;
  __half* h_s = nullptr;
  __half* h_a = nullptr;
  __half* h_t = nullptr;
  __half* h_b = nullptr;
  float* in_w = nullptr;
  __half* alloc_spinor_h();
  void ensure_fields_h();
  void ensure_hp();
  long n_prec_s_h = 0;

  // even-odd family: the fields the parity operators read (the resident ones
  // unless set; the drop-in supplies the even-odd reading of QWS's host
  // arrays), the parities of mtilde (pce_f/pco_f of qws_init_), work buffers
  const double* eoUd = nullptr;
  const double* eoCd = nullptr;
  const float* eoUs = nullptr;
  const float* eoCs = nullptr;
  int pce = 0, pco = 1;
  double* eo_d[6] = {};
  // multi-shift CG: the shifts' search vectors (ms_n fields back to back)
  double* ms_p = nullptr;
  int ms_n = 0;
  float* eo_s[2] = {};
  void ensure_eo();
  long n_mtilde = 0;

  // CUDA graphs of the SAP preconditioner's launch sequences (about 40
  // launches, no host synchronisation inside), captured on first use per
  // (operator, buffers, nsap, nm, kappa) and replayed afterwards.  Off while
  // kernel timing is on and on the legacy default stream.
  struct GraphKey {
    int op;
    const void* a;
    const void* b;
    int nsap, nm;
    double kappa;
    double tol = 0;  // the stopping tolerance a captured solver step compares with
    long gen = 0;    // graph_gen at capture (set by graphed)
    bool operator==(const GraphKey& o) const {
      return op == o.op && a == o.a && b == o.b && nsap == o.nsap && nm == o.nm &&
             kappa == o.kappa && tol == o.tol && gen == o.gen;
    }
  };
  struct GraphEntry {
    GraphKey key;
    cudaGraphExec_t exec;
    long d_jinv, d_prec_ddd, d_prec_s, d_prec_s_h, d_launches;  // counts one replay stands for
  };
  std::vector<GraphEntry> graphs;
  bool use_graphs = true;
  long n_graph_launches = 0;
  void clear_graphs();
  // bumped when the fields the graphs read change (a multi-RHS handle moved
  // to another parent): the graphs are then captured again and, where the
  // launch sequence is the same, updated in place instead of instantiated
  long graph_gen = 0;

  // set while this lattice takes part in a group solve (group.cu): its
  // read-backs wait for the group's merged launches
  GroupMember* gm = nullptr;
};

// kernel kinds for timing
enum {
  K_D_F64 = 0,      // full D, FP64 (outer residual)
  K_D_F32 = 1,      // full D, FP32
  K_DIN_F64 = 2,    // block-interior D, FP64
  K_DIN_F32 = 3,    // block-interior D, FP32
  K_JINV_F32 = 4,   // Richardson step on D_block
  K_SAPE_F32 = 5,   // SAP update s_e += in_e - D_blk a_e
  K_OUT_F64 = 6,    // face hops, FP64
  K_OUT_F32 = 7,    // face hops, FP32
  K_JINV_F16 = 8,   // the same three in FP16 storage
  K_SAPE_F16 = 9,
  K_OUT_F16 = 10,
  K_DIN_F16 = 11,   // block-interior D, FP16 storage
  K_NKIND = 12
};
const char* kernel_kind_name(int k);
// drain event records into per-kind totals (launches, ms, algorithmic bytes)
void kernel_stats(Ctx& c, long* launches, double* ms, double* bytes);

// operators on device planes -----------------------------------------------
void dslash_full_d(Ctx& c, double* out, const double* in);
void dslash_full_s(Ctx& c, float* out, const float* in);
// D_block on one colour (col >= 0) or one domain (dom >= 0)
template <typename R>
void dslash_inner(Ctx& c, R* out, const R* in, int col, int dom);
// out += factor A^-1 H_face in, on one colour or domain
template <typename R>
void dslash_outer(Ctx& c, R* out, const R* in, int col, int dom, double factor, int zero_col);
void jinv_s(Ctx& c, float* x, const float* b, int col, int nm);
void prec_ddd_s(Ctx& c, float* out, const float* in, int nsap, int nm);
void prec_s(Ctx& c, float* out, const float* in, int nsap, int nm);
// FP16-storage SAP preconditioner with the reference's half-precision sweep
// count (assign_mult_mSAP_s_h_, prec_ddd_s_h.h:63-231: nsap-1 sweeps + the
// final stage); FP32 in and out
void prec_s_h(Ctx& c, float* out, const float* in, int nsap, int nm);
// single applications of the kernels the SAP is built from, for checking
// each on its own: op 0 out_c = D_blk in_c ; op 1 out_c = J_c(in_c) (nm
// Richardson steps) ; op 2 out += factor A^-1 H_face in on colour c's face
// sites ; op 3 out_c += aux_c - D_blk in_c (the SAP update).  half: the
// operands are stored in FP16 with per-site scales first (as the SAP stores
// them) and the result converted back; else the FP32 kernels.
void sap_kernel(Ctx& c, float* out, const float* in, const float* aux, int op, int col, int nm,
                double factor, bool half);
// flexible inner BiCGStab with the FP16 SAP (bicgstab_precdd_s_h.cc:83-369)
int bicgstab_precdd_s_h(Ctx& c, float* x, const float* b, double tol, int maxiter, int nsap,
                        int nm, double* final_rel);
// outer FP64 loop around it (bicgstab_dd_mix2_hf.cc:110-373); reliable > 0
// adds restarts from the recomputed true residual until |b - Dx|/|b| < tol
void bicgstab_dd_mix2_hf(Ctx& c, double* x, const double* b, double tol, int maxiter,
                         double tol_s, int maxiter_s, int nsap, int nm, int reliable,
                         SolveStats* stats);
int bicgstab_precdd_s(Ctx& c, float* x, const float* b, double tol, int maxiter, int nsap, int nm,
                      double* final_rel);
void bicgstab_dd_mix(Ctx& c, double* x, const double* b, double tol, int maxiter, double tol_s,
                     int maxiter_s, int nsap, int nm, SolveStats* stats, double* hist,
                     int hist_len);
double true_residual(Ctx& c, const double* x, const double* b);

// group solve (group.cu): bicgstab_dd_mix2_hf on each item's lattice (one
// RHS, one kappa each; any volumes, block grids and solver parameters), with
// the kernels of all of them merged into common launches on stream st.
// status: 0, or the error code of that lattice's solve (error: its message);
// the other lattices carry on.  Throws only on a failure of the group itself.
struct GroupItem {
  Ctx* c;
  double* x;  // initial guess in, solution out (device planes)
  const double* b;
  double tol;
  int maxiter;
  double tol_s;
  int maxiter_s, nsap, nm, reliable;
  SolveStats stats;
  int status;
  std::string error;
};
struct GroupStats {
  long rounds;           // read-back points of the group (host synchronisations)
  long merged_launches;  // launches issued
  long member_launches;  // launches the lattices' own solves would have issued
  // host seconds: waiting for the members to reach their read-backs, merging,
  // issuing the launches and copies, waiting for the GPU
  double t_members, t_merge, t_launch, t_gpu_wait;
};
void group_bicgstab_dd_mix2_hf(std::vector<GroupItem>& items, cudaStream_t st, GroupStats* gs);
void group_park(GroupMember& me, const void* dev, void* host, size_t bytes);

// multi-RHS forms (solver_mrhs.cu) on a context with G.nr right-hand sides:
// per-RHS scalars and convergence, one launch per operator for all RHS.
// iters / st / rel hold G.nr entries.
int bicgstab_precdd_s_mrhs(Ctx& c, float* x, const float* b, double tol, int maxiter, int nsap,
                           int nm, int* iters);
int bicgstab_precdd_s_h_mrhs(Ctx& c, float* x, const float* b, double tol, int maxiter, int nsap,
                             int nm, int* iters);
void bicgstab_dd_mix_mrhs(Ctx& c, double* x, const double* b, double tol, int maxiter,
                          double tol_s, int maxiter_s, int nsap, int nm, SolveStats* st);
void bicgstab_dd_mix2_hf_mrhs(Ctx& c, double* x, const double* b, double tol, int maxiter,
                              double tol_s, int maxiter_s, int nsap, int nm, int reliable,
                              SolveStats* st);
void true_residual_mrhs(Ctx& c, const double* x, const double* b, double* rel);

// clover term of the resident gauge field on the device (clover_build.cu)
void build_clover(Ctx& c, double csw);
// seeded SU(3) + APE gauge field generated on the device (gauge_gen.cu)
double gen_gauge_device(Ctx& c, unsigned long long seed, int n_smear, double alpha);

void set_error(const std::string& m);

// even-odd family (eo_host.cu); which/dag/clov/mode as in EoArgs (kernels.h)
template <typename R>
void deo(Ctx& c, R* out, const R* in, int pe, int which, int dag, int clov, int mode,
         double factor, const R* in0);
template <typename R>
void clv(Ctx& c, R* out, const R* in, int pe);
void mtilde_d(Ctx& c, double* out, const double* in);      // qws.cc:551-556
void mtilde_dag_d(Ctx& c, double* out, const double* in);  // qws.cc:557-565
void mtilde_s(Ctx& c, float* out, const float* in);        // qws.cc:598-604
int bicgstab_vm(Ctx& c, double* x, const double* b, int maxiter);  // bicgstab.cc:68
void mtdagmt_d(Ctx& c, double* out, const double* in);              // qws.cc:566-571
// per-RHS kappa on a multi-RHS handle (no counterpart in the reference)
void set_rhs_kappas(Ctx& c, const double* kappas, double csw);
int cg_vm(Ctx& c, double* x, const double* b, int maxiter);        // cg.cc:65
// X: n solution fields back to back (spinor_elems() doubles each)
int mcg_vm(Ctx& c, double* X, const double* b, int n, const double* sigma,
           int maxiter);                                            // mcg.cc:65

}  // namespace qwsg

// the opaque handle of the C ABI (include/qwsg.h)
struct qwsg_lattice {
  qwsg::Ctx* c;
};
