/* qwsg: native C ABI of the B200 domain-decomposed Wilson-clover solver.
 *
 * Status-returning, handle-based interface under the reference-compatible
 * symbols of qws_dropin.h.  Every function returns 0 on success and a
 * non-zero code on failure (1 bad argument, 2 unsupported parameter,
 * 3 CUDA error, 4 not initialised); qwsg_last_error() gives the message.
 * No torch types; plain pointers and sizes.
 *
 * Device spinor buffers hold 24 * pad reals (pad from qwsg_geometry) in the
 * library's structure-of-arrays "DD order" (colour-major, SAP-block-major);
 * convert from/to host arrays with qwsg_spinor_to_device_* / _to_host_*.
 * Host arrays in "natural" layout are indexed
 *   spinor [site][3 colour][4 spin][2]            site = x + Lx*(y + Ly*(z + Lz*t))
 *   gauge  [4 mu][site][3 row][3 col][2]          U_mu(x), row-major
 *   clover [site][2][36]                          QWS's packed chiral blocks of the
 *                                                  inverse clover term
 *                                                  (clover_def.h:88-284)
 *
 * Block grid NB[4]: the lattice is cut into SAP blocks of L/NB sites.
 * The reference's partition on an MPI rank grid npe[4] (two x-halves per
 * rank, qws.cc:141-148) is NB = (2*npe0, npe1, npe2, npe3); NB[0] must be
 * even and NB[1..3] 1 or even.
 */
#ifndef QWSG_H
#define QWSG_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct qwsg_lattice qwsg_lattice;

typedef struct {
  int outer_iters;            /* the reference's conviter (bicgstab_dd_mix.cc:381) */
  long inner_iters;           /* total inner BiCGStab iterations */
  double rel_resid_recursive; /* sqrt(|r|^2/|b|^2) of the recursive residual at exit */
  double rel_resid_true;      /* |b - D x| / |b| recomputed in FP64 (-1 if not requested) */
} qwsg_solve_stats;

const char* qwsg_last_error(void);
const char* qwsg_version(void);
/* kernels this library has launched in this process (the kernels of a
 * replayed CUDA graph included) */
long qwsg_launch_count(void);

/* lattice handle; tbc = +1 periodic / -1 antiperiodic time boundary
 * (fbc_f[3] of qws_init_, qws.cc:298-310) */
int qwsg_create(qwsg_lattice** out, const int L[4], const int NB[4], int tbc);
int qwsg_destroy(qwsg_lattice* lat);
/* run all work on this cudaStream_t (NULL = the legacy default stream);
 * until called, the handle uses a private non-blocking stream */
int qwsg_set_stream(qwsg_lattice* lat, void* cuda_stream);
/* No counterpart in the reference: give the handle a new private
 * non-blocking stream of this CUDA priority (lower = higher priority; the
 * library destroys it with the handle) and return it.  Handles driven from
 * several host threads need streams of their own: a CUDA graph captured on
 * a stream takes in every launch made into that stream meanwhile, from any
 * thread. */
int qwsg_own_stream(qwsg_lattice* lat, int priority, void** cuda_stream);
int qwsg_set_kappa(qwsg_lattice* lat, double kappa);
int qwsg_geometry(const qwsg_lattice* lat, int* volume, int* pad);
int qwsg_sync(qwsg_lattice* lat);

/* No counterpart in the reference (it solves one right-hand side per call).
 * A multi-RHS handle on the gauge field, clover term and kappa of `parent`:
 * nrhs (a power of two, 1..32) right-hand sides share every operator launch,
 * each link and clover entry being loaded once for all of them.  Its device
 * spinor buffers hold 24*pad*nrhs reals; the spinor transfer functions move
 * nrhs natural-layout spinors stored back to back ([nrhs][volume][24]).  The
 * DD operators, SAP preconditioners and DD solvers accept it; per-RHS scalars
 * and convergence, a converged RHS frozen at its single-solve iterate.  The
 * stats of a solve summarise all RHS (most iterations, largest residuals);
 * qwsg_batch_stats gives each RHS's.  Fields, kappa and the even-odd family
 * stay on the parent.  Destroy with qwsg_destroy before the parent. */
int qwsg_create_batch(qwsg_lattice** out, qwsg_lattice* parent, int nrhs);
/* a different kappa for every RHS of a multi-RHS handle (no counterpart in
 * the reference): builds the clover term of the parent's gauge field for
 * kappas[r] (csw as qwsg_build_clover) into the handle's own per-RHS planes;
 * every operator and solver on the handle then applies kappas[r] and its
 * clover to RHS r.  Call again to change the kappas. */
int qwsg_batch_set_kappas(qwsg_lattice* batch, const double* kappas, double csw);
/* a stopping tolerance for every RHS of a multi-RHS handle (no counterpart in
 * the reference, whose solvers take one tol): the FP64 outer solvers
 * (qwsg_bicgstab_dd_mix, qwsg_bicgstab_dd_mix2_hf) stop RHS r at tols[r]
 * (and restart it from its true residual until that is below tols[r]) in
 * place of their tol argument.  NULL restores the tol argument for all RHS. */
int qwsg_batch_set_tols(qwsg_lattice* batch, const double* tols);
/* Re-attach a multi-RHS handle to another lattice of the same extents, block
 * grid and time boundary (no counterpart in the reference): its work buffers
 * then serve that lattice's fields and kappa, so a pool of handles per volume
 * serves many gauge fields without allocating.  Per-RHS kappas and
 * tolerances are dropped (set them again) and the handle's CUDA graphs are
 * updated to the new fields before their next use; the handle's pending
 * work (on its own stream) is finished first.  The old parent is not
 * touched and may already be destroyed. */
int qwsg_batch_set_parent(qwsg_lattice* batch, qwsg_lattice* parent);
int qwsg_nrhs(const qwsg_lattice* lat, int* nrhs);
/* per-RHS results of the last multi-RHS solve: stats of the DD solvers,
 * iteration counts of the inner solvers (either pointer may be NULL) */
int qwsg_batch_stats(qwsg_lattice* lat, qwsg_solve_stats* per_rhs, int* iters_per_rhs);

/* resident fields, from host natural-layout FP64 arrays; the FP32 copies are
 * casts (as qws_loadg_dd_/qws_loadc_dd_ make them, qws_bqcd.cc:125-382) */
int qwsg_load_gauge(qwsg_lattice* lat, const double* U);
int qwsg_load_clover(qwsg_lattice* lat, const double* C);
/* optional explicit FP32 copies (main.cc writes glus/clvs itself) */
int qwsg_load_gauge_s(qwsg_lattice* lat, const float* U);
int qwsg_load_clover_s(qwsg_lattice* lat, const float* C);

/* No counterpart in the reference (QWS loads a clover term built and
 * inverted by BQCD, qws_bqcd.cc:284-382).  Builds the clover term of the
 * loaded FP64 gauge field on the GPU for this lattice's kappa: clover-leaf
 * F_{mu nu}, T = 1 - csw*kappa * sum sigma_{mu nu} F_{mu nu}, and the packed
 * inverse chiral blocks (the conventions of qwsg_gen_clover); replaces the
 * FP64 and FP32 clover planes.  Code 2 if a block is singular. */
int qwsg_build_clover(qwsg_lattice* lat, double csw);
/* No counterpart in the reference.  A seeded SU(3) gauge field smoothed by
 * n_smear APE-style steps, generated directly into this lattice's FP64 and
 * FP32 gauge planes with the host generator's construction and random
 * streams (qwsg_gen_gauge; equal to rounding); *plaq gets the plaquette.
 * The smearing uses the FP64 clover planes as scratch: build or load the
 * clover term afterwards. */
int qwsg_gen_gauge_device(qwsg_lattice* lat, unsigned long long seed, int n_smear, double alpha,
                          double* plaq);

/* host natural <-> device DD-order planes */
int qwsg_spinor_to_device_d(qwsg_lattice* lat, double* dev, const double* host);
int qwsg_spinor_to_host_d(qwsg_lattice* lat, double* host, const double* dev);
int qwsg_spinor_to_device_s(qwsg_lattice* lat, float* dev, const float* host);
int qwsg_spinor_to_host_s(qwsg_lattice* lat, float* host, const float* dev);

/* ---- operators on device buffers ---------------------------------------- */
/* full D = 1 - kappa A^-1 H (ddd_d_ qws.cc:625-632, ddd_s_ qws.cc:641-644) */
int qwsg_ddd_d(qwsg_lattice* lat, double* out, const double* in);
int qwsg_ddd_s(qwsg_lattice* lat, float* out, const float* in);
/* block-interior D on the blocks of one colour (ddd_in_{d,s}_,
 * ddd_in_d.cc:66-196, ddd_in_s.cc:376); other sites untouched */
int qwsg_ddd_in_d(qwsg_lattice* lat, double* out, const double* in, int colour);
int qwsg_ddd_in_s(qwsg_lattice* lat, float* out, const float* in, int colour);
/* out += factor A^-1 H_face in on one colour's block faces
 * (ddd_out_pre_*+ddd_out_pos_*, ddd_out_s.cc:639,661) */
int qwsg_ddd_out_d(qwsg_lattice* lat, double* out, const double* in, int colour, double factor);
int qwsg_ddd_out_s(qwsg_lattice* lat, float* out, const float* in, int colour, double factor);
/* jinv_ddd_in_s_ (static_solver.cc:141): nm Richardson steps on one colour */
int qwsg_jinv_s(qwsg_lattice* lat, float* x, const float* b, int colour, int nm);
/* No counterpart in the reference.  Same computation as qwsg_jinv_s, for
 * callers that cannot let the library allocate device memory (a fixed,
 * pre-reserved memory budget, or a loop that must not be stalled by the
 * device synchronisation an allocation can cause).  The intermediate
 * Richardson iterate lives in a 32 MiB array compiled into the library,
 * reserved on every GPU that loads it; lattices whose padded volume exceeds
 * 349,525 sites are rejected (code 2).  The first call on a device looks up
 * the array's device address (make it before any stream capture).  All calls
 * share the array: calls that overlap on the GPU race.  Handles made by
 * qwsg_create_batch are rejected (code 1).  The 12-real links are read when
 * an earlier FP32 call on the handle made them (qwsg_jinv_s does on SU(3)
 * fields), else the full links (equal to a few FP32 roundoffs). */
int qwsg_jinv_s_noalloc(qwsg_lattice* lat, float* x, const float* b, int colour, int nm);
/* prec_ddd_s_ (qws.cc:776) out = D M_SAP in ; prec_s_ (qws.cc:929) out = M_SAP in */
int qwsg_prec_ddd_s(qwsg_lattice* lat, float* out, const float* in, int nsap, int nm);
int qwsg_prec_s(qwsg_lattice* lat, float* out, const float* in, int nsap, int nm);

/* ---- solvers ----------------------------------------------------------- */
/* bicgstab_precdd_s_ (bicgstab_precdd_s.cc:85): x solves (D M) x = b from 0 */
int qwsg_bicgstab_precdd_s(qwsg_lattice* lat, float* x, const float* b, double tol, int maxiter,
                           int nsap, int nm, int* iters, double* final_rel);
/* bicgstab_dd_mix_ (bicgstab_dd_mix.cc:105): FP64 outer, FP32 SAP inner;
 * x holds the initial guess on entry.  stats may be NULL. */
int qwsg_bicgstab_dd_mix(qwsg_lattice* lat, double* x, const double* b, double tol, int maxiter,
                         double tol_s, int maxiter_s, int nsap, int nm, qwsg_solve_stats* stats);
/* Fault injection on the host, for tests (no counterpart in the reference):
 * from now on the single-RHS FP64 outer loop of this handle
 * (qwsg_bicgstab_dd_mix, qwsg_bicgstab_dd_mix2_hf) takes the reduction
 * <r0, q> as exactly zero at outer iteration outer_iter, so the reference's
 * breakdown guard (alpha = 0 when |<r0, q>| == 0, bicgstab_dd_mix.cc:192)
 * decides that step.  0 turns it off.  Nothing on the GPU is disturbed. */
int qwsg_inject_breakdown(qwsg_lattice* lat, int outer_iter);
/* |b - D x| / |b| in FP64 (one value per RHS on a multi-RHS handle) */
int qwsg_true_residual(qwsg_lattice* lat, const double* x, const double* b, double* rel);

/* ---- precision form: FP16 storage with per-site FP32 scales, FP32
 *      arithmetic, for the SAP preconditioner ----------------------------- */
/* assign_mult_mSAP_s_h_ (prec_ddd_s_h.h:63): out = M_SAP in with nsap-1 sweeps
 * + the final stage, fields and spinors stored in FP16 (the reference stores
 * the spinor with one global scale and computes in FP16, qws_h.cc:175-269) */
int qwsg_prec_s_h(qwsg_lattice* lat, float* out, const float* in, int nsap, int nm);
/* Single applications of the FP16-storage kernels the SAP above is made of,
 * FP32 in and out: the operands are stored in FP16 with per-site scales (as
 * the SAP stores them), the kernel runs, the result is converted back.
 * ddd_in_h_ (ddd_in_h.h:54): out = D_blk in on one colour's blocks */
int qwsg_ddd_in_h(qwsg_lattice* lat, float* out, const float* in, int colour);
/* jinv_ddd_in_h_ (jinv_ddd_in_h.h:53): nm Richardson steps on one colour */
int qwsg_jinv_h(qwsg_lattice* lat, float* x, const float* b, int colour, int nm);
/* ddd_out_pre_h_ + ddd_out_pos_h_ (ddd_out_h.h:57,283): out += factor
 * A^-1 H_face in on one colour's block faces */
int qwsg_ddd_out_h(qwsg_lattice* lat, float* out, const float* in, int colour, double factor);
/* The SAP half-sweep update s_c += in_c - D_blk a_c on one colour, in FP32
 * and in FP16 storage: the reference's inline loops qws.cc:815-818 and
 * prec_ddd_s_h.h:143-150 (no separate entry point there). */
int qwsg_sap_update_s(qwsg_lattice* lat, float* s, const float* a, const float* in, int colour);
int qwsg_sap_update_h(qwsg_lattice* lat, float* s, const float* a, const float* in, int colour);
/* The FP32 spinor field `in` as the FP16 kernels store it and read it back,
 * into `out` (FP32, device): per site (and RHS) n = max_i |v_i|, each
 * component stored as the FP16 round-to-nearest-even of the FP32 product
 * v_i * (1/n), read back as FP16 value * n in FP32; a site with n < 1e-30 is
 * stored as zero.  The storage format of assign_q_s2h_ / assign_q_h2s_
 * (qws_h.cc:175-269), which store one global scale for the whole field. */
int qwsg_store_h(qwsg_lattice* lat, float* out, const float* in);
/* bicgstab_precdd_s_h_ (bicgstab_precdd_s_h.cc:83): flexible FP32 BiCGStab
 * with the FP16 SAP preconditioner; x solves D x = b */
int qwsg_bicgstab_precdd_s_h(qwsg_lattice* lat, float* x, const float* b, double tol, int maxiter,
                             int nsap, int nm, int* iters, double* final_rel);
/* bicgstab_dd_mix2_hf_ (bicgstab_dd_mix2_hf.cc:110): FP64 outer around it.
 * reliable > 0: restart from the recomputed FP64 true residual (at most that
 * many times) until |b - D x| / |b| < tol; stats->rel_resid_true is set. */
int qwsg_bicgstab_dd_mix2_hf(qwsg_lattice* lat, double* x, const double* b, double tol, int maxiter,
                             double tol_s, int maxiter_s, int nsap, int nm, int reliable,
                             qwsg_solve_stats* stats);

/* ---- group solves: several lattices in common launches ---------------- */
/* No counterpart in the reference, whose bicgstab_dd_mix2_hf_
 * (bicgstab_dd_mix2_hf.cc:110) solves one lattice per call.  Each item is
 * one qwsg_bicgstab_dd_mix2_hf solve on its own one-RHS lattice handle (any
 * volume, block grid, fields, kappa and solver parameters; every handle at
 * most once).  The solves run together: each kernel step is one launch over
 * all lattices at that step, so small lattices share the GPU instead of
 * paying a launch and a mostly idle GPU each.  Every item's solution and
 * statistics are those its own qwsg_bicgstab_dd_mix2_hf call gives.  x holds
 * the initial guess on entry.  Work runs on `stream` (NULL: the first
 * item's handle's stream) after each handle's own stream is drained.
 * status: 0 or the error code of that item's solve -- the other items carry
 * on; the call returns the first non-zero status (qwsg_last_error names the
 * item).  stats may be NULL. */
typedef struct {
  qwsg_lattice* lat;
  double* x;
  const double* b;
  double tol;
  int maxiter;
  double tol_s;
  int maxiter_s, nsap, nm, reliable;
  qwsg_solve_stats stats; /* out */
  int status;             /* out */
} qwsg_group_item;
typedef struct {
  long rounds;           /* host read-back points of the group */
  long merged_launches;  /* kernel launches issued */
  long member_launches;  /* launches the items' own solves would have issued */
  /* host seconds spent waiting for the items' solves to reach their next
   * read-back, merging their launches, issuing launches and copies, and
   * waiting for the GPU */
  double t_members, t_merge, t_launch, t_gpu_wait;
} qwsg_group_stats;
int qwsg_group_bicgstab_dd_mix2_hf(qwsg_group_item* items, int n, void* stream,
                                   qwsg_group_stats* stats);

/* ---- synthetic fields (host, OpenMP; conventions in qws_b200/csrc/fields.cu) */
/* seeded SU(3) links, n_smear APE-style projected averaging steps with
 * weight alpha; writes the average plaquette (Re tr / 3) to *plaq */
int qwsg_gen_gauge(double* U, const int L[4], unsigned long long seed, int n_smear, double alpha,
                   double* plaq);
int qwsg_plaquette(const double* U, const int L[4], double* plaq);
/* clover-leaf clover term T = 1 - csw*kappa*sum_{mu<nu} sigma F, stored as QWS
 * packed chiral blocks of T^-1; T_out (optional) receives T [V][12][12][2] */
int qwsg_gen_clover(double* C, const double* U, const int L[4], double csw, double kappa,
                    double* T_out);
/* sources: kind 0 Gaussian, 1 point at the origin (arg = 4*colour + spin),
 * 2 Z2 noise */
int qwsg_gen_source(double* S, const int L[4], unsigned long long seed, int kind, int arg);

/* ---- even-odd (site parity) family -------------------------------------
 * Parity vectors are full device fields whose other-parity sites are zero.
 * deo: sites of parity pe receive the hops from the other parity.
 *   which 1 = hops inside the rank box L/(NB0/2, NB1, NB2, NB3) (deo_in_*,
 *         deo_in_d.cc:65), 2 = hops across its faces (deo_out_pre/pos_*,
 *         deo_out_d.cc:88,156), 3 = both (deo_vm_, qws.cc:518);
 *   dag   1 = the adjoint hopping (deo_dag_*, deo_dag_in.cc:64);
 *   clov  1 = multiply by the parity's A^-1 (dee_*);
 *   mode  0 out = hops, 1 out += factor*hops, 2 out = in0 + factor*hops
 *         (one_minus_*). */
int qwsg_set_parities(qwsg_lattice* lat, int pce, int pco);
int qwsg_deo_d(qwsg_lattice* lat, double* out, const double* in, int pe, int which, int dag,
               int clov, int mode, double factor, const double* in0);
int qwsg_deo_s(qwsg_lattice* lat, float* out, const float* in, int pe, int which, int dag,
               int clov, int mode, double factor, const float* in0);
/* clvd_vm2_/clv_s_ (qws.cc:390-441): out = A^-1 in on the parity-pe sites */
int qwsg_clv_d(qwsg_lattice* lat, double* out, const double* in, int pe);
int qwsg_clv_s(qwsg_lattice* lat, float* out, const float* in, int pe);
/* mtilde_vm_ (qws.cc:551): 1 - kappa^2 A_ee^-1 D_eo A_oo^-1 D_oe on parity pce;
 * mtilde_dag_vm_ (qws.cc:557); mtilde_s_ (qws.cc:598) */
int qwsg_mtilde_d(qwsg_lattice* lat, double* out, const double* in);
int qwsg_mtilde_dag_d(qwsg_lattice* lat, double* out, const double* in);
int qwsg_mtilde_s(qwsg_lattice* lat, float* out, const float* in);
/* bicgstab_vm_ (bicgstab.cc:68): BiCGStab on mtilde, x = initial guess in,
 * solution out; iters = the reference's conviter */
int qwsg_bicgstab_vm(qwsg_lattice* lat, double* x, const double* b, int maxiter, int* iters);
/* mtdagmt_vm_ (qws.cc:566): mtilde_dag(mtilde(in)) on parity pce */
int qwsg_mtdagmt_d(qwsg_lattice* lat, double* out, const double* in);
/* cg_vm_ (cg.cc:65): CG on mtdagmt, x = initial guess in, solution out,
 * stopping at sqrt(|r|^2/|b|^2) < 1e-14 or iteration maxiter-1; iters = the
 * last iteration (the reference does not return it) */
int qwsg_cg_vm(qwsg_lattice* lat, double* x, const double* b, int maxiter, int* iters);
/* mcg_vm_ (mcg.cc:65): multi-shift CG, (mtdagmt + sigma[k]) x_k = b for
 * k < nshift (1..32), x_k from zero; x holds the nshift solutions back to
 * back (24*pad reals each, qwsg_geometry); sigma is a host array */
int qwsg_mcg_vm(qwsg_lattice* lat, double* x, const double* b, int nshift, const double* sigma,
                int maxiter, int* iters);

/* BQCD-format arrays converted on the device (the reference's loaders,
 * qws_bqcd.cc:66-642, reorder on the host into QWS's layout instead).
 * Links u[ri + 2*row + 6*col + 18*slot + 18*V*mu], clover
 * c[perm[k] + 36*ud + 72*slot] (qws_bqcd.cc:125-377), spinors as an even and
 * an odd array of V/2 sites, element 2*s + 8*c + ri + 24*(i-1)
 * (qws_bqcd.cc:500-642; nrhs arrays back to back on a batch handle).
 * slot = (i-1) + V/2*eo for the site's 1-based index i within its parity
 * eo.  site_map: host array, site_map[n] = slot of natural site
 * n = x + Lx*(y + Ly*(z + Lz*t)); NULL = i-1 = n/2 (the numbering the
 * drop-in uses when the host program has no std_xyzt2i_). */
int qwsg_load_gauge_bqcd(qwsg_lattice* lat, const double* u, const int* site_map);
int qwsg_load_clover_bqcd(qwsg_lattice* lat, const double* c, const int* site_map);
int qwsg_spinor_from_bqcd_d(qwsg_lattice* lat, double* dev, const double* even,
                            const double* odd, const int* site_map);
int qwsg_spinor_from_bqcd_s(qwsg_lattice* lat, float* dev, const double* even, const double* odd,
                            const int* site_map);
int qwsg_spinor_to_bqcd_d(qwsg_lattice* lat, double* even, double* odd, const double* dev,
                          const int* site_map);
int qwsg_spinor_to_bqcd_s(qwsg_lattice* lat, double* even, double* odd, const float* dev,
                          const int* site_map);

/* CUDA graphs for the SAP preconditioner's launch sequences (default on):
 * captured on first use per buffers/nsap/nm/kappa, replayed afterwards; not
 * used while kernel timing is on or on the legacy default stream */
int qwsg_set_graphs(qwsg_lattice* lat, int enable);
/* FP32 links in 12-real form (no counterpart in the reference): with mode
 * 1 (default) the FP32 Dirac kernels read the first two rows of each link
 * and rebuild the third when every loaded link is SU(3) to 1e-5 (checked
 * on the device once per load); mode 0 always reads all 18 reals.
 * qwsg_link_compression reports whether the 12-real form is in use. */
int qwsg_set_link_compression(qwsg_lattice* lat, int mode);
int qwsg_link_compression(qwsg_lattice* lat, int* active);
/* threads per CTA of the Dirac-operator kernels on this handle (64, 128
 * (default) or 256); a batch handle starts with its parent's value.  No
 * counterpart in the reference (its loops are OpenMP threads over sites). */
int qwsg_set_hop_threads(qwsg_lattice* lat, int threads);
/* per-kernel CUDA-event timing on the handle's stream: enable (clears the
 * records) or disable; stats fills, per kernel kind k < *nkind, the number
 * of launches, the summed device milliseconds and the summed algorithmic
 * bytes (bytes each launch must move: spinors, links, clover) */
int qwsg_kernel_timing(qwsg_lattice* lat, int enable);
int qwsg_kernel_stats(qwsg_lattice* lat, int* nkind, long* launches, double* ms, double* bytes);
const char* qwsg_kernel_name(int kind);

/* per-region call counters (reference region names, timing.h) */
int qwsg_counters(qwsg_lattice* lat, long* prec_ddd_s, long* prec_s, long* jinv,
                  long* inner_iters, long* ddd_d);

#ifdef __cplusplus
}
#endif
#endif
