/* CPU restatement of QWS's domain-decomposed Wilson-clover solver path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker the CUDA path is compared
 * against.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg may load it; the product never links or calls it.
 *
 * Parity pinning: the restatement reproduces the reference's own golden
 * files data/CASE0 and data/CASE_4111_1111 (operator norms and the DD-solve
 * bnorm^2/rnorm^2/xnorm^2 under check.sh's tolerances) and is compared
 * vector-by-vector against the reference's sources compiled from source
 * (oracle/_ref, see oracle/Makefile).
 *
 * Layout ("natural"): site s = x + Lx*(y + Ly*(z + Lz*t)) over the GLOBAL
 * lattice.  Spinor T[V][3 colour][4 spin][2 re/im]  (QWS's own inner order,
 * qws.h:134-139).  Gauge T[4 mu][V][3 row][3 col][2].  Clover T[V][2][36]
 * in QWS's packed chiral-block format (clover_def.h:88-284).
 *
 * Blocks: the lattice is cut into NB[0]xNB[1]xNB[2]xNB[3] boxes.  The
 * reference's partition on an MPI grid npe[4] is NB = (2*npe0, npe1, npe2,
 * npe3): each rank's local volume split into two x-halves ("domains",
 * qws.cc:141-148, 224-225).  Block colour = (ibx+iby+ibz+ibt) % 2, which is
 * the reference's domain_e/domain_o assignment (qws.cc:224-225, 275-276).
 * Block "domain" = ibx % 2 (the x-half index the reference's ddd_* take).
 */
#ifndef QWS_ORACLE_H
#define QWS_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_lat orc_lat;

/* geometry; tbc multiplies hops across the global t boundary (fbc_f[3]). */
orc_lat* orc_create(const int L[4], const int NB[4], int tbc);
void orc_destroy(orc_lat*);
void orc_set_kappa(orc_lat*, double kappa);
long orc_volume(const orc_lat*);

/* fields in natural layout; the FP32 copies are (float) of the FP64 ones
 * unless set explicitly (main.cc:436-496 writes both from the same draws). */
void orc_set_gauge_d(orc_lat*, const double* U);
void orc_set_clover_d(orc_lat*, const double* C);
void orc_set_gauge_s(orc_lat*, const float* U);
void orc_set_clover_s(orc_lat*, const float* C);

/* main.cc:406-518 generator: std::mt19937(12345) Box-Muller fields on one
 * local lattice Lloc, tiled over the rank grid npe (every rank seeds
 * identically, main.cc:129).  Writes U (natural, global), C, and then
 * draws `nsrc` spinors (generate_random_sc, main.cc:498-523) into
 * src[nsrc][V][24] (tiled likewise). */
void orc_gen_main_fields(const int Lloc[4], const int npe[4], double* U,
                         double* C, int nsrc, double* src);

/* ---- DD operator ------------------------------------------------------- */
/* selection of blocks: kind 0 = by colour, kind 1 = by domain (ibx%2);
 * orc_ddd_out_s also takes kind 2 = by domain with the FP32 face packer's
 * x-half pairing across rank faces (ddd_out_s.cc:128-131), which is what the
 * reference computes when every rank passes the same domain index. */
void orc_ddd_in_d(orc_lat*, double* out, const double* in, int kind, int sel);
void orc_ddd_out_d(orc_lat*, double* out, const double* in, int kind, int sel,
                   double factor);
void orc_ddd_d(orc_lat*, double* out, const double* in);
void orc_ddd_in_s(orc_lat*, float* out, const float* in, int kind, int sel);
void orc_ddd_out_s(orc_lat*, float* out, const float* in, int kind, int sel,
                   float factor);
void orc_ddd_s(orc_lat*, float* out, const float* in);
void orc_clover_d(orc_lat*, double* inout);
void orc_clover_s(orc_lat*, float* inout);

/* ---- SAP preconditioner and solvers ----------------------------------- */
void orc_jinv_s(orc_lat*, float* x, const float* b, int colour, int nm);
void orc_prec_ddd_s(orc_lat*, float* out, const float* in, int nsap, int nm);
void orc_prec_s(orc_lat*, float* out, const float* in, int nsap, int nm);
/* returns the number of inner iterations executed (the reference keeps that
 * count only under _DEBUG_, bicgstab_precdd_s.cc:117-120) */
int orc_bicgstab_precdd_s(orc_lat*, float* x, const float* b, double tol,
                          int maxiter, int nsap, int nm, double* final_rel);
/* stats[0]=outer iterations (the reference's conviter), stats[1]=total inner
 * iterations, stats[2]=last rnorm^2/bnorm^2 (recursive), hist: optional
 * array of 2*maxiter recursive residuals sqrt(rnorm/bnorm) (NaN-padded). */
void orc_bicgstab_dd_mix(orc_lat*, double* x, const double* b, double tol,
                         int maxiter, double tol_s, int maxiter_s, int nsap,
                         int nm, double* stats, double* hist);

/* test hook: the outer loop of orc_bicgstab_dd_mix takes <r0, q> as zero at
 * outer iteration `outer_iter` (0: never), exercising the reference's
 * breakdown guard (bicgstab_dd_mix.cc:192) */
void orc_plant_breakdown(int outer_iter);

/* ---- half-precision solver pair, restated in FP32 ----------------------- */
/* assign_mult_mSAP_s_h_ (prec_ddd_s_h.h:63-231) is prec_s_ with nsap-1 sweeps;
 * the flexible inner solver (bicgstab_precdd_s_h.cc:83-369) with that M and the
 * FP32 D, and its FP64 outer loop (bicgstab_dd_mix2_hf.cc:110-373,
 * iter = 0..maxiter-1).  Same return conventions as the plain pair. */
int orc_bicgstab_precdd_s_h(orc_lat*, float* x, const float* b, double tol, int maxiter,
                            int nsap, int nm, double* final_rel);
void orc_bicgstab_dd_mix2_hf(orc_lat*, double* x, const double* b, double tol, int maxiter,
                             double tol_s, int maxiter_s, int nsap, int nm, double* stats);

/* ---- even-odd (site parity) family, natural layout, parity 0 = pce ------ */
void orc_mtilde_d(orc_lat*, double* out, const double* in);      /* qws.cc:551 */
void orc_mtilde_dag_d(orc_lat*, double* out, const double* in);  /* qws.cc:557 */
void orc_mtdagmt_d(orc_lat*, double* out, const double* in);     /* qws.cc:566 */
int orc_bicgstab_vm(orc_lat*, double* x, const double* b, int maxiter);  /* bicgstab.cc:68 */
/* cg_vm_ (cg.cc:65): x = initial guess in, solution out, returns the last
 * iteration; mcg_vm_ (mcg.cc:65): X holds n solutions back to back, zeroed first */
int orc_cg_vm(orc_lat*, double* x, const double* b, int maxiter);
int orc_mcg_vm(orc_lat*, double* X, const double* b, int n, const double* sigma, int maxiter);

/* ---- norms -------------------------------------------------------------- */
double orc_norm2_d(const double* v, long n);
double orc_norm2_s(const float* v, long n);

#ifdef __cplusplus
}
#endif
#endif
