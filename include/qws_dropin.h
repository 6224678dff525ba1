/* Drop-in C ABI: the reference's own entry points and host data layouts,
 * implemented by libqws_b200.so on one B200 that holds the whole lattice.
 *
 * A program written against QWS (its main.cc, or BQCD through libqws.a) links
 * against this library instead: same symbol names (Fortran-style trailing
 * underscores, every argument by pointer), same host arrays, same globals.
 * Arrays stay in host memory in QWS's SIMD-lane layout; each call moves them
 * to the GPU's planes, computes there and moves results back.  Gauge and
 * clover fields are uploaded once and kept resident; they are re-uploaded
 * after the loaders run, after qwsg_mark_fields_dirty(), or at every call
 * when the environment variable QWSG_ALWAYS_UPLOAD=1 (for callers that write
 * glud/glus/clvd/clvs directly between calls, as main.cc:416-518 does once).
 *
 * Layout widths: VLEND/VLENS (qws.h:53-58) are compile-time in QWS.  The
 * library reads QWSG_VLEND / QWSG_VLENS from the environment at qws_init_
 * (defaults 8 and 16, QWS's defaults) or takes qwsg_set_host_vlen() before
 * qws_init_; the caller's macros must match.
 *
 * Single GPU: the rank grid npe must be all 1 (the whole lattice is one
 * "rank" whose two x-halves are the SAP blocks).  For the reference's
 * partition on a larger rank grid use the qwsg_* API (qwsg.h) with
 * NB = (2*npe0, npe1, npe2, npe3).
 */
#ifndef QWS_DROPIN_H
#define QWS_DROPIN_H
#include <stdio.h>

#ifndef VLEND
#define VLEND 8
#endif
#ifndef VLENS
#define VLENS 16
#endif
#define NEO 2
#define NDIM 4
#define NCOL 3
#ifndef CLS
#define CLS 256
#endif

/* Types with the reference's memory layout (qws.h:111-192): every real is a
 * vector over VLEN consecutive x sites of one x-half.  Links are stored
 * column-major, c[col][row]. */
typedef struct {
  double v[VLEND];
} rvecd_t;
typedef union {
  double c[3][3][2][VLEND];
} glud_t, *pglud_t;
typedef union {
  double c[2][36][VLEND];
  rvecd_t cv[2][36];
} clvd_t, *pclvd_t;
typedef union {
  double c[3][4][2][VLEND];
  rvecd_t cv[3][4][2];
  rvecd_t cs[12][2];
  rvecd_t ccs[24];
} scd_t;
typedef struct {
  float v[VLENS];
} rvecs_t;
typedef union {
  float c[3][3][2][VLENS];
} glus_t, *pglus_t;
typedef union {
  float c[2][36][VLENS];
  rvecs_t cv[2][36];
} clvs_t, *pclvs_t;
typedef union {
  float c[3][4][2][VLENS];
  rvecs_t cv[3][4][2];
  rvecs_t cs[12][2];
  rvecs_t ccs[24];
} scs_t;

#ifdef __cplusplus
extern "C" {
#endif

/* ---- globals the reference exports and main.cc reads/writes
 *      (qws.cc:74-127, main.cc:94-121) ---------------------------------- */
extern pglud_t glud;
extern pglus_t glus;
extern pclvd_t clvd;
extern pclvs_t clvs;
extern double kappa, kappa2, mkappa;
extern int nx, ny, nz, nt, nxh, nxd, nxs, vold, vols;
extern int rank, npe[4], domain_e, domain_o;
extern double fbc[4][2];
extern FILE* para_outputfile;

/* ---- set-up (qws.cc:130-316, 319-336) ----------------------------------- */
void qws_init_(int* lx, int* ly, int* lz, int* lt, int* npe_f, int* fbc_f, int* pce_f,
               int* pco_f, int* block_size);
void qws_finalize_(void);

/* ---- BQCD-layout loaders (qws_bqcd.cc:125-182, 284-382, 500-642);
 *      they call the host program's std_xyzt2i_/e_o_ when it defines them
 *      (qws_bqcd.cc:56-57), else index sites lexicographically within
 *      parity (i = lex/2 + 1, eo = (x+y+z+t)%2) ---------------------------- */
void qws_loadg_dd_(double* u, int* volh_tot, double* in_kappa);
void qws_loadc_dd_(double* c, int* volh);
void qws_loadfd_dd_(scd_t* out, double* ine, double* ino);
void qws_storefd_dd_(double* oute, double* outo, scd_t* in);
void qws_loadfs_dd_(scs_t* out, double* ine, double* ino);
void qws_storefs_dd_(double* oute, double* outo, scs_t* in);
/* even-odd layout (qws_bqcd.cc:66-123, 184-282, 384-498): site (x,y,z,t) of
 * parity p sits in x-half slot p at compressed x/2; the spinor loaders move
 * the even sites of a half array only */
void qws_loadg_bqcd_(double* u, int* volh_tot, double* in_kappa);
void qws_loadc_bqcd_(double* c, int* volh);
void qws_loadfd_bqcd_(scd_t* out, double* in);
void qws_loadfs_bqcd_(scs_t* out, double* in);
void qws_storefd_bqcd_(double* out, scd_t* in);
void qws_storefs_bqcd_(double* out, scs_t* in);

/* ---- even-odd (site parity) operators (qws.cc:390-605, deo_in_d.cc:65,
 *      deo_in_s.cc:65, deo_out_d.cc:88, deo_out_s.cc:93, deo_dag_in.cc,
 *      deo_dag_out.cc).  Arguments are one-parity half arrays of the
 *      even-odd layout: out of parity *pe, in of parity *po = 1 - *pe,
 *      in0 of parity *pe.  H_eo = hopping from po to pe sites (in: inside
 *      the rank box, out: across its faces), A^-1 the clover inverse:
 *        deo_*          out  = H in        dee_deo_*   out = A^-1 H in
 *        *_dag_*        the adjoint hop    one_minus_* out = in0 + f A^-1 H in
 *        *_out_pre_*    keeps `in` for the following *_out_pos_*
 *        *_out_pos_*    out += factor (A^-1) H_out (the kept field)
 *      mtilde_* act on parity-pce half arrays (qws_init_'s pce_f):
 *        mtilde = 1 - kappa^2 A_ee^-1 H_eo A_oo^-1 H_oe ----------------------- */
void deo_in_vm_(int* pe, int* po, scd_t* out, scd_t* in);
void dee_deo_in_vm_(int* pe, int* po, scd_t* out, scd_t* in);
void deo_dag_in_vm_(int* pe, int* po, scd_t* out, scd_t* in);
void dee_deo_dag_in_vm_(int* pe, int* po, scd_t* out, scd_t* in);
void one_minus_dee_deo_in_vm_(int* pe, int* po, scd_t* out, scd_t* in, scd_t* in0, double factor);
void one_minus_deo_dag_in_vm_(int* pe, int* po, scd_t* out, scd_t* in, scd_t* in0, double factor);
void deo_out_pre_vm_(int* pe, int* po, scd_t* out, scd_t* in);
void deo_dag_out_pre_vm_(int* pe, int* po, scd_t* out, scd_t* in);
void deo_out_pos_vm_(int* pe, int* po, scd_t* out, scd_t* in, double factor);
void deo_dag_out_pos_vm_(int* pe, int* po, scd_t* out, scd_t* in, double factor);
void dee_deo_out_pos_vm_(int* pe, int* po, scd_t* out, scd_t* in, double factor);
void dee_deo_dag_out_pos_vm_(int* pe, int* po, scd_t* out, scd_t* in, double factor);
void clvd_vm_(int* pe, scd_t* inout);
void clvd_vm2_(int* pe, scd_t* out, scd_t* in);
void deo_vm_(int* pe, int* po, scd_t* out, scd_t* in);
void dee_deo_vm_(int* pe, int* po, scd_t* out, scd_t* in);
void one_minus_dee_deo_vm_(int* pe, int* po, scd_t* out, scd_t* in, scd_t* in0);
void deo_dag_vm_(int* pe, int* po, scd_t* out, scd_t* in);
void dee_deo_dag_vm_(int* pe, int* po, scd_t* out, scd_t* in);
void one_minus_deo_dag_vm_(int* pe, int* po, scd_t* out, scd_t* in, scd_t* in0);
void mtilde_vm_(scd_t* out, scd_t* in);
void mtilde_dag_vm_(scd_t* out, scd_t* in);
void mtdagmt_vm_(scd_t* out, scd_t* in);
/* bicgstab.cc:68 ; x: initial guess in, solution out; conviter = iterations */
void bicgstab_vm_(scd_t* x, scd_t* b, int* conviter, int* maxiter);
/* cg.cc:65 (conviter: written here with the last iteration; the reference
 * leaves it unset) and mcg.cc:65 (xx: *n half arrays of vold scd_t back to
 * back, zeroed and solved for shifts sigma[0..*n-1], *n <= 32) */
void cg_vm_(scd_t* x, scd_t* b, int* conviter, int* maxiter);
void mcg_vm_(scd_t* xx, scd_t* b, int* n, double* sigma, int* maxiter);
void deo_in_s_(int* pe, int* po, scs_t* out, scs_t* in);
void dee_deo_in_s_(int* pe, int* po, scs_t* out, scs_t* in);
void one_minus_dee_deo_in_s_(int* pe, int* po, scs_t* out, scs_t* in, scs_t* in0, float factor);
void deo_out_pre_s_(const int* pe, const int* po, const scs_t* out, const scs_t* in);
/* writes *out although the reference declares it const (qws.cc:578) */
void deo_out_pos_s_(const int* pe, const int* po, const scs_t* out, const scs_t* in, float factor);
void dee_deo_out_pos_s_(int* pe, int* po, scs_t* out, scs_t* in, float factor);
void clv_s_(int* pe, scs_t* inout);
void deo_s_(int* pe, int* po, scs_t* out, scs_t* in);
void dee_deo_s_(int* pe, int* po, scs_t* out, scs_t* in);
void one_minus_dee_deo_s_(int* pe, int* po, scs_t* out, scs_t* in, scs_t* in0);
void mtilde_s_(scs_t* out, scs_t* in);

/* ---- solvers ------------------------------------------------------------- */
/* bicgstab_dd_mix.cc:105 ; conviter = outer iterations */
void bicgstab_dd_mix_(scd_t* x, scd_t* b, double* tol, int* conviter, int* maxiter,
                      double* tol_s, int* maxiter_s, int* nsap, int* nm);
/* bicgstab_precdd_s.cc:85 ; conviter = iterations run (the reference keeps
 * that count only under _DEBUG_ and returns 0 otherwise) */
void bicgstab_precdd_s_(scs_t* x, scs_t* b, double* tol, int* conviter, int* maxiter, int* nsap,
                        int* nm);

/* ---- half-precision pair (qws_h.h:60-62, bicgstab_precdd_s_h.cc:83,
 *      bicgstab_dd_mix2_hf.cc:110, qws_bqcd.cc:647).  Here the SAP runs with
 *      FP16 storage and per-site FP32 scales, arithmetic in FP32. ---------- */
void qws_h_init_(const glus_t* glus, const clvs_t* clvs);
void bqcd_qws_h_init_(void);
void assign_mult_mSAP_s_h_(scs_t* xs, const scs_t* bs, const int* nsap, const int* nm);
void assign_mult_wd_s_(scs_t* x, const scs_t* b);
void bicgstab_precdd_s_h_(scs_t* x, const scs_t* b, const double* tol, int* conviter,
                          const int* maxiter, const int* nsap, const int* nm);
void bicgstab_dd_mix2_hf_(scd_t* x, const scd_t* b, const double* tol, int* conviter,
                          const int* maxiter, const double* tol_s, const int* maxiter_s,
                          const int* nsap, const int* nm);

/* ---- SAP preconditioner (qws.cc:776, 929; static_solver.cc:141) --------- */
void prec_ddd_s_(scs_t* out, scs_t* in, int* nsap, int* nm);
void prec_s_(scs_t* out, scs_t* in, int* nsap, int* nm);
/* x, b: the half arrays of domain *DEO */
void jinv_ddd_in_s_(scs_t* x, scs_t* b, int* DEO, int* maxiter);

/* ---- DD operator (qws.cc:625-644, ddd_in_d.cc:66, ddd_in_s.cc:376,
 *      ddd_out_d.cc:84,164, ddd_out_s.cc:633-673) ------------------------- */
void ddd_d_(scd_t* out, scd_t* in);
void ddd_s_(scs_t* out, scs_t* in);
void ddd_eo_s_(scs_t* out, scs_t* in, int* domain);
/* out, in: the half arrays of domain *DEO */
void ddd_in_d_(scd_t* out, scd_t* in, int* DEO);
void ddd_in_s_(scs_t* out, scs_t* in, int* DEO);
/* pre: captures the faces of the full field `in` for domain *DEO;
 * pos: out (half array of *DEO) += factor A^-1 H_face (captured faces)
 *      (the FP64 version uses factor = -kappa, ddd_out_d.cc:225) */
void ddd_out_pre_d_(scd_t* in, int* DEO);
void ddd_out_pos_d_(scd_t* out, scd_t* in, int* DEO);
void ddd_out_pre_s_(scs_t* in, int* DEO);
void ddd_out_pos_s_(scs_t* out, scs_t* in, int* DEO, float factor);
void ddd_out_pre_s_no_timer_(scs_t* in, int* DEO);
void ddd_out_pos_s_no_timer_(scs_t* out, scs_t* in, int* DEO, float factor);

/* ---- precision / layout converters (reordering.cc:59-204) --------------- */
void fermi_reorder_s2d_dd_(scd_t* out, const scs_t* in);
void fermi_reorder_d2s_dd_(scs_t* out, const scd_t* in);
void fermi_reorder_s2d_dd_renorm_(scd_t* out, const scs_t* in, const double* dnorm);
void fermi_reorder_d2s_dd_renorm_(scs_t* out, const scd_t* in, double* dnorm);

/* ---- helpers (qws.cc:445-502, timing.c) ---------------------------------- */
void print_scdnorm2(const char* a, scd_t* in, int size);
void print_scsnorm2(const char* a, scs_t* in, int size);
void zero_scd_field(scd_t* inout, int size);
void zero_scs_field(scs_t* inout, int size);
double get_clock(void);
void print_timing_(void);

/* ---- additions of this library (no counterpart in the reference) ------- */
/* host lane widths of the QWS layout; call before qws_init_ */
int qwsg_set_host_vlen(int vlend, int vlens);
/* glud/glus/clvd/clvs were written directly: upload them at the next call */
int qwsg_mark_fields_dirty(void);
/* the qwsg_lattice behind the drop-in state (NULL before qws_init_) */
struct qwsg_lattice* qwsg_dropin_lattice(void);

#ifdef __cplusplus
}
#endif
#endif
