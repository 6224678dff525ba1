// Kernel launch interface shared by the host-side solver code.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstring>
#include <functional>
#include <vector>

#include "lattice.cuh"

namespace qwsg {

// ---------------------------------------------------------------------------
// Group solves (group.cu): several lattices, each solved by its own host
// thread running the unchanged one-lattice solver, with every kernel launch
// recorded instead of issued.  At each point where a solver reads a result
// back, the launches the lattices recorded since their last read-back are
// merged position by position into one launch over all of them.  A record
// holds the launch's argument block and the function that merges it.
// ---------------------------------------------------------------------------
struct GroupRec;
struct GroupBatch;
using GroupMergeFn = void (*)(const GroupRec* const* recs, int n, GroupBatch& b);
struct GroupRec {
  GroupMergeFn merge;  // also the launch's identity: the same function merges
  alignas(16) unsigned char data[512];
};
struct GroupRecorder {
  std::vector<GroupRec> recs;
};
// the recorder of the calling thread (null outside a group solve)
extern thread_local GroupRecorder* g_group_rec;
template <typename A>
inline bool group_record(GroupMergeFn f, const A& a) {
  static_assert(sizeof(A) <= sizeof(GroupRec::data), "group record too large");
  if (!g_group_rec) return false;
  g_group_rec->recs.emplace_back();
  GroupRec& r = g_group_rec->recs.back();
  r.merge = f;
  std::memcpy(r.data, &a, sizeof(A));
  return true;
}
template <typename A>
inline const A& group_arg(const GroupRec* r) {
  return *reinterpret_cast<const A*>(r->data);
}
// One round's merged launches: argument tables staged on the host, uploaded
// in one copy, then the launches run with the device address of the copy.
struct GroupBatch {
  std::vector<unsigned char> host;
  std::vector<std::function<void(const unsigned char* dev, cudaStream_t st)>> launches;
  size_t put(const void* p, size_t n) {  // 16-byte aligned offset of the copy
    const size_t off = (host.size() + 15) & ~size_t(15);
    host.resize(off + n);
    std::memcpy(host.data() + off, p, n);
    return off;
  }
  // block starts of a merged launch: starts[l] = first block of member l,
  // starts[n] = the total; returns the offset of the table
  size_t put_starts(const std::vector<int>& starts) {
    return put(starts.data(), sizeof(int) * starts.size());
  }
};
[[noreturn]] void group_unrecorded_launch();

// kernels launched by this library in this process (host-side count; a CUDA
// graph replay adds the launches it captured).  Every launcher counts its
// launch; one reached while the thread records for a group solve is a launch
// the group cannot merge, which is an error.
extern std::atomic<long> g_kernel_launches;
inline void count_launch() {
  if (g_group_rec) group_unrecorded_launch();
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

#ifdef __CUDACC__
// the member whose blocks include block b of a merged launch: the largest l
// with starts[l] <= b (members without blocks have starts[l] == starts[l+1])
__device__ __forceinline__ int group_member(const int* __restrict__ starts, int n, int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(starts + mid) <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}
// copy a member's argument block into shared memory (all threads take part)
template <typename A>
__device__ __forceinline__ void group_load_args(A& dst, const A* __restrict__ src) {
  static_assert(sizeof(A) % sizeof(int) == 0, "argument block size");
  const int* s = reinterpret_cast<const int*>(src);
  int* d = reinterpret_cast<int*>(&dst);
  for (int k = threadIdx.x; k < (int)(sizeof(A) / sizeof(int)); k += blockDim.x) d[k] = s[k];
  __syncthreads();
}
#endif

enum { HOP_INNER = 1, HOP_OUTER = 2, HOP_ALL = 3 };
enum { EPI_D = 0, EPI_ADD = 1, EPI_JINV = 2, EPI_SAPE = 3 };

// T: storage tag (float, double, H16 = FP16 storage / FP32 arithmetic)
template <typename T>
struct HopArgs {
  using S = typename Store<T>::type;
  Geom G;
  const S* src;   // field the hops read
  const S* aux;   // b (EPI_JINV) or the SAP right-hand side `in` (EPI_SAPE)
  S* out;
  const S* U;     // gauge planes
  const S* U12;   // FP32 only: links in 12-real form (null: use U)
  // per-RHS kappa (multi-RHS handles): clover planes per (site, RHS) entry
  // (stride spad) and kappa per RHS; the epilogue's coefficient is then
  // kap[rhs] with coef's sign (coef is +-kappa in every such launch)
  const S* Cr;
  const typename Arith<T>::R* kap;
  const S* C;     // clover planes
  typename Arith<T>::R coef;
  const int* list;  // if set: thread i handles site list[i], else site0 + i
  int site0;      // first site (DD order) handled
  int nsites;     // number of sites handled
  int dom;        // >= 0: only sites whose block has ibx % 2 == dom
  int zero_col;   // >= 0: face hops landing on this colour contribute zero
};

template <typename R>
void launch_hop(int sel, int epi, const HopArgs<R>& a, cudaStream_t st);

// even-odd (site parity) hopping, eo.cu
template <typename T>
struct EoArgs {
  using S = typename Store<T>::type;
  Geom G;
  const S* src;
  const S* in0;
  S* out;
  const S* U;
  const S* C;
  typename Arith<T>::R coef;
  int pe;      // parity of the output sites
  int box[4];  // the rank's local extents (inside / face classification)
};
template <typename T>
void launch_eo(int which, int dag, int clov, int mode, const EoArgs<T>& a, cudaStream_t st);
template <typename T>
void launch_clv(const EoArgs<T>& a, cudaStream_t st);
// dst = src on the sites of parity pe, 0 elsewhere
template <typename T>
void parity_select(const Geom& G, typename Store<T>::type* dst, const typename Store<T>::type* src,
                   int pe, cudaStream_t st);
[[noreturn]] void throw_unsupported_eo();

// ---------------------------------------------------------------------------
// BLAS-1 on spinor planes (complex per-site vectors of 12 components), over
// every right-hand side of the field.  Reductions are per RHS, written to
// res[4*rhs + k] (device, double) deterministically.
// ---------------------------------------------------------------------------
struct RedBuf {
  double* partial;    // [nblk * 32 rhs * 4]
  unsigned* counter;  // completion counter of the running reduction
  int nblk;           // most blocks a reduction launch uses
};

template <typename R>
void blas_copy(const Geom& G, R* y, const R* x, int site0, int n, cudaStream_t st);
template <typename R>
void blas_zero(const Geom& G, R* y, int site0, int n, cudaStream_t st);
// res[0] = |x|^2   (res[4*rhs] for each right-hand side, and so on below)
template <typename R>
void blas_norm2(const Geom& G, const R* x, double* res, RedBuf& rb, cudaStream_t st);
// res[0..1] = <x,y> = sum conj(x) y
template <typename R>
void blas_cdot(const Geom& G, const R* x, const R* y, double* res, RedBuf& rb, cudaStream_t st);
// res[0] = |y|^2, res[1..2] = <y,x>  (omega step: |t|^2, <t,r>)
template <typename R>
void blas_norm_cdot(const Geom& G, const R* y, const R* x, double* res, RedBuf& rb,
                    cudaStream_t st);
// x += a p ; r -= a q ; res[0] = |r|^2 ; optionally res[1..2] = <r0, r>
// (cf: per-RHS (ar, ai) table on the device, cf[4*rhs + 0..1], else the values)
template <typename R>
void blas_bicg_update(const Geom& G, R* x, R* r, const R* p, const R* q, double ar, double ai,
                      const R* r0, double* res, RedBuf& rb, cudaStream_t st,
                      const double* cf = nullptr);
// p = r + b (p - w q)   (cf: per-RHS (br, bi, wr, wi))
template <typename R>
void blas_bicg_p(const Geom& G, R* p, const R* r, const R* q, double br, double bi, double wr,
                 double wi, cudaStream_t st, const double* cf = nullptr);
// r = b - q ; p = r ; r0 = r ; res[0] = |b|^2 ; res[1] = |r|^2
template <typename R>
void blas_bicg_init(const Geom& G, const R* b, const R* q, R* r, R* p, R* r0, double* res,
                    RedBuf& rb, cudaStream_t st);
// r += a q ; res[0] = |r|^2   (real a; the residual step of mcg.cc:118-138)
template <typename R>
void blas_axpy_norm(const Geom& G, R* r, const R* q, double a, double* res, RedBuf& rb,
                    cudaStream_t st);
// one multi-shift CG step for n shifts (mcg.cc:141-205), single RHS:
// x_k -= c_k pp_k for every shift k; then, when `update`,
// pp_k = z_k r + d_k pp_k and p = r + beta p.  x and pp hold the n shift
// fields back to back (24 * spad(G) doubles each); cf[4k + 0..3] = (c_k, z_k,
// d_k, active_k): shifts with active_k == 0 are left as they are
void blas_mshift(const Geom& G, double* x, double* pp, int n, const double* r, double* p,
                 double beta, const double* cf, bool update, cudaStream_t st);
// BQCD-format arrays (already on the device) <-> planes, bqcd.cu.  map:
// device array of each natural site's BQCD slot (i-1 + volh*eo), or null for
// the default numbering; spinors: the even array followed by the odd one
template <typename R>
void bqcd_to_planes_gauge(const Geom& G, R* dst, const double* u, const int* map, cudaStream_t st);
template <typename R>
void bqcd_to_planes_clover(const Geom& G, R* dst, const double* c, const int* map,
                           cudaStream_t st);
template <typename R>
void bqcd_to_planes_spinor(const Geom& G, R* dst, const double* both, const int* map, int rhs,
                           cudaStream_t st);
template <typename R>
void planes_to_bqcd_spinor(const Geom& G, double* both, const R* src, const int* map, int rhs,
                           cudaStream_t st);
// 12-real FP32 links: worst deviation of the FP32 links from SU(3)
// (max over sites and directions of |U U^+ - 1| and |det U - 1|, into *dev
// as float bits) and the compressed copy (first two rows)
void links_su3_deviation(const Geom& G, const float* Us, unsigned* dev, cudaStream_t st);
void links_compress12(const Geom& G, float* U12, const float* Us, cudaStream_t st);
// FP32 planes <-> FP16 planes with per-site scales (IO<H16> format)
void spinor_s2h(const Geom& G, __half* dst, const float* src, cudaStream_t st);
void spinor_h2s(const Geom& G, float* dst, const __half* src, cudaStream_t st);
void spinor_h2h(const Geom& G, __half* dst, const __half* src, cudaStream_t st);
// FP16 copies of the FP32 gauge (9 complex planes per mu) and clover planes
void fields_s2h(const Geom& G, __half* Uh, const float* Us, __half* Ch, const float* Cs,
                cudaStream_t st);
// FP16 copy of per-RHS FP32 clover planes (entries of a multi-RHS handle)
void clover_s2h_entries(const Geom& G, __half* Ch, const float* Cs, cudaStream_t st);
// Device-side scalars of the flexible inner BiCGStab of one right-hand side
// (bicgstab_precdd_s_h.cc:83-369): the loop's reductions land in res, a
// one-thread kernel turns them into the next update's coefficients, kept
// in cf in the layout the update kernels read as a per-RHS table (alpha at
// 0-1, omega at 4-5, beta and omega of the p update at 8-11), and decides
// convergence, so the host reads back one small record per half iteration
// instead of every reduction.  done: converged (or b = 0) -- the remaining
// updates of the iteration use zero coefficients; iters: the iteration the
// residual fell below tol; bad: a non-finite residual.
struct InnerScalars {
  double cf[12];
  float bnorm, rnorm, rho0r, rho0i, ar, ai, wr, wi;
  int done, iters, bad, iter;
};
// phase 0: after r = b (res[0] = |b|^2); 1: after <r0, q>; 2: after the alpha
// update (res[0] = |r|^2); 3: after |t|^2, <t, r>; 4: after the omega update
// (|r|^2, <r0, r>), which also sets beta
void inner_scalars(InnerScalars* s, const double* res, int phase, double tol, cudaStream_t st);
inline double* inner_coefs(InnerScalars* s, int k) {  // device address of cf + k
  return reinterpret_cast<double*>(reinterpret_cast<char*>(s) + offsetof(InnerScalars, cf)) + k;
}

// y = (float)(x * s)   /   y = (double)x * s   (cf: per-RHS s, cf[4*rhs])
void blas_d2s(const Geom& G, float* y, const double* x, double s, cudaStream_t st,
              const double* cf = nullptr);
void blas_s2d(const Geom& G, double* y, const float* x, double s, cudaStream_t st,
              const double* cf = nullptr);

// ---------------------------------------------------------------------------
// layout conversion: QWS host layout (lane width vlen) <-> device planes.
// The QWS array covers the whole (single-rank) lattice: two x-half domains.
// ---------------------------------------------------------------------------
template <typename R>
void qws_to_planes_spinor(const Geom& G, R* dst, const R* qws, int vlen, int site0, int n,
                          cudaStream_t st);
template <typename R>
void planes_to_qws_spinor(const Geom& G, R* qws, const R* src, int vlen, int site0, int n,
                          cudaStream_t st);
// eo = true reads the arrays the way the even-odd operators do: parity p of
// site (x,y,z,t) selects the x-half slot, x/2 the position inside it.
template <typename R>
void qws_to_planes_gauge(const Geom& G, R* dst, const R* qws, int vlen, cudaStream_t st,
                         bool eo = false);
template <typename R>
void qws_to_planes_clover(const Geom& G, R* dst, const R* qws, int vlen, cudaStream_t st,
                          bool eo = false);
// one-parity half arrays of the even-odd operators (vol elements, x/2 compressed)
// <-> full planes; the upload zeroes the other parity, the download writes
// parity p only
template <typename R>
void qws_eo_to_planes_spinor(const Geom& G, R* dst, const R* qws_half, int vlen, int p,
                             cudaStream_t st);
template <typename R>
void planes_to_qws_eo_spinor(const Geom& G, R* qws_half, const R* src, int vlen, int p,
                             cudaStream_t st);
// natural layout (site = x + Lx*(y + Ly*(z + Lz*t))) <-> device planes;
// rhs selects one right-hand side of a multi-RHS field
template <typename R>
void nat_to_planes_spinor(const Geom& G, R* dst, const R* nat, cudaStream_t st, int rhs = 0);
template <typename R>
void planes_to_nat_spinor(const Geom& G, R* nat, const R* src, cudaStream_t st, int rhs = 0);
template <typename Rin, typename R>
void nat_to_planes_gauge(const Geom& G, R* dst, const Rin* nat, cudaStream_t st);
template <typename Rin, typename R>
void nat_to_planes_clover(const Geom& G, R* dst, const Rin* nat, cudaStream_t st);

}  // namespace qwsg
