// Group solves: the precision form's DD solve (bicgstab_dd_mix2_hf) of
// several lattices of any volumes -- each with its own fields, kappa,
// tolerance and block grid -- with each kernel step run as ONE launch over
// all of them.  No counterpart in the reference, whose bicgstab_dd_mix2_hf_
// (bicgstab_dd_mix2_hf.cc:110-373) solves one lattice per call.
//
// Each member lattice runs the unchanged one-lattice solver on a host thread
// of its own, with its launches recorded (kernels.h) instead of issued.
// Every point where that solver reads a result back (Ctx::fetch,
// Ctx::fetch_inner) parks the thread.  When every member is parked, the
// coordinator merges the recorded launches: members whose sequences of
// launches are the same (the common case: the same step of the same
// algorithm) get one launch per position in the sequence, over all of them;
// members at a different step form their own merged sequence.  It then
// copies every parked member's read-back, waits for the stream, and
// releases the members.  A merged kernel runs, for each member, the blocks
// of that member's own launch with its own arguments, so every member's
// results are bitwise those of its own solve; what changes is that the small
// lattices no longer pay a launch, and a half-empty GPU, each.
#include <chrono>
#include <condition_variable>
#include <map>
#include <mutex>
#include <thread>

#include "ctx.h"

namespace qwsg {

thread_local GroupRecorder* g_group_rec = nullptr;

void group_unrecorded_launch() {
  throw Error(3, "group solve: a launch that cannot be merged across lattices "
                 "(multi-RHS handles, per-RHS kappa and buffer allocation inside the solve "
                 "are not supported)");
}

struct GroupState {
  std::mutex m;
  std::condition_variable cv_coord, cv_work;
  int n_live = 0, n_parked = 0;
  bool abort = false;
};

using GroupSig = std::vector<GroupMergeFn>;

struct GroupMember {
  GroupState* g = nullptr;
  Ctx* c = nullptr;
  GroupRecorder rec;
  // the read-back this member waits for (none when bytes == 0)
  const void* rb_dev = nullptr;
  void* rb_host = nullptr;
  size_t rb_bytes = 0;
  bool finished = false, left = false;
  long go = 0;        // incremented by the coordinator to release the member
  bool ran = false;   // its launches ran in the last round
  int held = 0;       // rounds it has been held back in a row
  GroupSig last_sig;  // the launch sequence it ran last
  // device addresses of the lattice's page-locked read-back buffers (null:
  // not mapped, read back with a copy call)
  void* h_res_dev = nullptr;
  void* h_isc_dev = nullptr;
};

// called by a member's solver thread at a read-back: hand over the
// recorded launches and wait until the coordinator has run them and copied
// the result
void group_park(GroupMember& me, const void* dev, void* host, size_t bytes) {
  GroupState& g = *me.g;
  std::unique_lock<std::mutex> lk(g.m);
  me.rb_dev = dev;
  me.rb_host = host;
  me.rb_bytes = bytes;
  const long go = me.go;
  g.n_parked++;
  g.cv_coord.notify_one();
  g.cv_work.wait(lk, [&] { return me.go != go || g.abort; });
  if (g.abort) throw Error(3, "group solve aborted");
}

namespace {

void member_thread(GroupMember& me, GroupItem& it, int device) {
  cudaSetDevice(device);
  g_group_rec = &me.rec;
  try {
    bicgstab_dd_mix2_hf(*me.c, it.x, it.b, it.tol, it.maxiter, it.tol_s, it.maxiter_s, it.nsap,
                        it.nm, it.reliable, &it.stats);
    it.status = 0;
  } catch (const Error& e) {
    it.status = e.code;
    it.error = e.what();
    me.rec.recs.clear();  // an unfinished step of a failed solve
  } catch (const std::exception& e) {
    it.status = 3;
    it.error = e.what();
    me.rec.recs.clear();
  }
  g_group_rec = nullptr;
  // the last launches (after its last read-back) still run in the next round
  std::lock_guard<std::mutex> lk(me.g->m);
  me.rb_bytes = 0;
  me.finished = true;
  me.g->n_parked++;
  me.g->cv_coord.notify_one();
}

// the read-backs of one round in one launch: block l copies member l's
// result words into its page-locked host buffer (reachable from the device
// through unified addressing), in place of one copy call per member
struct Readback {
  const unsigned long long* src;
  unsigned long long* dst;
  int words;
  int pad_;
};
__global__ void k_group_readback(const Readback* __restrict__ rb) {
  const Readback r = rb[blockIdx.x];
  for (int k = threadIdx.x; k < r.words; k += blockDim.x) r.dst[k] = r.src[k];
}

// page-locked and device staging of one round's argument tables
struct Staging {
  unsigned char* host = nullptr;
  unsigned char* dev = nullptr;
  size_t cap = 0;
  ~Staging() {
    if (host) cudaFreeHost(host);
    if (dev) cudaFree(dev);
  }
  void reserve(size_t n) {  // (the stream is idle between rounds)
    if (n <= cap) return;
    size_t c = cap ? cap : (size_t)1 << 20;
    while (c < n) c *= 2;
    if (host) cudaFreeHost(host);
    if (dev) cudaFree(dev);
    host = nullptr;
    dev = nullptr;
    cap = 0;
    QWSG_CUDA(cudaMallocHost(&host, c));
    QWSG_CUDA(cudaMalloc(&dev, c));
    cap = c;
  }
};

// One round: the parked members, grouped by the launch sequence they
// recorded, merge and run -- except a group held back one round so that
// another group catches up with it.  The coordinator learns which sequence
// follows which (the two halves of an inner iteration alternate, say);
// when group A's next sequence is group B's current one, B waits one round
// and A's members arrive at B's step, after which both merge.  The smaller
// of the two waits, and no member waits two rounds in a row.  Returns the
// merged launches issued; marks in `ran` the members to release.
static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

long run_round(std::vector<GroupMember>& mem, std::map<GroupSig, GroupSig>& next, Staging& stg,
               cudaStream_t st, long* member_launches, double* t) {
  Region region_("group_round");
  const double t0 = now_s();
  std::map<GroupSig, std::vector<int>> sigs;
  std::vector<GroupSig> cur(mem.size());
  for (int l = 0; l < (int)mem.size(); l++) {
    GroupMember& m = mem[l];
    if (m.left) continue;
    cur[l].reserve(m.rec.recs.size());
    for (const auto& r : m.rec.recs) cur[l].push_back(r.merge);
    if (m.ran && !m.last_sig.empty() && !cur[l].empty()) next[m.last_sig] = cur[l];
    sigs[cur[l]].push_back(l);
  }
  struct Grp {
    const GroupSig* sig;
    std::vector<int>* ls;
    bool held;
    bool may_hold;
  };
  std::vector<Grp> grps;
  for (auto& s : sigs) {
    bool may = !s.first.empty();
    for (int l : s.second) may = may && !mem[l].finished && mem[l].held == 0;
    grps.push_back({&s.first, &s.second, false, may});
  }
  std::stable_sort(grps.begin(), grps.end(),
                   [](const Grp& a, const Grp& b) { return a.ls->size() > b.ls->size(); });
  for (size_t i = 0; i < grps.size(); i++) {
    if (grps[i].held) continue;
    auto it = next.find(*grps[i].sig);
    if (it == next.end()) continue;
    for (size_t j = i + 1; j < grps.size(); j++)
      if (!grps[j].held && grps[j].may_hold && *grps[j].sig == it->second) grps[j].held = true;
  }
  GroupBatch b;
  std::vector<const GroupRec*> recs;
  for (auto& gr : grps) {
    for (int l : *gr.ls) {
      mem[l].ran = !gr.held;
      mem[l].held = gr.held ? mem[l].held + 1 : 0;
    }
    if (gr.held) continue;
    for (size_t i = 0; i < gr.sig->size(); i++) {
      recs.clear();
      for (int l : *gr.ls) recs.push_back(&mem[l].rec.recs[i]);
      (*gr.sig)[i](recs.data(), (int)recs.size(), b);
    }
    *member_launches += (long)(gr.sig->size() * gr.ls->size());
  }
  std::vector<Readback> rbs;
  std::vector<GroupMember*> copies;
  for (auto& m : mem)
    if (!m.left && m.ran && !m.finished && m.rb_bytes) {
      void* dst = m.rb_host == m.c->h_res ? m.h_res_dev
                  : m.rb_host == m.c->h_isc ? m.h_isc_dev : nullptr;
      if (dst && m.rb_bytes % 8 == 0)
        rbs.push_back({static_cast<const unsigned long long*>(m.rb_dev),
                       static_cast<unsigned long long*>(dst), (int)(m.rb_bytes / 8), 0});
      else
        copies.push_back(&m);
    }
  if (!rbs.empty()) {
    const size_t off = b.put(rbs.data(), sizeof(Readback) * rbs.size());
    const int nrb = (int)rbs.size();
    b.launches.push_back([=](const unsigned char* dev, cudaStream_t s2) {
      count_launch();
      k_group_readback<<<nrb, 32, 0, s2>>>(reinterpret_cast<const Readback*>(dev + off));
    });
  }
  const double t1 = now_s();
  if (!b.launches.empty()) {
    stg.reserve(b.host.size());
    std::memcpy(stg.host, b.host.data(), b.host.size());
    QWSG_CUDA(cudaMemcpyAsync(stg.dev, stg.host, b.host.size(), cudaMemcpyHostToDevice, st));
    for (auto& f : b.launches) f(stg.dev, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw Error(3, std::string("group solve launch: ") + cudaGetErrorString(e));
  }
  for (GroupMember* m : copies)
    QWSG_CUDA(cudaMemcpyAsync(m->rb_host, m->rb_dev, m->rb_bytes, cudaMemcpyDeviceToHost, st));
  for (int l = 0; l < (int)mem.size(); l++) {
    GroupMember& m = mem[l];
    if (m.left || !m.ran) continue;
    m.rec.recs.clear();
    m.last_sig = std::move(cur[l]);
  }
  const double t2 = now_s();
  QWSG_CUDA(cudaStreamSynchronize(st));
  t[0] += t1 - t0;
  t[1] += t2 - t1;
  t[2] += now_s() - t2;
  return (long)b.launches.size();
}

}  // namespace

void group_bicgstab_dd_mix2_hf(std::vector<GroupItem>& items, cudaStream_t st, GroupStats* gs) {
  Region region_("group_bicgstab_dd_mix2_hf");
  const int n = (int)items.size();
  if (n == 0) return;
  for (int i = 0; i < n; i++) {
    Ctx* c = items[i].c;
    if (c->G.nr != 1 || !c->rhs_kappas.empty())
      throw Error(1, "group solve: every lattice must be a one-RHS handle with one kappa");
    if (items[i].nsap > 10 || items[i].nm > 10)
      throw Error(2, "assign_mult_mSAP_s_h_: nsap and nm must be <= 10 (prec_ddd_s_h.h:100-101)");
    for (int j = 0; j < i; j++)
      if (items[j].c == c) throw Error(1, "group solve: a lattice appears twice");
  }
  // everything the solve would allocate or build on first use, now (a
  // launch inside the recorded solve must be one the group can merge)
  for (int i = 0; i < n; i++) {
    Ctx& c = *items[i].c;
    c.ensure_outer();
    c.ensure_hp();
    c.ensure_face_lists();
    c.ensure_links12();
    c.check_launch("group solve set-up");
    QWSG_CUDA(cudaStreamSynchronize(c.st));
  }
  int device = 0;
  QWSG_CUDA(cudaGetDevice(&device));
  GroupState g;
  std::vector<GroupMember> mem(n);
  std::vector<bool> timing(n);
  // the lattices leave group mode on every way out
  auto restore = [&] {
    for (int i = 0; i < n; i++) {
      items[i].c->gm = nullptr;
      items[i].c->timing = timing[i];
    }
  };
  for (int i = 0; i < n; i++) {
    timing[i] = items[i].c->timing;
    items[i].c->timing = false;
    items[i].status = -1;
    items[i].error.clear();
    mem[i].g = &g;
    mem[i].c = items[i].c;
    items[i].c->gm = &mem[i];
    // (page-locked memory is mapped for the device under unified addressing;
    // where it is not, the read-backs fall back to copies)
    if (cudaHostGetDevicePointer(&mem[i].h_res_dev, items[i].c->h_res, 0) != cudaSuccess)
      mem[i].h_res_dev = nullptr;
    if (cudaHostGetDevicePointer(&mem[i].h_isc_dev, items[i].c->h_isc, 0) != cudaSuccess)
      mem[i].h_isc_dev = nullptr;
    (void)cudaGetLastError();
  }
  g.n_live = n;
  Staging stg;
  std::map<GroupSig, GroupSig> next;
  long rounds = 0, merged = 0, member_launches = 0;
  double t_round[3] = {0, 0, 0}, t_wait = 0;
  std::vector<std::thread> th;
  try {
    th.reserve(n);
    for (int i = 0; i < n; i++)
      th.emplace_back(member_thread, std::ref(mem[i]), std::ref(items[i]), device);
  } catch (...) {  // the threads that started unwind at their first read-back
    {
      std::lock_guard<std::mutex> lk(g.m);
      g.abort = true;
    }
    g.cv_work.notify_all();
    for (auto& t : th) t.join();
    restore();
    cudaStreamSynchronize(st);
    throw Error(3, "group solve: could not start a thread per lattice");
  }
  std::string fail;
  {
    std::unique_lock<std::mutex> lk(g.m);
    while (g.n_live > 0) {
      const double w0 = now_s();
      g.cv_coord.wait(lk, [&] { return g.n_parked == g.n_live; });
      t_wait += now_s() - w0;
      // every live member is parked: their state is ours until released
      lk.unlock();
      try {
        merged += run_round(mem, next, stg, st, &member_launches, t_round);
      } catch (const std::exception& e) {
        fail = e.what();
      }
      rounds++;
      lk.lock();
      // release the members that ran (a finished one leaves the group)
      for (auto& m : mem) {
        if (m.left || !m.ran) continue;
        g.n_parked--;
        if (m.finished) {
          m.left = true;
          g.n_live--;
        } else {
          m.go++;
        }
      }
      if (!fail.empty()) g.abort = true;
      g.cv_work.notify_all();
      if (g.abort) {
        // the members unwind (their parks throw) and finish
        g.cv_coord.wait(lk, [&] {
          int live = 0;
          for (auto& m : mem) live += !m.finished;
          return live == 0;
        });
        break;
      }
    }
  }
  for (auto& t : th) t.join();
  restore();
  if (gs) {
    gs->rounds = rounds;
    gs->merged_launches = merged;
    gs->member_launches = member_launches;
    gs->t_members = t_wait;
    gs->t_merge = t_round[0];
    gs->t_launch = t_round[1];
    gs->t_gpu_wait = t_round[2];
  }
  if (!fail.empty()) {
    cudaStreamSynchronize(st);
    throw Error(3, "group solve: " + fail);
  }
}

}  // namespace qwsg
