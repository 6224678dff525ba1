"""Continuous-batching solve service on one GPU.

Requests (gauge field, kappa, csw, source, tolerance) arrive at any time.
The service keeps gauge fields resident on the device, builds each
request's clover term there (qwsg_build_clover), admits work against an
HBM budget, merges compatible pending requests -- same lattice, gauge
field and csw; each keeps its own kappa, whose clover term is built on the
GPU for its RHS (qwsg_batch_set_kappas), and its own tolerance, at which its
RHS stops (qwsg_batch_set_tols) -- into one multi-RHS solve
(qwsg_create_batch), and runs several solves at once on separate CUDA
streams, so requests that arrive while others are on the GPU start as soon
as a worker slot and memory are free.  Requests for a field that is busy
wait for its running solve and join the next batch on it together with
every compatible request that arrived meanwhile.  Every result carries its
own latency (completion minus arrival); `summarize` gives p50/p99 and
solves/s.

Failures are reported on the request (`error`), never by the service
stopping: a request that cannot fit the HBM budget fails at once
(MemoryError); one whose `deadline_s` passes before it starts fails with
DeadlineExceeded; `Service.cancel` withdraws a request that has not started
(Cancelled); a solver error -- a non-finite residual from a NaN or infinite
source, say -- fails the requests of that solve, and the field and the
service stay usable.

The solver is the precision form (bicgstab_dd_mix2_hf: FP64 outer with
reliable restarts, flexible FP32 inner, FP16-storage SAP).  A request's
result does not depend on what it was merged or overlapped with beyond the
solve tolerance: per-RHS scalars and convergence in the batch, and each
resident field is held by one job at a time.

    python -m qws_b200.serve --rate 20 --window 10
"""
from __future__ import annotations

import argparse
import itertools
import json
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

# bytes per padded site of the pieces a job holds on the device
_FIELD_BYTES = 72 * (8 + 4 + 2) * 2 + 4 * 12 * 4  # gauge + clover, FP64/FP32/FP16
#                                                   copies; 12-real FP32 links
_WORK_BYTES_PER_RHS = (6 * 192      # FP64 outer work spinors
                       + 9 * 96     # FP32: inner solver 5, approximate inverse 3, flexible w
                       + 4 * 52     # FP16-storage SAP spinors
                       + 3 * 96     # FP32 SAP buffers (when the FP32 SAP runs on the handle)
                       + 3 * 192)   # the job's x and b, and the library's staging buffer
_HANDLE_BYTES = 16 << 20            # reduction and coefficient buffers, face lists


def _pad(V):
    return (V + 127) // 128 * 128


def field_bytes(L):
    return _FIELD_BYTES * _pad(int(np.prod(L)))


_RHS_CLOVER_BYTES = 72 * (8 + 4 + 2)  # per-RHS clover planes of a merged solve


def work_bytes(L, nr):
    """device bytes of an nr-RHS work handle on lattice L: the solver's work
    spinors, the job's own x and b (kept on the handle, so they are counted
    here and not left in torch's cache), the library's staging buffer, the
    per-RHS clover planes of a merged solve, and the handle's small buffers"""
    per = _WORK_BYTES_PER_RHS + (_RHS_CLOVER_BYTES if nr > 1 else 0)
    return per * _pad(int(np.prod(L))) * nr + _HANDLE_BYTES


def stream_priority(L):
    """CUDA stream priority of the jobs on a lattice of extents L: one level
    higher for every factor 4 of volume below 2^24 sites (at most 3 levels),
    so that when several solves share the GPU the block scheduler serves
    the short ones first and their latency does not queue behind the
    kernels of a large lattice (a lower number is a higher priority)."""
    V = int(np.prod(L))
    level = 0
    while level < 3 and V * 4 ** (level + 1) <= 1 << 24:
        level += 1
    return -level


@dataclass
class Request:
    L: tuple
    gauge: int
    kappa: float
    csw: float
    tol: float
    source: np.ndarray            # natural layout [V, 24] FP64 (page-locked: faster upload)
    # where the solution goes: None -> a new host array; or a C-contiguous
    # FP64 [V, 24] array of the caller's (page-locked: faster download)
    out: np.ndarray | None = None
    # the request fails with DeadlineExceeded if it has not started this many
    # seconds after it arrived (None: no deadline)
    deadline_s: float | None = None
    rid: int = -1
    t_arrival: float = 0.0
    # filled in by the service
    x: np.ndarray | None = None
    stats: dict | None = None
    t_start: float = 0.0
    t_done: float = 0.0
    # phases of the job that ran it (s): field made resident (0 if it was),
    # clover terms, host->device + solve + device->host
    t_resident: float = 0.0
    t_clover: float = 0.0
    t_solve: float = 0.0
    batch: int = 0
    group: int = 0                # requests in the group solve that ran it (1: alone)
    error: str | None = None
    done: threading.Event = field(default_factory=threading.Event)

    def key(self):
        """Requests with the same key merge into one multi-RHS solve (each
        keeps its own kappa, per-RHS clover terms, qwsg_batch_set_kappas, and
        its own tolerance, qwsg_batch_set_tols)."""
        return (self.L, self.gauge, self.csw)

    def wait(self, timeout):
        """Block until the request is finished; TimeoutError after `timeout` s."""
        if not self.done.wait(timeout):
            raise TimeoutError(f"request {self.rid} not finished after {timeout} s")
        return self

    @property
    def latency(self):
        return self.t_done - self.t_arrival


class _Resident:
    """One gauge field on the device (a Lattice), with the clover term of the
    kappa/csw it was last built for.  Held by one job at a time."""

    def __init__(self, L, gauge_id, U, NB, hop_threads=128, graphs=True):
        import torch

        import qws_b200

        self.L, self.gid = L, gauge_id
        # (kappa is set per job; a merged job's kernels take only its sign)
        self.lat = qws_b200.Lattice(L, NB, tbc=-1, kappa=0.125)
        # a stream of its own (torch's streams are pooled and shared)
        self.stream = self.lat.use_own_stream(stream_priority(L))
        self.lat.set_hop_threads(hop_threads)
        self.lat.set_graphs(graphs)
        self.graphs = graphs
        if isinstance(U, dict):  # {"seed", "n_smear", "alpha"}: generate on the device
            self.plaquette = self.lat.gen_gauge_device(U["seed"], U["n_smear"], U["alpha"])
        else:
            self.lat.load_gauge(U)
        self.clover_key = None
        self.busy = False
        self.bytes = field_bytes(L)
        self.work = {}  # nrhs -> BatchLattice on this field
        self.last_used = time.monotonic()

    def prepare(self, kappa, csw):
        if self.clover_key != (kappa, csw):
            self.lat.set_kappa(kappa)
            self.lat.build_clover(csw)
            self.clover_key = (kappa, csw)

    def close(self):
        for w in self.work.values():
            close_work(w)
        self.work.clear()
        self.lat.close()


def close_work(w):
    """Free a work handle and its job buffers, and give torch's cached blocks
    back to the device so the library's own allocations can use them."""
    import torch

    w.job_b = w.job_x = None
    w.close()
    torch.cuda.empty_cache()


class _Placeholder:
    """Reserved slot for a field that a worker is about to make resident."""

    def __init__(self, L, gid):
        self.L, self.gid = L, gid
        self.lat = None
        self.busy = True
        self.work = {}
        self.bytes = field_bytes(L)
        self.last_used = time.monotonic()

    def close(self):
        pass


class Service:
    """The request loop.  gauge_source(L, gauge_id) -> host gauge field
    [4, V, 18] FP64, or {"seed", "n_smear", "alpha"} to generate it on the
    device (called each time the field is made resident)."""

    def __init__(self, gauge_source, budget_bytes=150e9, workers=3, max_batch=16,
                 block_grid=None, maxiter=100, tol_s=1e-6, maxiter_s=50, nsap=None, nm=None,
                 reliable=5, graphs=True, lifo_after_s=None, group=1, group_max_sites=None):
        self.gauge_source = gauge_source
        # group > 1: a worker takes up to this many one-request jobs (any
        # volumes) at once and runs them as one group solve, every kernel
        # step one launch over all of them (qws_b200.group_solve); merging
        # into multi-RHS solves is then off (max_batch 1)
        self.group = max(1, int(group))
        # only lattices of at most this many sites join a group; a larger one
        # (whose own launches fill the GPU) runs alone on its worker's stream
        # while a group runs beside it (None: every lattice joins)
        self.group_max_sites = float("inf") if group_max_sites is None else int(group_max_sites)
        if self.group > 1:
            max_batch = 1
        self.group_rounds = 0
        self.group_launches = [0, 0]  # launches issued, launches the solves alone would issue
        self.group_phase_s = [0.0, 0.0, 0.0]  # jobs' set-up, group solve, jobs' results
        # inside the group solves: host time per activity (qwsg_group_stats)
        self.group_host_s = dict.fromkeys(("t_members", "t_merge", "t_launch", "t_gpu_wait"), 0.0)
        # adaptive LIFO: once the oldest pending request has waited longer
        # than this (s), the newest pending requests are served first -- under
        # overload the oldest are the ones a deadline sheds, and serving them
        # first would make every served request wait about as long (None:
        # always in arrival order)
        self.lifo_after_s = lifo_after_s
        # CUDA graphs of the SAP sequences are captured per (buffers, kappa);
        # they pay off when requests repeat a kappa
        self.graphs = bool(graphs)
        self.budget = float(budget_bytes)
        self.max_batch = int(max_batch)
        # SAP block grid / sweep counts / CTA size per volume: as given, else
        # the autotuner's cached choice for this GPU, else the reference's
        # one-rank partition with (nsap, nm) = (4, 2)
        self.fixed = {"NB": block_grid, "nsap": nsap, "nm": nm}
        self.configs = {}
        self.solver = dict(maxiter=maxiter, tol_s=tol_s, maxiter_s=maxiter_s, reliable=reliable)
        self.pending = []                 # requests not yet started, arrival order
        self.cv = threading.Condition()
        self.residents = {}               # (L, gid) -> _Resident or _Placeholder
        self.used = 0.0                   # bytes held by residents and work handles
        self.jobs = queue.Queue()
        self.idle_workers = int(workers)
        self.ids = itertools.count()
        self.completed = []
        self.merged = 0
        self.evicted = 0                  # resident fields freed for others
        self.handles_moved = 0            # work handles taken over by another field
        self.stall_s = 5.0                # see _stalled
        self.failed = None                # set when the scheduler had to stop
        self._stall_since = None
        self.stop = False
        self.workers = [threading.Thread(target=self._worker, daemon=True) for _ in range(workers)]
        for t in self.workers:
            t.start()
        self.sched = threading.Thread(target=self._scheduler, daemon=True)
        self.sched.start()

    def config(self, L):
        """Launch configuration of volume L (block grid, nsap, nm, hop threads)."""
        c = self.configs.get(L)
        if c is None:
            from . import autotune

            hit = autotune.lookup(L, "hf", 1) or {}
            c = {"NB": tuple(hit.get("NB", autotune.REFERENCE_NB)), "nsap": hit.get("nsap", 4),
                 "nm": hit.get("nm", 2), "hop_threads": hit.get("hop_threads", 128),
                 "tuned": bool(hit)}
            for k, v in self.fixed.items():
                if v is not None:
                    c[k] = tuple(v) if k == "NB" else v
            self.configs[L] = c
        return c

    # ---- client side -----------------------------------------------------------
    def submit(self, req: Request) -> Request:
        req.rid = next(self.ids)
        req.t_arrival = time.monotonic()
        with self.cv:
            self.pending.append(req)
            if self.failed:
                self._reject(req, self.failed)
            self.cv.notify_all()
        return req

    def submit_all(self, reqs) -> list:
        """Submit several requests at once: the scheduler sees them together
        (a group service then starts them as one group)."""
        with self.cv:
            for req in reqs:
                req.rid = next(self.ids)
                req.t_arrival = time.monotonic()
                self.pending.append(req)
                if self.failed:
                    self._reject(req, self.failed)
            self.cv.notify_all()
        return list(reqs)

    def cancel(self, req: Request) -> bool:
        """Withdraw a request that has not started: it finishes at once with
        error "Cancelled".  False if it has started (a running solve is not
        interrupted) or is already finished."""
        with self.cv:
            if req in self.pending:
                self._reject(req, "Cancelled")
                self.cv.notify_all()
                return True
            return False

    def close(self):
        with self.cv:
            self.stop = True
            self.cv.notify_all()
        self.sched.join()
        for _ in self.workers:
            self.jobs.put(None)
        for t in self.workers:
            t.join()
        for r in self.residents.values():
            r.close()
        self.residents.clear()
        import torch

        torch.cuda.empty_cache()  # the result buffers' blocks cached per stream

    # ---- scheduling ------------------------------------------------------------
    def _idle(self, keep=None):
        keep = keep if isinstance(keep, tuple) else (keep,)
        return sorted((r for r in self.residents.values()
                       if not r.busy and r.lat is not None and all(r is not k for k in keep)),
                      key=lambda r: r.last_used)

    def _donor(self, L, nr, exclude=None):
        """An idle resident field of volume L holding a work handle of nr RHS
        that a job on another field of that volume can take over
        (qwsg_batch_set_parent), least recently used first."""
        for r in self._idle(exclude):
            if r.L == L and nr in r.work:
                return r
        return None

    def _evict(self, need, keep=None):
        """Free idle work handles, then idle resident fields (least recently
        used first; never `keep`) until `need` more bytes fit the budget.
        Frees nothing when even all of that would not make room.  Called with
        cv held."""
        if self.used + need <= self.budget:
            return True
        idle = self._idle(keep)
        freeable = sum(r.bytes + sum(work_bytes(r.L, nr) for nr in r.work) for r in idle)
        if self.used - freeable + need > self.budget:
            return False
        for r in idle:
            for nr in list(r.work):
                if self.used + need <= self.budget:
                    return True
                close_work(r.work.pop(nr))
                self.used -= work_bytes(r.L, nr)
        for r in idle:
            if self.used + need <= self.budget:
                return True
            r.close()
            self.residents.pop((r.L, r.gid))
            self.used -= r.bytes
            self.evicted += 1
        return self.used + need <= self.budget

    def _expire(self):
        """Fail the pending requests whose deadline has passed (cv held)."""
        now = time.monotonic()
        for q in [q for q in self.pending
                  if q.deadline_s is not None and now - q.t_arrival > q.deadline_s]:
            self._reject(q, f"DeadlineExceeded: not started within {q.deadline_s} s")

    def _reject(self, q, why):
        self.pending.remove(q)
        q.error = why
        q.t_start = q.t_done = time.monotonic()
        self.completed.append(q)
        q.done.set()

    def _pick(self, accept=None):
        """The oldest request that can start now (and that `accept` takes,
        when given), with the compatible pending
        requests merged into its batch (a power of two, at most max_batch, and
        no larger than the memory allows).  Once a request waits for memory
        that only running jobs can give back, later requests start only if
        they fit the free budget without evicting anything: the idle memory
        the waiting request will need stays in place, and a short job that
        takes free memory gives it back when it ends.  A request that cannot
        fit the budget at all fails at once.  Called with cv held; reserves
        the memory and the resident field."""
        self._expire()
        tried = set()
        blocked = False
        order = list(self.pending)
        if (self.lifo_after_s is not None and order and
                time.monotonic() - order[0].t_arrival > self.lifo_after_s):
            order.reverse()
        for r in order:
            if r.key() in tried or (accept is not None and not accept(r)):
                continue
            tried.add(r.key())
            if field_bytes(r.L) + work_bytes(r.L, 1) > self.budget:
                self._reject(r, f"MemoryError: a {'x'.join(map(str, r.L))} solve needs "
                                f"{(field_bytes(r.L) + work_bytes(r.L, 1)) / 1e9:.1f} GB, "
                                f"over the {self.budget / 1e9:.1f} GB budget")
                continue
            res = self.residents.get((r.L, r.gauge))
            if res is not None and res.busy:
                continue
            group = [q for q in order if q.key() == r.key()]
            nr = 1
            while nr * 2 <= min(len(group), self.max_batch, 32):
                nr *= 2
            fit = None
            donor = None
            while fit is None and nr >= 1:
                have = res is not None and nr in res.work
                base = field_bytes(r.L) if res is None else 0
                fresh = base + work_bytes(r.L, nr)
                # new work buffers when they fit the free budget (a field
                # keeps its buffers, and their CUDA graphs, for its next
                # job); else the buffers of an idle field of the same volume
                # (they move to this field, their graphs updated to its
                # fields); if making room needs that field evicted, new
                # buffers after all
                if have:
                    options = [(base, None)]
                elif self.used + fresh <= self.budget:
                    options = [(fresh, None)]
                else:
                    d = self._donor(r.L, nr, exclude=res)
                    options = ([(base, d)] if d is not None else []) + [(fresh, None)]
                for need, d in options:
                    if need == 0 or self.used + need <= self.budget or \
                            (not blocked and self._evict(need, keep=(res, d))):
                        fit, donor = need, d
                        break
                if fit is None:
                    nr //= 2
            if fit is None:
                blocked = True
                continue
            group = group[:nr]
            self.used += fit
            if res is None:
                res = _Placeholder(r.L, r.gauge)
                self.residents[(r.L, r.gauge)] = res
            if donor is not None:
                res.work[nr] = donor.work.pop(nr)
                self.handles_moved += 1
            res.busy = True
            for q in group:
                self.pending.remove(q)
            if nr > 1:
                self.merged += nr - 1
            return res, group
        return None

    def _next_job(self):
        """The next job for an idle worker: (resident, requests), or with
        group > 1 a list of every such job that can start now, up to `group`
        of them, for one group solve.  Called with cv held."""
        job = self._pick()
        if job is None or self.group <= 1:
            return job
        small = lambda r: int(np.prod(r.L)) <= self.group_max_sites
        if not small(job[1][0]):
            return job  # a lattice that fills the GPU by itself: its own stream
        jobs = [job]
        while len(jobs) < self.group and self.pending:
            j = self._pick(accept=small)
            if j is None:
                break
            jobs.append(j)
        return jobs

    def _stalled(self, job, now):
        """Failure detection for admission: with every worker idle nothing
        can give memory back, so pending requests that still cannot start
        after `stall_s` never will -- fail them (AdmissionStalled) instead of
        leaving their callers waiting.  Called with cv held."""
        if job is not None or not self.pending or self.idle_workers < len(self.workers):
            self._stall_since = None
            return
        if self._stall_since is None:
            self._stall_since = now
        elif now - self._stall_since > self.stall_s:
            for q in list(self.pending):
                self._reject(q, "AdmissionStalled: no memory can be freed for it while "
                                "nothing runs")
            self._stall_since = None

    def _scheduler(self):
        with self.cv:
            while True:
                if self.stop and not self.pending:
                    return
                try:
                    if self.idle_workers == 0:
                        self._expire()
                    job = self._next_job() if self.idle_workers > 0 and self.pending else None
                    self._stalled(job, time.monotonic())
                except Exception as e:  # the scheduler cannot go on (a CUDA error, say)
                    self._fail_pending(f"ServiceFailed: {type(e).__name__}: {e}")
                    return
                if job is None:
                    self.cv.wait(0.02)
                    continue
                self.idle_workers -= 1
                self.jobs.put(job)

    def _fail_pending(self, why):
        """The scheduler stops: every pending request and every later one
        fails with `why` instead of leaving its caller waiting.  Called with
        cv held."""
        self.failed = why
        for q in list(self.pending):
            self._reject(q, why)

    # ---- execution -------------------------------------------------------------
    def _worker(self):
        while True:
            job = self.jobs.get()
            if job is None:
                return
            jobs = job if isinstance(job, list) else [job]
            try:
                if isinstance(job, list):
                    self._run_group(jobs)
                else:
                    self._run(*job)
            except Exception as e:  # reported on the requests, the service goes on
                for _, group in jobs:
                    for q in group:
                        if q.t_done == 0.0:
                            q.error = f"{type(e).__name__}: {e}"
                            q.t_done = time.monotonic()
            with self.cv:
                for res, group in jobs:
                    live = self.residents.get((res.L, res.gid))
                    if live is not None:
                        live.busy = False
                        live.last_used = time.monotonic()
                    for q in group:
                        self.completed.append(q)
                        q.done.set()
                self.idle_workers += 1
                self.cv.notify_all()

    def _run(self, res, group):
        p = self._stage(res, group)
        s = self.solver
        with self._torch.cuda.stream(p["B"].stream):
            p["stats"] = p["B"].bicgstab_dd_mix2_hf(
                p["xd"], p["bd"], max(q.tol for q in group), s["maxiter"], s["tol_s"],
                s["maxiter_s"], p["cfg"]["nsap"], p["cfg"]["nm"], reliable=s["reliable"])
        self._finish(p)

    def _run_group(self, jobs):
        """Several one-request jobs (any volumes) as one group solve
        (qws_b200.group_solve): each kernel step is one launch over all of
        them.  A request whose solve fails gets its error; the others finish."""
        import qws_b200

        def stage(job):
            res, group = job
            try:
                return self._stage(res, group)
            except Exception as e:
                for q in group:
                    q.error = f"{type(e).__name__}: {e}"
                    q.t_done = time.monotonic()
                return None

        # the jobs' own host work (field set-up, uploads; downloads) on a
        # pool of threads, as separate workers would do it
        t0 = time.monotonic()
        staged = [p for p in self._pool_map(stage, jobs) if p is not None]
        if not staged:
            return
        solves = [dict(lattice=p["B"], x=p["xd"], b=p["bd"], tol=p["group"][0].tol,
                       nsap=p["cfg"]["nsap"], nm=p["cfg"]["nm"], **self.solver) for p in staged]
        t1 = time.monotonic()
        st, gs = qws_b200.group_solve(solves, check=False)
        t2 = time.monotonic()
        self.group_rounds += gs["rounds"]
        self.group_launches[0] += gs["merged_launches"]
        self.group_launches[1] += gs["member_launches"]
        for k in self.group_host_s:
            self.group_host_s[k] += gs[k]
        done = []
        for p, s in zip(staged, st):
            if s["status"] != 0:
                for q in p["group"]:
                    q.error = f"QwsgError: solve failed in its group (qwsg error {s['status']})"
                    q.t_done = time.monotonic()
                continue
            p["stats"] = s
            p["group_size"] = len(staged)
            done.append(p)
        self._pool_map(self._finish, done)
        t3 = time.monotonic()
        for k, dt in enumerate((t1 - t0, t2 - t1, t3 - t2)):
            self.group_phase_s[k] += dt

    def _pool_map(self, fn, items):
        if len(items) <= 1:
            return [fn(x) for x in items]
        from concurrent.futures import ThreadPoolExecutor

        with ThreadPoolExecutor(max_workers=min(16, len(items))) as ex:
            return list(ex.map(fn, items))

    def _stage(self, res, group):
        """Make the field resident, build the clover term(s), take the work
        handle and upload the source(s): everything of a job before its solve."""
        import torch

        self._torch = torch
        t0 = time.monotonic()
        for q in group:
            q.t_start = t0
        cfg = self.config(res.L)
        made = isinstance(res, _Placeholder)
        if made:  # first use of this field: make it resident
            U = self.gauge_source(res.L, res.gid)
            live = _Resident(res.L, res.gid, U, cfg["NB"], cfg["hop_threads"], self.graphs)
            live.work = res.work  # a work handle taken over from another field
            live.busy = True
            with self.cv:
                self.residents[(res.L, res.gid)] = live
            res = live
            res.stream.synchronize()
        t1 = time.monotonic()
        r0 = group[0]
        nr = len(group)
        if nr == 1:
            res.prepare(r0.kappa, r0.csw)  # the field's own clover term
        B = res.work.get(nr)
        if B is not None and B.parent is not res.lat:  # taken over from another field
            B.set_parent(res.lat)
        if B is None:  # work buffers of an nr-RHS solve, kept for reuse
            # on a stream of its own: a handle that moves to another field
            # has nothing but its own work to wait for, and no other thread
            # launches into a stream whose graphs it captures
            B = res.lat.batch(nr)
            try:
                B.use_own_stream(stream_priority(res.L))
                B.set_graphs(self.graphs)
                with torch.cuda.stream(B.stream):
                    B.job_b, B.job_x = B.empty("f64"), B.empty("f64")
            except Exception:
                B.job_b = B.job_x = None
                B.close()
                raise
            res.work[nr] = B
        if nr > 1:  # every request its own kappa (per-RHS clover terms) and tolerance
            B.set_kappas([q.kappa for q in group], r0.csw)
            B.set_tols([q.tol for q in group])
        res.stream.synchronize()
        B.stream.synchronize()  # (per-RHS clover terms are built on the handle's stream)
        t2 = time.monotonic()
        with torch.cuda.stream(B.stream):
            S = np.ascontiguousarray(group[0].source, np.float64) if nr == 1 else None
            if S is None or not torch.from_numpy(S).is_pinned():
                # pageable (or several) sources: a multi-threaded copy into the
                # handle's page-locked buffer, from which the upload is a DMA
                P = getattr(B, "pinned_sources", None)
                if P is None:
                    shape = (B.V, 24) if nr == 1 else (nr, B.V, 24)
                    P = torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
                    B.pinned_sources = P
                if nr == 1:
                    torch.from_numpy(P).copy_(torch.from_numpy(S.reshape(P.shape)))
                else:
                    for k, q in enumerate(group):
                        torch.from_numpy(P[k]).copy_(torch.from_numpy(
                            np.ascontiguousarray(q.source, np.float64).reshape(P[k].shape)))
                S = P
            bd = B.to_device(S, out=B.job_b)
            xd = B.job_x
            xd.zero_()
        return {"res": res, "group": group, "cfg": cfg, "made": made, "B": B, "bd": bd,
                "xd": xd, "t0": t0, "t1": t1, "t2": t2, "group_size": 1}

    def _finish(self, p):
        """True residuals, download, per-request results of a solved job."""
        res, group, B, bd, xd = p["res"], p["group"], p["B"], p["bd"], p["xd"]
        nr = len(group)
        r0 = group[0]
        torch = self._torch
        with torch.cuda.stream(B.stream):
            per = B.batch_stats()[0] if nr > 1 else [p["stats"]]
            # the solver's own final true residual (reliable restarts
            # compute it), else one more D application
            if all(s.get("rel_resid_true", -1.0) >= 0 for s in per):
                truer = [s["rel_resid_true"] for s in per]
                truer = truer[0] if nr == 1 else truer
            else:
                truer = B.true_residual(xd, bd)
            if nr == 1 and r0.out is not None:
                X = B.to_host(xd, out=r0.out)
            else:
                # download into the handle's page-locked buffer (DMA), then
                # a multi-threaded copy into fresh host memory, which also
                # spreads the new pages' first-touch faults over the threads
                P = getattr(B, "pinned_result", None)
                if P is None:
                    shape = (B.V, 24) if nr == 1 else (nr, B.V, 24)
                    P = torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
                    B.pinned_result = P
                B.to_host(xd, out=P)
                X = np.empty_like(P)
                torch.from_numpy(X).copy_(torch.from_numpy(P))
        truer = [truer] if nr == 1 else truer
        t3 = time.monotonic()
        t0, t1, t2 = p["t0"], p["t1"], p["t2"]
        for k, q in enumerate(group):
            if nr > 1 and q.out is not None:
                q.out[...] = X[k]
            q.x = X if nr == 1 else (X[k] if q.out is None else q.out)
            q.stats = {"outer_iters": per[k]["outer_iters"], "true_rel_resid": truer[k],
                       "inner_iters": per[k]["inner_iters"]}
            q.batch = nr
            q.group = p["group_size"]
            q.t_resident, q.t_clover, q.t_solve = (t1 - t0) if p["made"] else 0.0, t2 - t1, t3 - t2
            q.t_done = t3


def summarize(reqs, t_begin=None, t_end=None):
    """p50/p99 latency (ms), solves/s over the span from the first arrival to
    the last completion, batch sizes and errors."""
    ok = [q for q in reqs if q.error is None and q.t_done > 0]
    kinds = {}
    for q in reqs:
        if q.error is not None:
            kinds[q.error[:160]] = kinds.get(q.error[:160], 0) + 1
    if not ok:
        return {"completed": 0, "errors": len(reqs), "error_kinds": kinds}
    lat = np.array([q.latency for q in ok]) * 1e3
    t0 = min(q.t_arrival for q in ok) if t_begin is None else t_begin
    t1 = max(q.t_done for q in ok) if t_end is None else t_end
    return {"completed": len(ok), "errors": len(reqs) - len(ok), "error_kinds": kinds,
            "solves_per_s": len(ok) / max(t1 - t0, 1e-9),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
            "mean_batch": float(np.mean([q.batch for q in ok])),
            # where the latency goes (p50 / p99 of each phase, ms)
            "phases_ms": {k: [round(float(np.percentile(v, 50)), 1), round(float(np.percentile(v, 99)), 1)]
                          for k, v in (("queue", [1e3 * (q.t_start - q.t_arrival) for q in ok]),
                                       ("resident", [1e3 * q.t_resident for q in ok]),
                                       ("clover", [1e3 * q.t_clover for q in ok]),
                                       ("solve", [1e3 * q.t_solve for q in ok]))},
            "requests_with_field_load": sum(q.t_resident > 0 for q in ok),
            # per lattice: requests, p50 latency, p50 of the solve phase (ms)
            "by_volume": {"x".join(map(str, L)): [
                len(v), round(float(np.percentile([q.latency * 1e3 for q in v], 50)), 1),
                round(float(np.percentile([q.t_solve * 1e3 for q in v], 50)), 1)]
                for L in sorted({q.L for q in ok}, key=lambda L: int(np.prod(L)))
                for v in [[q for q in ok if q.L == L]]},
            "max_true_rel_resid": max(q.stats["true_rel_resid"] for q in ok),
            "above_tol": sum(q.stats["true_rel_resid"] >= q.tol for q in ok)}


def seeded_gauge(seed0=1000, n_smear=5, alpha=0.36, device=True):
    """gauge_source for the service: seeded SU(3) + APE fields, one per
    (lattice, gauge id), generated on the device (or on the host)."""
    import qws_b200

    def make(L, gid):
        seed = seed0 + 7919 * gid + sum(L)
        if device:
            return {"seed": seed, "n_smear": n_smear, "alpha": alpha}
        U, _ = qws_b200.gen_gauge(L, seed, n_smear, alpha)
        return U
    return make


def poisson_workload(service, rate, window, volumes, weights, n_gauges, kappa_range=(0.130, 0.137),
                     csw=1.7, tols=(1e-8, 1e-10, 1e-12), seed=0, sources_per_volume=2,
                     deadline_s=None, scratch_out=False):
    """Poisson arrivals at `rate` per second for `window` seconds.  Each
    request draws a volume (with `weights`), a gauge id, kappa uniform in
    kappa_range, a tolerance and a Gaussian or point source.  Sources come from
    a small pool of page-locked host arrays made before the window opens, so
    the feeder keeps up with the arrival times.  scratch_out: every request
    of a volume writes its solution into one shared page-locked array that
    nobody reads (a load generator that keeps thousands of 48^3x96 solutions,
    2 GB each, would run the host out of memory; concurrent writes into it
    are harmless because the array is discarded).  Each result's true
    residual is computed on the device before the download either way.
    Returns the submitted requests (wait on req.done)."""
    import qws_b200

    import torch

    def pinned(a):  # the client's source in page-locked memory (DMA to the GPU)
        p = torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy()
        p[...] = a
        return p

    rng = np.random.default_rng(seed)
    sinks = {L: torch.empty((int(np.prod(L)), 24), dtype=torch.float64, pin_memory=True).numpy()
             for L in volumes} if scratch_out else {}
    pool = {}
    for L in volumes:
        pool[L] = [pinned(qws_b200.gen_source(L, 5000 + k, "gauss")) for k in range(sources_per_volume)]
        pool[L] += [pinned(qws_b200.gen_source(L, 0, "point", k)) for k in range(2)]
    t = 0.0
    arrivals = []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= window:
            break
        arrivals.append(t)
    p = np.asarray(weights, float) / np.sum(weights)
    reqs = []
    t0 = time.monotonic()
    for ta in arrivals:
        vi = rng.choice(len(volumes), p=p)
        L = tuple(volumes[vi])
        req = Request(L=L, gauge=int(rng.integers(n_gauges)),
                      kappa=float(rng.uniform(*kappa_range)), csw=csw,
                      tol=float(rng.choice(tols)), source=pool[L][int(rng.integers(len(pool[L])))],
                      deadline_s=deadline_s, out=sinks.get(L))
        delay = t0 + ta - time.monotonic()
        if delay > 0:
            time.sleep(delay)
        reqs.append(service.submit(req))
    return reqs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--window", type=float, default=10.0)
    ap.add_argument("--volumes", default="16x16x16x32,24x24x24x48,32x32x32x64,48x48x48x96")
    ap.add_argument("--weights", default="0.4,0.3,0.2,0.1")
    ap.add_argument("--gauges", type=int, default=4, help="resident gauge fields per volume")
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--workers", type=int, default=3)
    ap.add_argument("--max-batch", type=int, default=16)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--deadline", type=float, default=None,
                    help="a request not started this many seconds after arrival fails "
                         "(load shedding when the arrival rate exceeds what the GPU sustains)")
    ap.add_argument("--lifo-after", type=float, default=None,
                    help="serve the newest requests first once the oldest has waited this "
                         "long (default with --deadline: min(2 s, deadline/4); else never)")
    ap.add_argument("--warm", action="store_true",
                    help="make every (volume, gauge field) resident before the window opens")
    a = ap.parse_args()
    vols = [tuple(int(v) for v in s.split("x")) for s in a.volumes.split(",")]
    weights = [float(w) for w in a.weights.split(",")]
    svc = Service(seeded_gauge(), budget_bytes=a.budget_gb * 1e9, workers=a.workers,
                  max_batch=a.max_batch,
                  lifo_after_s=(a.lifo_after if a.lifo_after is not None else
                                (None if a.deadline is None else min(2.0, a.deadline / 4))))
    try:
        warm_s = 0.0
        if a.warm:
            import qws_b200

            t0 = time.monotonic()
            warm = [svc.submit(Request(L=L, gauge=g, kappa=0.1335, csw=1.7, tol=1e-8,
                                       source=qws_b200.gen_source(L, 4000 + g, "gauss")))
                    for L in vols for g in range(a.gauges)]
            for q in warm:
                q.wait(600)
            warm_s = time.monotonic() - t0
        merged0 = svc.merged
        t0 = time.monotonic()
        reqs = poisson_workload(svc, a.rate, a.window, vols, weights, a.gauges, seed=a.seed,
                                deadline_s=a.deadline, scratch_out=True)
        for q in reqs:
            q.wait(3600)
        out = summarize(reqs, t0, max(q.t_done for q in reqs))
        ok = [q for q in reqs if q.error is None]
        out.update({"rate": a.rate, "window_s": a.window, "requests": len(reqs),
                    "merged": svc.merged - merged0, "workers": a.workers,
                    "budget_gb": a.budget_gb, "gauges_per_volume": a.gauges,
                    "deadline_s": a.deadline, "lifo_after_s": svc.lifo_after_s,
                    "warmup_s": round(warm_s, 2),
                    "shed": sum((q.error or "").startswith("DeadlineExceeded") for q in reqs),
                    "batch_sizes": {str(b): sum(q.batch == b for q in ok)
                                    for b in sorted({q.batch for q in ok})},
                    "fields_evicted": svc.evicted, "work_handles_moved": svc.handles_moved})
        print(json.dumps(out), flush=True)
    finally:
        svc.close()


if __name__ == "__main__":
    main()
