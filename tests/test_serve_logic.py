"""The solve service's scheduling on CPU (no GPU work): compatible pending
requests (same lattice, gauge field, csw; any kappa and tolerance) merge
into a power-of-two batch of at most max_batch, the oldest request goes
first, a busy field holds back its requests, and admission evicts idle work
buffers, then idle fields, least recently used first, never the field the
job needs.  Requests past their deadline and cancelled requests finish with
an error instead of running; waiting on a request has a timeout."""
import threading

import numpy as np

from qws_b200 import serve


class FakeHandle:
    def __init__(self):
        self.closed = False

    def close(self):
        self.closed = True


class FakeResident:
    def __init__(self, L, gid, last_used, busy=False, work=()):
        self.L, self.gid, self.last_used, self.busy = L, gid, last_used, busy
        self.lat = FakeHandle()
        self.bytes = serve.field_bytes(L)
        self.work = {nr: FakeHandle() for nr in work}
        self.closed = False

    def close(self):
        self.closed = True


def make_service(budget, max_batch=16):
    svc = serve.Service.__new__(serve.Service)  # the scheduling state only, no threads
    svc.budget, svc.max_batch = float(budget), max_batch
    svc.pending, svc.residents, svc.used, svc.merged, svc.evicted = [], {}, 0.0, 0, 0
    svc.completed = []
    svc.cv = threading.Condition()
    svc.lifo_after_s = None
    svc.group = 1
    svc.handles_moved = 0
    svc.failed = None
    svc.group_max_sites = float("inf")
    svc.group_rounds = 0
    svc.group_launches = [0, 0]
    svc.group_phase_s = [0.0, 0.0, 0.0]
    svc.group_host_s = dict.fromkeys(("t_members", "t_merge", "t_launch", "t_gpu_wait"), 0.0)
    return svc


def req(L, gauge, kappa, tol=1e-10):
    return serve.Request(L=L, gauge=gauge, kappa=kappa, csw=1.7, tol=tol, source=np.zeros(1))


L1, L2 = (8, 8, 8, 8), (16, 16, 16, 32)


def test_merge_power_of_two_and_order():
    svc = make_service(1e12, max_batch=4)
    # kappas and tolerances differ: still compatible (per-RHS kappa and tol)
    a = [req(L1, 0, 0.13 + 0.001 * k, tol=(1e-8, 1e-10, 1e-12)[k % 3]) for k in range(5)]
    b = req(L1, 1, 0.12, tol=1e-8)  # another gauge field
    svc.pending = [b] + a
    res, group = svc._pick()
    assert group == [b]                      # the oldest request first
    res.busy = False
    res2, group2 = svc._pick()
    assert group2 == a[:4] and svc.merged == 3  # 5 compatible -> a batch of 4
    assert svc.pending == [a[4]]


def test_busy_field_waits():
    svc = make_service(1e12)
    svc.residents[(L1, 0)] = FakeResident(L1, 0, 1.0, busy=True)
    r1, r2 = req(L1, 0, 0.13), req(L2, 1, 0.13)
    svc.pending = [r1, r2]
    res, group = svc._pick()
    assert group == [r2]      # r1's field is busy: the next request starts
    assert svc.pending == [r1]


def test_eviction_lru_and_keep():
    nr_bytes = serve.work_bytes(L2, 1)
    old = FakeResident(L2, 0, last_used=1.0, work=(1,))
    new = FakeResident(L2, 1, last_used=2.0, work=(1,))
    busy = FakeResident(L2, 2, last_used=0.5, busy=True)
    svc = make_service(budget=3 * serve.field_bytes(L2) + 2 * nr_bytes)
    svc.residents = {(L2, 0): old, (L2, 1): new, (L2, 2): busy}
    svc.used = 3 * serve.field_bytes(L2) + 2 * nr_bytes
    # a new field for another volume: idle work buffers go first (oldest
    # first), then the least recently used idle field; never the busy one
    need = serve.field_bytes(L2) + 2 * nr_bytes
    assert svc._evict(need)
    assert old.work == {} and new.work == {}
    assert old.closed and (L2, 0) not in svc.residents
    assert not new.closed and not busy.closed
    # `keep` is never evicted, even when it is the only idle field
    svc2 = make_service(budget=serve.field_bytes(L2))
    k = FakeResident(L2, 3, last_used=0.1)
    svc2.residents = {(L2, 3): k}
    svc2.used = serve.field_bytes(L2)
    assert not svc2._evict(1, keep=k) and not k.closed


def test_admission_reserves_bytes():
    one2 = serve.field_bytes(L2) + serve.work_bytes(L2, 1)
    svc = make_service(budget=one2)
    svc.pending = [req(L1, 0, 0.13), req(L1, 0, 0.13), req(L2, 0, 0.13)]
    res, group = svc._pick()
    assert len(group) == 2 and svc.used == serve.field_bytes(L1) + serve.work_bytes(L1, 2)
    assert svc._pick() is None  # L2 does not fit while L1's field is busy


def test_batch_capped_by_memory():
    """Four compatible requests whose 4-RHS batch would not fit the budget
    run as a batch of two (a batch that can never fit must not wait for
    ever)."""
    svc = make_service(budget=serve.field_bytes(L2) + serve.work_bytes(L2, 2) + 1)
    svc.pending = [req(L2, 0, 0.13 + 0.001 * k) for k in range(4)]
    res, group = svc._pick()
    assert len(group) == 2 and len(svc.pending) == 2


def test_never_fits_fails_at_once():
    svc = make_service(budget=serve.field_bytes(L2))
    big, small = req(L2, 0, 0.13), req(L1, 0, 0.13)
    svc.pending = [big, small]
    res, group = svc._pick()
    assert group == [small]
    assert big.done.is_set() and "MemoryError" in big.error and svc.pending == []


def test_no_futile_eviction():
    """Idle fields stay when evicting all of them would still not make room."""
    svc = make_service(budget=2 * serve.field_bytes(L2))
    idle = FakeResident(L2, 0, last_used=1.0)
    busy = FakeResident(L2, 1, last_used=1.0, busy=True)
    svc.residents = {(L2, 0): idle, (L2, 1): busy}
    svc.used = 2 * serve.field_bytes(L2)
    assert not svc._evict(2 * serve.field_bytes(L2))
    assert not idle.closed and (L2, 0) in svc.residents


def test_waiting_request_not_overtaken():
    """A request that waits for memory held by a running job blocks later
    requests that would have to evict idle memory; one that needs no new
    memory, or fits the free budget, still starts."""
    f2, w2 = serve.field_bytes(L2), serve.work_bytes(L2, 1)
    warm_bytes = serve.field_bytes(L1) + serve.work_bytes(L1, 1)

    def setup(budget):
        svc = make_service(budget=budget)
        busy = FakeResident(L2, 0, last_used=1.0, busy=True, work=(1,))
        warm = FakeResident(L1, 0, last_used=1.0, work=(1,))
        svc.residents = {(L2, 0): busy, (L1, 0): warm}
        svc.used = f2 + w2 + warm_bytes
        waiting, later, ready = req(L2, 1, 0.13), req(L1, 1, 0.13), req(L1, 0, 0.13)
        svc.pending = [waiting, later, ready]
        return svc, warm, waiting, later, ready

    # `later` (a new L1 field; it would take over `warm`'s idle work
    # buffers, so it needs a field's bytes) would need `warm` evicted: it waits
    f1 = serve.field_bytes(L1)
    svc, warm, waiting, later, ready = setup(f2 + w2 + warm_bytes + f1 - 1)
    res, group = svc._pick()
    assert group == [ready] and res is warm and not warm.closed
    assert svc.pending == [waiting, later]
    # with room for it in the free budget, `later` starts before `ready`
    svc, warm, waiting, later, ready = setup(f2 + w2 + warm_bytes + f1)
    res, group = svc._pick()
    assert group == [later] and not warm.closed
    assert svc.pending == [waiting, ready]


def test_stream_priority_by_volume():
    """Smaller lattices get higher CUDA stream priority (lower numbers), one
    level per factor 4 of volume, at most three levels above the default."""
    vols = [(48, 48, 48, 96), (32, 32, 32, 64), (24, 24, 24, 48), (16, 16, 16, 32), (8, 8, 8, 8)]
    pr = [serve.stream_priority(L) for L in vols]
    assert pr == sorted(pr, reverse=True) and pr[0] == 0 and min(pr) == -3


def test_summarize_phases_errors_and_volumes():
    """summarize: failed requests are counted by kind and left out of the
    latencies; phases and per-volume figures come from the completed ones."""
    def done(L, lat, solve, err=None, res=0.0):
        q = req(L, 0, 0.13)
        q.t_arrival, q.t_start, q.t_done = 0.0, 0.01, lat
        q.t_resident, q.t_clover, q.t_solve = res, 0.001, solve
        q.stats, q.batch, q.error = {"true_rel_resid": 1e-12}, 1, err
        return q

    reqs = [done(L1, 0.05, 0.02), done(L1, 0.07, 0.03), done(L2, 0.5, 0.3, res=0.1),
            done(L2, 0.0, 0.0, err="MemoryError: too big")]
    st = serve.summarize(reqs)
    assert st["completed"] == 3 and st["errors"] == 1
    assert st["error_kinds"] == {"MemoryError: too big": 1}
    assert st["requests_with_field_load"] == 1 and st["above_tol"] == 0
    assert st["by_volume"]["8x8x8x8"][0] == 2 and st["by_volume"]["16x16x16x32"] == [1, 500.0, 300.0]
    assert st["phases_ms"]["queue"][0] == 10.0


def test_deadline_expires_before_start():
    svc = make_service(1e12)
    svc.residents[(L1, 0)] = FakeResident(L1, 0, 1.0, busy=True)
    late = req(L1, 0, 0.13)
    late.deadline_s = 0.5
    late.t_arrival = -10.0  # arrived long ago, its field still busy
    ok = req(L2, 1, 0.13)
    ok.deadline_s = 3600.0
    svc.pending = [late, ok]
    import time as _t
    ok.t_arrival = _t.monotonic()
    res, group = svc._pick()
    assert group == [ok]
    assert late.done.is_set() and late.error.startswith("DeadlineExceeded")
    assert late in svc.completed and svc.pending == []


def test_cancel_pending_only():
    svc = make_service(1e12)
    a, b = req(L1, 0, 0.13), req(L1, 0, 0.13)
    svc.pending = [a, b]
    assert svc.cancel(a)
    assert a.done.is_set() and a.error == "Cancelled" and svc.pending == [b]
    assert not svc.cancel(a)  # already finished
    res, group = svc._pick()
    assert group == [b]
    assert not svc.cancel(b)  # started: a running solve is not interrupted


def test_wait_times_out():
    import pytest

    q = req(L1, 0, 0.13)
    with pytest.raises(TimeoutError):
        q.wait(0.01)
    q.done.set()
    assert q.wait(0.01) is q


def test_adaptive_lifo_under_overload():
    """Once the oldest pending request has waited longer than lifo_after_s,
    the newest compatible requests are served first (the oldest are the
    ones a deadline sheds); before that, arrival order."""
    import time as _t

    svc = make_service(1e12, max_batch=2)
    svc.lifo_after_s = 1.0
    now = _t.monotonic()
    reqs = [req(L1, 0, 0.13) for _ in range(4)]
    for k, q in enumerate(reqs):
        q.t_arrival = now - 0.1 * (4 - k)  # all recent: arrival order
    svc.pending = list(reqs)
    res, group = svc._pick()
    assert group == reqs[:2]
    res.busy = False
    svc.pending = list(reqs)
    reqs[0].t_arrival = now - 5.0  # the oldest has waited long: newest first
    res, group = svc._pick()
    assert group == [reqs[3], reqs[2]]


def test_group_jobs_take_every_startable_request():
    """With group > 1 an idle worker takes every job that can start now (one
    request each: merging into multi-RHS solves is off), up to `group`; a
    request whose field is busy waits for a later group."""
    svc = make_service(1e12, max_batch=1)
    svc.group = 3
    reqs = [req(L1, g, 0.13) for g in range(4)] + [req(L2, 0, 0.13)]
    busy = FakeResident(L1, 1, 0.0, busy=True)
    svc.residents[(L1, 1)] = busy
    svc.pending = list(reqs)
    jobs = svc._next_job()
    assert [g for _, g in jobs] == [[reqs[0]], [reqs[2]], [reqs[3]]]
    jobs = svc._next_job()
    assert [g for _, g in jobs] == [[reqs[4]]]
    assert svc.pending == [reqs[1]] and svc._next_job() is None
    svc.group = 1
    busy.busy = False
    res, group = svc._next_job()
    assert group == [reqs[1]]


def test_group_failed_solve_fails_only_its_request(monkeypatch):
    """A group solve reports a status per request: a failed one gets its
    error, the others their results."""
    import qws_b200

    svc = make_service(1e12, max_batch=1)
    svc.solver = dict(maxiter=10, tol_s=1e-6, maxiter_s=50, reliable=0)
    reqs = [req(L1, g, 0.13) for g in range(3)]
    finished = []

    def stage(res, group):
        return {"res": res, "group": group, "B": object(), "xd": None, "bd": None,
                "cfg": {"nsap": 4, "nm": 2}}

    def finish(p):
        for q in p["group"]:
            q.t_done = 1.0
        finished.append((p["group"][0], p["group_size"], p["stats"]["status"]))

    def group_solve(solves, check=True):
        assert not check and len(solves) == 3
        return ([{"status": 3 if k == 1 else 0, "outer_iters": 1, "inner_iters": 9,
                  "rel_resid_recursive": 0.0, "rel_resid_true": -1.0} for k in range(3)],
                {"rounds": 5, "merged_launches": 10, "member_launches": 30, "t_members": 0.1,
                 "t_merge": 0.1, "t_launch": 0.1, "t_gpu_wait": 0.1})

    monkeypatch.setattr(svc, "_stage", stage, raising=False)
    monkeypatch.setattr(svc, "_finish", finish, raising=False)
    monkeypatch.setattr(qws_b200, "group_solve", group_solve)
    svc._run_group([(FakeResident(L1, g, 0.0), [q]) for g, q in enumerate(reqs)])
    assert sorted(finished, key=lambda f: reqs.index(f[0])) == [(reqs[0], 3, 0), (reqs[2], 3, 0)]
    assert reqs[1].error.startswith("QwsgError") and reqs[1].t_done > 0
    assert reqs[0].error is None and svc.group_rounds == 5


def test_group_leaves_large_lattices_alone():
    """With group_max_sites, a lattice above it starts as a job of its own
    (its own stream) and the group takes only the smaller ones."""
    svc = make_service(1e12, max_batch=1)
    svc.group = 8
    svc.group_max_sites = 20000
    big = req(L2, 0, 0.13)                     # 131072 sites
    smalls = [req(L1, g, 0.13) for g in range(3)]
    svc.pending = [smalls[0], big, smalls[1], smalls[2]]
    jobs = svc._next_job()
    assert [g for _, g in jobs] == [[smalls[0]], [smalls[1]], [smalls[2]]]
    res, group = svc._next_job()
    assert group == [big]


def test_idle_work_handle_moves_to_another_field_of_the_volume():
    """A job on a field without work buffers takes over an idle field's
    buffers of the same volume and RHS count (no new allocation, no
    eviction) instead of allocating its own."""
    fb, wb = serve.field_bytes(L1), serve.work_bytes(L1, 1)
    svc = make_service(2 * fb + wb)           # room for two fields and one handle
    donor = FakeResident(L1, 0, 1.0, work=(1,))
    target = FakeResident(L1, 1, 2.0)
    svc.residents = {(L1, 0): donor, (L1, 1): target}
    svc.used = 2 * fb + wb
    handle = donor.work[1]
    q = req(L1, 1, 0.13)
    svc.pending = [q]
    res, group = svc._pick()
    assert res is target and group == [q]
    assert target.work == {1: handle} and donor.work == {}
    assert not handle.closed and not donor.closed and svc.handles_moved == 1
    assert svc.used == 2 * fb + wb            # nothing allocated, nothing freed
    # a field that is not resident yet: the placeholder takes the handle
    target.busy = False
    q2 = req(L1, 2, 0.13)
    svc.budget = 3 * fb + wb
    svc.pending = [q2]
    res2, group2 = svc._pick()
    assert isinstance(res2, serve._Placeholder) and res2.work == {1: handle}
    assert target.work == {}


def test_takeover_that_cannot_fit_falls_back_to_new_buffers():
    """When room for a new field can only be made by evicting the idle field
    whose work buffers the job would take over, the job gets new buffers
    and that field is evicted (nothing running could ever free the memory
    otherwise, and the request would wait for ever)."""
    fb, wb = serve.field_bytes(L2), serve.work_bytes(L2, 1)
    svc = make_service(fb + wb + fb // 2)      # one field and its buffers, not two fields
    donor = FakeResident(L2, 0, 1.0, work=(1,))
    svc.residents = {(L2, 0): donor}
    svc.used = fb + wb
    q = req(L2, 1, 0.13)
    svc.pending = [q]
    res, group = svc._pick()
    assert group == [q] and isinstance(res, serve._Placeholder)
    assert donor.closed and (L2, 0) not in svc.residents
    assert res.work == {} and svc.used == fb + wb and svc.handles_moved == 0


def test_stalled_admission_fails_the_requests():
    """With every worker idle nothing can free memory: requests that still
    cannot start after stall_s fail with AdmissionStalled (a bug elsewhere
    must not leave their callers waiting for ever)."""
    svc = make_service(1e12)
    svc.workers = [None, None]
    svc.idle_workers = 2
    svc.stall_s = 1.0
    svc._stall_since = None
    q = req(L1, 0, 0.13)
    svc.pending = [q]
    svc._stalled(None, 100.0)
    assert svc.pending == [q]
    svc._stalled(None, 100.5)
    assert svc.pending == [q]
    svc._stalled(None, 101.5)
    assert svc.pending == [] and q.error.startswith("AdmissionStalled") and q.done.is_set()
    # a running job resets the clock
    q2 = req(L1, 0, 0.13)
    svc.pending = [q2]
    svc._stalled(None, 200.0)
    svc.idle_workers = 1
    svc._stalled(None, 300.0)
    svc.idle_workers = 2
    svc._stalled(None, 300.5)
    assert svc.pending == [q2]


def test_scheduler_failure_fails_requests_instead_of_hanging(monkeypatch):
    """An exception in the scheduler (a CUDA error while freeing memory, say)
    fails every pending and every later request with ServiceFailed; nobody
    waits for ever."""
    svc = make_service(1e12)
    svc.stop = False
    svc.idle_workers = 1
    svc.workers = [None]
    svc._stall_since = None
    svc.stall_s = 5.0
    svc.jobs = None
    svc.ids = iter(range(100))
    q = req(L1, 0, 0.13)
    svc.pending = [q]

    def boom():
        raise RuntimeError("CUDA error: an illegal memory access was encountered")

    monkeypatch.setattr(svc, "_next_job", boom)
    svc._scheduler()  # returns instead of looping
    assert q.done.is_set() and q.error.startswith("ServiceFailed: RuntimeError")
    q2 = svc.submit(req(L1, 1, 0.13))
    assert q2.wait(0.1).error.startswith("ServiceFailed")
