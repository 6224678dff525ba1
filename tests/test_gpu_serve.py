"""The solve service (qws_b200.serve): every request's result is the same
alone and in the mix -- merged into a multi-RHS batch with compatible
requests, or overlapped on the GPU with requests on other fields -- within
the stated tolerance, and admission against a small HBM budget (evicting
idle fields) still completes everything."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VOLS = [(8, 8, 8, 16), (8, 8, 8, 8)]


def make_requests(serve, n, seed):
    import qws_b200

    rng = np.random.default_rng(seed)
    src = {L: [qws_b200.gen_source(L, 50 + k) for k in range(3)] for L in VOLS}
    kappas = [0.1300, 0.1340]  # few values, so that some requests are compatible
    out = []
    for i in range(n):
        L = VOLS[i % 2]
        out.append(serve.Request(L=L, gauge=int(rng.integers(2)), kappa=kappas[int(rng.integers(2))],
                                 csw=1.7, tol=1e-10, source=src[L][i % 3]))
    return out


def clone(serve, r):
    return serve.Request(L=r.L, gauge=r.gauge, kappa=r.kappa, csw=r.csw, tol=r.tol, source=r.source)


def test_alone_and_in_the_mix():
    from qws_b200 import serve

    reqs = make_requests(serve, 16, 1)
    svc = serve.Service(serve.seeded_gauge(), budget_bytes=40e9, workers=3, max_batch=8)
    try:
        alone = []
        for r in reqs:
            q = svc.submit(clone(serve, r))
            q.wait(600)
            assert q.error is None, q.error
            alone.append(q)
        mix = [svc.submit(clone(serve, r)) for r in reqs]
        for q in mix:
            q.wait(600)
            assert q.error is None, q.error
        assert max(q.batch for q in mix) > 1, "no request was merged"
        assert svc.merged > 0
        for a, m in zip(alone, mix):
            assert a.stats["true_rel_resid"] < a.tol and m.stats["true_rel_resid"] < m.tol
            d = np.linalg.norm(a.x - m.x) / np.linalg.norm(a.x)
            assert d < 1e-8, (a.rid, m.batch, d)
        st = serve.summarize(mix)
        assert st["completed"] == len(mix) and st["above_tol"] == 0
        assert st["p99_ms"] >= st["p50_ms"] > 0
    finally:
        svc.close()


def test_small_budget_evicts_and_completes():
    from qws_b200 import serve

    reqs = make_requests(serve, 8, 2)
    # room for one field and one single-RHS job of the larger volume at a time
    budget = serve.field_bytes(VOLS[0]) + serve.work_bytes(VOLS[0], 1) + 1
    svc = serve.Service(serve.seeded_gauge(), budget_bytes=budget, workers=2, max_batch=1)
    try:
        subs = [svc.submit(clone(serve, r)) for r in reqs]
        for q in subs:
            q.wait(600)
            assert q.error is None, q.error
            assert q.stats["true_rel_resid"] < q.tol
        assert svc.used <= budget
    finally:
        svc.close()


def test_caller_output_buffers():
    """A request's solution lands in the caller's array (page-locked or not),
    alone and when merged into a batch; sources may be page-locked."""
    import torch

    from qws_b200 import serve

    reqs = make_requests(serve, 12, 3)
    svc = serve.Service(serve.seeded_gauge(), budget_bytes=40e9, workers=2, max_batch=8)
    try:
        ref = []
        for r in reqs:
            q = svc.submit(clone(serve, r))
            q.wait(600)
            assert q.error is None, q.error
            ref.append(q.x)
        subs = []
        for k, r in enumerate(reqs):
            q = clone(serve, r)
            shape = (int(np.prod(r.L)), 24)
            pin = torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
            pin[...] = r.source
            q.source = pin
            q.out = (torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy() if k % 2
                     else np.empty(shape))
            subs.append(svc.submit(q))
        for q, x in zip(subs, ref):
            q.wait(600)
            assert q.error is None, q.error
            assert q.x is q.out
            assert np.linalg.norm(q.out - x) / np.linalg.norm(x) < 1e-8
        assert max(q.batch for q in subs) > 1
    finally:
        svc.close()


def test_tolerances_merge_and_failures_are_per_request():
    """Requests with different tolerances on one field merge into one batch,
    each stopping at its own tolerance; a request whose source holds a NaN
    fails alone with a solver error, and the field serves the next request."""
    import qws_b200
    from qws_b200 import serve

    L = VOLS[0]
    svc = serve.Service(serve.seeded_gauge(), budget_bytes=40e9, workers=1, max_batch=4)
    try:
        warm = svc.submit(serve.Request(L=L, gauge=0, kappa=0.13, csw=1.7, tol=1e-8,
                                        source=qws_b200.gen_source(L, 1)))
        # queued behind `warm` on the same field, these four merge
        tols = [1e-6, 1e-8, 1e-10, 1e-12]
        reqs = [svc.submit(serve.Request(L=L, gauge=0, kappa=0.13 + 0.001 * k, csw=1.7,
                                         tol=t, source=qws_b200.gen_source(L, 10 + k)))
                for k, t in enumerate(tols)]
        for q in [warm] + reqs:
            q.wait(600)
            assert q.error is None, q.error
        assert max(q.batch for q in reqs) > 1
        for q in reqs:
            assert q.stats["true_rel_resid"] < q.tol
        # the loosest request stopped at its own tolerance, earlier than the
        # tightest: its true residual is far above the tightest one's
        assert reqs[0].stats["true_rel_resid"] > 10 * reqs[-1].stats["true_rel_resid"]
        bad_src = qws_b200.gen_source(L, 20)
        bad_src[3, 1] = np.nan
        bad = svc.submit(serve.Request(L=L, gauge=0, kappa=0.13, csw=1.7, tol=1e-10,
                                       source=bad_src)).wait(600)
        assert bad.error is not None and "non-finite" in bad.error
        good = svc.submit(serve.Request(L=L, gauge=0, kappa=0.13, csw=1.7, tol=1e-10,
                                        source=qws_b200.gen_source(L, 21))).wait(600)
        assert good.error is None and good.stats["true_rel_resid"] < 1e-10
    finally:
        svc.close()


def test_deadline_and_cancel_on_a_busy_service():
    """With one worker busy on a long solve, a queued request whose deadline
    passes fails with DeadlineExceeded and a cancelled one with Cancelled;
    the rest complete."""
    import qws_b200
    from qws_b200 import serve

    big = (32, 32, 32, 64)
    svc = serve.Service(serve.seeded_gauge(), budget_bytes=40e9, workers=1, max_batch=1)
    try:
        long_job = svc.submit(serve.Request(L=big, gauge=0, kappa=0.136, csw=1.7, tol=1e-12,
                                            source=qws_b200.gen_source(big, 1)))
        late = serve.Request(L=VOLS[1], gauge=0, kappa=0.13, csw=1.7, tol=1e-8,
                             source=qws_b200.gen_source(VOLS[1], 2), deadline_s=0.05)
        gone = serve.Request(L=VOLS[1], gauge=1, kappa=0.13, csw=1.7, tol=1e-8,
                             source=qws_b200.gen_source(VOLS[1], 3))
        late, gone = svc.submit(late), svc.submit(gone)
        assert svc.cancel(gone)
        for q in (long_job, late, gone):
            q.wait(600)
        assert long_job.error is None
        assert gone.error == "Cancelled"
        assert late.error is not None and late.error.startswith("DeadlineExceeded")
    finally:
        svc.close()
