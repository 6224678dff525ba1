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
            q.done.wait()
            assert q.error is None, q.error
            alone.append(q)
        mix = [svc.submit(clone(serve, r)) for r in reqs]
        for q in mix:
            q.done.wait()
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
            q.done.wait()
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
            q.done.wait()
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
            q.done.wait()
            assert q.error is None, q.error
            assert q.x is q.out
            assert np.linalg.norm(q.out - x) / np.linalg.norm(x) < 1e-8
        assert max(q.batch for q in subs) > 1
    finally:
        svc.close()
