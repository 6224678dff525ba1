"""Multi-RHS handles (qwsg_create_batch): every operator launch serves all
right-hand sides, so each RHS must get exactly what a single-RHS call gives
(the per-(site, RHS) arithmetic is identical: bit-equal operators), and the
batched solvers must return, for every RHS, a solution within the solve
tolerance of the single-RHS solve of that RHS -- alone and in the mix.

Fields: seeded SU(3) links with 5 APE steps and the clover-leaf term
(qws_b200.gen_*), 8x8x8x16 on the block grid (2,2,2,2) and the reference
partition (2,1,1,1).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KAPPA, CSW = 0.1365, 1.7


@pytest.fixture(scope="module", params=[(2, 2, 2, 2), (2, 1, 1, 1)], ids=["blk2222", "ref2111"])
def lat(request):
    import qws_b200

    L = (8, 8, 8, 16)
    U, _ = qws_b200.gen_gauge(L, 7, 5, 0.36)
    C = qws_b200.gen_clover(U, L, CSW, KAPPA)
    lt = qws_b200.Lattice(L, request.param, tbc=-1, kappa=KAPPA)
    lt.load_fields(U, C)
    yield lt
    lt.close()


def sources(L, n, seed):
    import qws_b200

    return np.stack([qws_b200.gen_source(L, seed + k, "gauss") for k in range(n)])


def rel(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("nr", [1, 4, 16])
def test_operators_bit_equal(lat, nr):
    B = lat.batch(nr)
    try:
        S = sources(lat.L, nr, 100)
        S32 = S.astype(np.float32)
        xd, xs = B.to_device(S), B.to_device(S32)
        got = {"ddd_d": B.to_host(B.ddd(xd)), "ddd_s": B.to_host(B.ddd(xs)),
               "prec_ddd": B.to_host(B.prec_ddd(xs, 4, 2)), "prec": B.to_host(B.prec(xs, 4, 2)),
               "prec_h": B.to_host(B.prec_h(xs, 4, 2)),
               "ddd_out": B.to_host(B.ddd_out(xs, 1, -KAPPA, out=B.to_device(S32)))}
        for k in range(nr):
            d, s = lat.to_device(S[k]), lat.to_device(S32[k])
            want = {"ddd_d": lat.to_host(lat.ddd(d)), "ddd_s": lat.to_host(lat.ddd(s)),
                    "prec_ddd": lat.to_host(lat.prec_ddd(s, 4, 2)),
                    "prec": lat.to_host(lat.prec(s, 4, 2)), "prec_h": lat.to_host(lat.prec_h(s, 4, 2)),
                    "ddd_out": lat.to_host(lat.ddd_out(s, 1, -KAPPA, out=lat.to_device(S32[k])))}
            for name in want:
                got_k = got[name] if nr == 1 else got[name][k]
                np.testing.assert_array_equal(got_k, want[name], err_msg=f"{name} rhs {k}")
    finally:
        B.close()


def test_inner_solver_per_rhs(lat):
    nr = 4
    B = lat.batch(nr)
    try:
        S = sources(lat.L, nr, 200).astype(np.float32)
        S /= np.linalg.norm(S.reshape(nr, -1), axis=1)[:, None, None]
        xb, itb, _ = B.bicgstab_precdd(B.to_device(S), 1e-6, 50)
        xb = B.to_host(xb)
        _, its = B.batch_stats()
        for k in range(nr):
            xs, it, _ = lat.bicgstab_precdd(lat.to_device(S[k]), 1e-6, 50)
            assert abs(its[k] - it) <= 1, (k, its[k], it)
            assert rel(xb[k], lat.to_host(xs)) < 1e-4, k  # FP32 iterates, 1e-6 tolerance
        assert itb == max(its)
    finally:
        B.close()


@pytest.mark.parametrize("form", ["plain", "precision"])
def test_dd_solver_alone_and_in_the_mix(lat, form):
    """Each RHS of a 4-RHS solve (mixed with three others) against its own
    single-RHS solve: true residual below tol for both, solutions within
    1e-8 relative (a few times tol), outer iterations within 1."""
    nr, tol = 4, 1e-10
    B = lat.batch(nr)
    try:
        S = sources(lat.L, nr, 300)
        S[2] *= 1e3  # scales differ inside the mix
        xb = B.empty("f64")
        bd = B.to_device(S)
        if form == "plain":
            B.bicgstab_dd_mix(xb, bd, tol, 100, 1e-6, 50)
        else:
            B.bicgstab_dd_mix2_hf(xb, bd, tol, 100, 1e-6, 50, reliable=5)
        per, _ = B.batch_stats()
        truer = B.true_residual(xb, bd)
        X = B.to_host(xb)
        for k in range(nr):
            x = lat.empty("f64")
            b = lat.to_device(S[k])
            if form == "plain":
                st = lat.bicgstab_dd_mix(x, b, tol, 100, 1e-6, 50)
            else:
                st = lat.bicgstab_dd_mix2_hf(x, b, tol, 100, 1e-6, 50, reliable=5)
            assert truer[k] < tol and lat.true_residual(x, b) < tol, (k, truer[k])
            assert abs(per[k]["outer_iters"] - st["outer_iters"]) <= 1, (k, per[k], st)
            assert rel(X[k], lat.to_host(x)) < 1e-8, k
    finally:
        B.close()


def test_zero_rhs_in_a_batch(lat):
    """A zero right-hand side (padding of a batch) stays exactly zero and does
    not disturb the others."""
    nr = 4
    B = lat.batch(nr)
    try:
        S = sources(lat.L, nr, 400)
        S[1] = 0
        xb = B.empty("f64")
        bd = B.to_device(S)
        B.bicgstab_dd_mix2_hf(xb, bd, 1e-10, 100, 1e-6, 50, reliable=5)
        X = B.to_host(xb)
        assert np.all(X[1] == 0)
        assert np.all(np.isfinite(X))
        r = B.true_residual(xb, bd)
        assert all(r[k] < 1e-10 for k in (0, 2, 3)), r
    finally:
        B.close()


def test_graphs_replay_matches_direct(lat):
    """The SAP preconditioner replayed from its captured CUDA graph gives the
    same bits as the directly launched sequence."""
    import torch

    import qws_b200

    # graphs need a stream other than the legacy default one
    B = lat.batch(1, stream=torch.cuda.Stream())
    try:
        b = B.to_device(qws_b200.gen_source(lat.L, 77).astype(np.float32))
        B.set_graphs(False)
        want = B.to_host(B.prec_ddd(b, 4, 2))
        want_h = B.to_host(B.prec_h(b, 4, 2))
        B.set_graphs(True)
        n0 = qws_b200.launch_count()
        for _ in range(3):  # first call captures, later calls replay
            np.testing.assert_array_equal(B.to_host(B.prec_ddd(b, 4, 2)), want)
            np.testing.assert_array_equal(B.to_host(B.prec_h(b, 4, 2)), want_h)
        assert qws_b200.launch_count() - n0 > 6 * 10  # replays count their kernels
    finally:
        B.close()
