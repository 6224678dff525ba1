"""A different kappa for each RHS of a multi-RHS handle
(qwsg_batch_set_kappas): every operator applied to RHS r is bit-equal to the
one-RHS operator of a lattice with the same gauge field at kappa_r (the
clover terms are built by the same kernel, and the kernels' per-lane
arithmetic is the one-RHS arithmetic); the batched solvers reach each RHS's
solution within the solve tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L, NB, CSW = (8, 8, 8, 16), (2, 2, 2, 2), 1.7
KAPPAS = [0.1300, 0.1345, 0.1365, 0.1280]


@pytest.fixture(scope="module")
def setup():
    import qws_b200

    U, _ = qws_b200.gen_gauge(L, 21, 5, 0.36)
    parent = qws_b200.Lattice(L, NB, tbc=-1, kappa=0.1330)
    parent.load_gauge(U)
    parent.build_clover(CSW)
    B = parent.batch(len(KAPPAS))
    B.set_kappas(KAPPAS, CSW)
    singles = []
    for k in KAPPAS:
        s = qws_b200.Lattice(L, NB, tbc=-1, kappa=k)
        s.load_gauge(U)
        s.build_clover(CSW)
        singles.append(s)
    S = np.stack([qws_b200.gen_source(L, 40 + r, "gauss") for r in range(len(KAPPAS))])
    yield B, singles, S
    B.close()
    for s in singles:
        s.close()
    parent.close()


def test_operators_bit_equal(setup):
    B, singles, S = setup
    S32 = S.astype(np.float32)
    got = {"ddd_d": B.to_host(B.ddd(B.to_device(S))), "ddd_s": B.to_host(B.ddd(B.to_device(S32))),
           "prec": B.to_host(B.prec(B.to_device(S32), 4, 2)),
           "prec_h": B.to_host(B.prec_h(B.to_device(S32), 4, 2))}
    for r, s in enumerate(singles):
        want = {"ddd_d": s.to_host(s.ddd(s.to_device(S[r]))),
                "ddd_s": s.to_host(s.ddd(s.to_device(S32[r]))),
                "prec": s.to_host(s.prec(s.to_device(S32[r]), 4, 2)),
                "prec_h": s.to_host(s.prec_h(s.to_device(S32[r]), 4, 2))}
        for k in want:
            assert np.array_equal(got[k][r], want[k]), (k, r)


@pytest.mark.parametrize("solver", ["plain", "hf"])
def test_solves(setup, solver):
    B, singles, S = setup
    bd = B.to_device(S)
    xb = B.empty("f64")
    if solver == "plain":
        B.bicgstab_dd_mix(xb, bd, 1e-10, 50, 1e-6, 50, 4, 2)
    else:
        B.bicgstab_dd_mix2_hf(xb, bd, 1e-10, 50, 1e-6, 50, 4, 2, reliable=5)
    assert max(B.true_residual(xb, bd)) < 1e-10
    X = B.to_host(xb)
    for r, s in enumerate(singles):
        b1 = s.to_device(S[r])
        x1 = s.empty("f64")
        if solver == "plain":
            s.bicgstab_dd_mix(x1, b1, 1e-10, 50, 1e-6, 50, 4, 2)
        else:
            s.bicgstab_dd_mix2_hf(x1, b1, 1e-10, 50, 1e-6, 50, 4, 2, reliable=5)
        x1h = s.to_host(x1)
        assert np.linalg.norm(X[r] - x1h) / np.linalg.norm(x1h) < 1e-8, r
        # and it is the solution of that kappa's system
        assert s.true_residual(s.to_device(X[r]), b1) < 1e-9, r


def test_kappas_change(setup):
    """A second set_kappas call rebuilds the clover terms (graphs stay valid:
    they read the kappa tables and planes at run time)."""
    import qws_b200

    B, singles, S = setup
    S32 = S.astype(np.float32)
    B.set_kappas(KAPPAS[::-1], CSW)
    try:
        got = B.to_host(B.prec_h(B.to_device(S32), 4, 2))
        for r, s in enumerate(singles[::-1]):
            assert np.array_equal(got[r], s.to_host(s.prec_h(s.to_device(S32[r]), 4, 2))), r
    finally:
        B.set_kappas(KAPPAS, CSW)
