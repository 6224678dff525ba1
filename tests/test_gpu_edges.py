"""Edge cases of the GPU path against the oracle: a periodic time boundary
(tbc = +1), blocks of odd extent and lattices whose volume is not a
multiple of the 128-site plane padding, the largest RHS count (32), a
zero source, and the host checks that reject bad geometries.  Tolerances as
in test_gpu_dd.py: FP64 operators 1e-13, FP32 operators 1e-6, the FP32 SAP
5e-6, the mixed solve 1e-10 at tolerance 1e-12."""
import numpy as np
import pytest

from qwsref import Oracle

pytestmark = pytest.mark.gpu

KAPPA, CSW = 0.1300, 1.7


def rel(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def fields(L, seed=3):
    import qws_b200

    U, _ = qws_b200.gen_gauge(L, seed, 3, 0.36)
    C = qws_b200.gen_clover(U, L, CSW, KAPPA)
    return U, C


@pytest.mark.parametrize("L,NB,tbc", [
    ((8, 4, 4, 8), (2, 1, 1, 1), +1),     # periodic time
    ((12, 6, 6, 6), (2, 2, 2, 2), -1),    # blocks 6x3x3x3: odd extents
    ((6, 6, 2, 10), (2, 1, 1, 2), -1),    # V = 720: not a multiple of 128
])
def test_operators_and_solve(L, NB, tbc):
    import qws_b200

    U, C = fields(L)
    o = Oracle(L, NB, tbc=tbc, kappa=KAPPA)
    o.set_fields(U, C)
    lat = qws_b200.Lattice(L, NB, tbc=tbc, kappa=KAPPA)
    try:
        lat.load_fields(U, C)
        b = qws_b200.gen_source(L, 5, "gauss")
        bs = b.astype(np.float32)
        assert rel(lat.to_host(lat.ddd(lat.to_device(b))), o.ddd_d(b)) < 1e-13
        assert rel(lat.to_host(lat.ddd(lat.to_device(bs))), o.ddd_s(bs)) < 1e-6
        assert rel(lat.to_host(lat.prec_ddd(lat.to_device(bs), 4, 2)), o.prec_ddd_s(bs, 4, 2)) < 5e-6
        xo, stats, _ = o.bicgstab_dd_mix(b, np.zeros_like(b), 1e-12, 50, 1e-6, 50, 4, 2)
        x = lat.empty("f64")
        bd = lat.to_device(b)
        st = lat.bicgstab_dd_mix(x, bd, 1e-12, 50, 1e-6, 50, 4, 2)
        assert abs(st["outer_iters"] - stats[0]) <= 1
        assert lat.true_residual(x, bd) < 1e-12
        assert rel(lat.to_host(x), xo) < 1e-10
    finally:
        lat.close()


def test_32_rhs_bit_equal():
    import qws_b200

    L = (8, 4, 4, 8)
    U, C = fields(L)
    lat = qws_b200.Lattice(L, (2, 2, 2, 2), tbc=-1, kappa=KAPPA)
    B = None
    try:
        lat.load_fields(U, C)
        B = lat.batch(32)
        S = np.stack([qws_b200.gen_source(L, 100 + k, "gauss") for k in range(32)]).astype(np.float32)
        got_h = B.to_host(B.prec_h(B.to_device(S), 4, 2))
        got_d = B.to_host(B.ddd(B.to_device(S.astype(np.float64))))
        for k in (0, 13, 31):
            assert np.array_equal(got_h[k], lat.to_host(lat.prec_h(lat.to_device(S[k]), 4, 2)))
            assert np.array_equal(got_d[k], lat.to_host(lat.ddd(lat.to_device(S[k].astype(np.float64)))))
    finally:
        if B is not None:
            B.close()
        lat.close()


def test_zero_source():
    """x = 0 for b = 0 (no division by the zero norm), in both solvers."""
    import qws_b200

    L = (8, 4, 4, 8)
    U, C = fields(L)
    lat = qws_b200.Lattice(L, (2, 2, 2, 2), tbc=-1, kappa=KAPPA)
    try:
        lat.load_fields(U, C)
        b = lat.empty("f64")
        for solve in (lambda x: lat.bicgstab_dd_mix(x, b, 1e-10, 20, 1e-6, 50, 4, 2),
                      lambda x: lat.bicgstab_dd_mix2_hf(x, b, 1e-10, 20, 1e-6, 50, 4, 2, reliable=5)):
            x = lat.empty("f64")
            solve(x)
            assert np.isfinite(lat.to_host(x)).all() and not lat.to_host(x).any()
    finally:
        lat.close()


@pytest.mark.parametrize("L,NB,nr", [
    ((8, 4, 4, 8), (1, 1, 1, 1), 1),   # NB[0] odd: the reference has two x-halves per rank
    ((8, 4, 4, 8), (2, 3, 1, 1), 1),   # 4 not divisible by 3
    ((8, 4, 4, 8), (2, 1, 1, 1), 3),   # RHS count not a power of two
    ((8, 4, 4, 8), (2, 1, 1, 1), 64),  # more than 32 RHS
])
def test_rejected(L, NB, nr):
    import qws_b200

    with pytest.raises(qws_b200.QwsgError):
        lat = qws_b200.Lattice(L, NB, tbc=-1, kappa=KAPPA)
        try:
            lat.batch(nr).close()
        finally:
            lat.close()


def test_forced_breakdown_matches_oracle():
    """<r0, q> = 0 at the first outer iteration, planted on the host in both
    the GPU solver (qwsg_inject_breakdown) and the oracle: the reference's
    guard (alpha = 0, bicgstab_dd_mix.cc:192) keeps x and r for that half
    step, the omega half step goes on, and both still converge with the same
    outer count (+-1) to the same solution."""
    import qws_b200
    from qwsref import load_oracle

    L, NB = (8, 4, 4, 8), (2, 1, 1, 1)
    U, C = fields(L)
    b = qws_b200.gen_source(L, 9)
    o = Oracle(L, NB, tbc=-1, kappa=KAPPA)
    o.set_fields(U, C)
    lib = load_oracle()
    lib.orc_plant_breakdown(1)
    try:
        xo, so, _ = o.bicgstab_dd_mix(b, np.zeros_like(b), 1e-12, 30, 1e-6, 50, 4, 2)
    finally:
        lib.orc_plant_breakdown(0)
    xo_clean, so_clean, _ = o.bicgstab_dd_mix(b, np.zeros_like(b), 1e-12, 30, 1e-6, 50, 4, 2)
    lat = qws_b200.Lattice(L, NB, tbc=-1, kappa=KAPPA)
    try:
        lat.load_fields(U, C)
        bd, x = lat.to_device(b), lat.empty("f64")
        lat.inject_breakdown(1)
        st = lat.bicgstab_dd_mix(x, bd, 1e-12, 30, 1e-6, 50, 4, 2)
        lat.inject_breakdown(0)
        assert abs(st["outer_iters"] - so[0]) <= 1
        assert so[0] >= so_clean[0]  # the lost half step costs iterations, not the answer
        assert np.isfinite(lat.to_host(x)).all()
        assert lat.true_residual(x, bd) < 1e-11
        assert rel(lat.to_host(x), xo) < 1e-10
    finally:
        lat.close()


def test_nan_source_fails_cleanly():
    """A source holding a NaN makes the residual non-finite: the solve
    returns error code 3 (no NaN solution is handed back as a result), and
    the handle and the device stay usable for the next solve."""
    import qws_b200

    L, NB = (8, 4, 4, 8), (2, 1, 1, 1)
    U, C = fields(L)
    b = qws_b200.gen_source(L, 9)
    lat = qws_b200.Lattice(L, NB, tbc=-1, kappa=KAPPA)
    try:
        lat.load_fields(U, C)
        bad = b.copy()
        bad[5, 3] = np.nan
        x = lat.empty("f64")
        with pytest.raises(qws_b200.QwsgError, match="non-finite"):
            lat.bicgstab_dd_mix(x, lat.to_device(bad), 1e-10, 30, 1e-6, 50, 4, 2)
        with pytest.raises(qws_b200.QwsgError, match="non-finite"):
            lat.bicgstab_dd_mix2_hf(x, lat.to_device(bad), 1e-10, 30, 1e-6, 50, 4, 2, reliable=3)
        x.zero_()
        bd = lat.to_device(b)
        st = lat.bicgstab_dd_mix(x, bd, 1e-10, 30, 1e-6, 50, 4, 2)
        assert st["outer_iters"] < 30 and lat.true_residual(x, bd) < 1e-10
    finally:
        lat.close()
