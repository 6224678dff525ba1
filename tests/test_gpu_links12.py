"""FP32 links in 12-real form (qwsg_set_link_compression): used only when
every link is SU(3) to 1e-5, and then the FP32 operators stay within FP32
rounding of the oracle and of the 18-real path (the rebuilt third row
differs from the stored one by a few FP32 ulp); the reference's own test
fields (main.cc's Gaussian, non-unitary links) keep the 18-real path; the
DD solve converges to the same solution."""
import numpy as np
import pytest

from qwsref import Oracle, gen_main_fields

pytestmark = pytest.mark.gpu

L = (8, 8, 8, 16)
KAPPA, CSW = 0.1365, 1.7


def rel(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def su3():
    import qws_b200

    U, _ = qws_b200.gen_gauge(L, 7, 5, 0.36)
    C = qws_b200.gen_clover(U, L, CSW, KAPPA)
    b = qws_b200.gen_source(L, 4, "gauss")
    o = Oracle(L, (2, 2, 2, 2), tbc=-1, kappa=KAPPA)
    o.set_fields(U, C)
    on = qws_b200.Lattice(L, (2, 2, 2, 2), tbc=-1, kappa=KAPPA)
    on.load_fields(U, C)
    off = qws_b200.Lattice(L, (2, 2, 2, 2), tbc=-1, kappa=KAPPA)
    off.set_link_compression(0)
    off.load_fields(U, C)
    yield o, on, off, b
    on.close()
    off.close()


def test_used_only_for_su3(su3):
    import qws_b200

    _, on, off, _ = su3
    assert on.link_compression() and not off.link_compression()
    Lc = (32, 6, 4, 3)
    U, C, _ = gen_main_fields(Lc, (1, 1, 1, 1), 2)
    lat = qws_b200.Lattice(Lc, (2, 1, 1, 1), tbc=-1, kappa=0.05)
    try:
        lat.load_fields(U, C)
        assert not lat.link_compression()
    finally:
        lat.close()


def test_operators(su3):
    o, on, off, b = su3
    bs = b.astype(np.float32)
    for name, f_on, f_off, ref in (
            ("ddd_s", lambda: on.ddd(on.to_device(bs)), lambda: off.ddd(off.to_device(bs)),
             o.ddd_s(bs)),
            ("prec_ddd", lambda: on.prec_ddd(on.to_device(bs), 4, 2),
             lambda: off.prec_ddd(off.to_device(bs), 4, 2), o.prec_ddd_s(bs, 4, 2))):
        got_on, got_off = on.to_host(f_on()), off.to_host(f_off())
        assert rel(got_on, got_off) < 2e-6, name
        assert rel(got_on, ref) < 5e-6, name
    # FP64 operators never use the 12-real links
    assert np.array_equal(on.to_host(on.ddd(on.to_device(b))), off.to_host(off.ddd(off.to_device(b))))


def test_solve(su3):
    o, on, off, b = su3
    xo, stats, _ = o.bicgstab_dd_mix(b, np.zeros_like(b), 1e-12, 50, 1e-6, 50, 4, 2)
    bd = on.to_device(b)
    x = on.empty("f64")
    st = on.bicgstab_dd_mix(x, bd, 1e-12, 50, 1e-6, 50, 4, 2)
    assert abs(st["outer_iters"] - stats[0]) <= 1
    assert on.true_residual(x, bd) < 1e-12
    assert rel(on.to_host(x), xo) < 1e-10
