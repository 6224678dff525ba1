"""Fields built on the GPU against the host generators that follow the same
conventions: the clover term (qwsg_build_clover vs qwsg_gen_clover) and the
seeded smoothed gauge field (qwsg_gen_gauge_device vs qwsg_gen_gauge).  The
FP64 operator with either field agrees to 1e-13 / 1e-12, the FP32 one to
FP32 rounding, and a solve gives the same iterations.  The free field
(U = 1, F = 0) must give the trivial clover term 1/2 on the diagonal.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L = (8, 8, 8, 16)
KAPPA, CSW = 0.1365, 1.7


def rel(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("NB", [(2, 1, 1, 1), (2, 2, 2, 2)])
def test_device_clover_matches_host(NB):
    import qws_b200

    U, _ = qws_b200.gen_gauge(L, 5, 5, 0.36)
    C = qws_b200.gen_clover(U, L, CSW, KAPPA)
    b = qws_b200.gen_source(L, 9)
    host = qws_b200.Lattice(L, NB, tbc=-1, kappa=KAPPA)
    dev = qws_b200.Lattice(L, NB, tbc=-1, kappa=KAPPA)
    try:
        host.load_fields(U, C)
        dev.load_gauge(U)
        dev.build_clover(CSW)
        for dt, tol in ((np.float64, 1e-13), (np.float32, 1e-6)):
            x = b.astype(dt)
            assert rel(dev.to_host(dev.ddd(dev.to_device(x))),
                       host.to_host(host.ddd(host.to_device(x)))) < tol, dt
        xs = [lat.empty("f64") for lat in (host, dev)]
        st = [lat.bicgstab_dd_mix(x, lat.to_device(b), 1e-10, 100, 1e-6, 50)
              for lat, x in zip((host, dev), xs)]
        assert abs(st[0]["outer_iters"] - st[1]["outer_iters"]) <= 1
        assert rel(dev.to_host(xs[1]), host.to_host(xs[0])) < 1e-8
    finally:
        host.close()
        dev.close()


def test_free_field_clover_is_trivial():
    import qws_b200

    V = int(np.prod(L))
    U = np.zeros((4, V, 3, 3, 2))
    for c in range(3):
        U[:, :, c, c, 0] = 1.0
    lat = qws_b200.Lattice(L, (2, 2, 2, 2), tbc=-1, kappa=KAPPA)
    ref = qws_b200.Lattice(L, (2, 2, 2, 2), tbc=-1, kappa=KAPPA)
    try:
        lat.load_gauge(U)
        lat.build_clover(CSW)
        C = np.zeros((V, 72))
        C[:, 0:6] = 0.5
        C[:, 36:42] = 0.5
        ref.load_fields(U, C)
        b = qws_b200.gen_source(L, 3)
        got = lat.to_host(lat.ddd(lat.to_device(b)))
        want = ref.to_host(ref.ddd(ref.to_device(b)))
        assert rel(got, want) < 1e-15
    finally:
        lat.close()
        ref.close()


def test_device_gauge_matches_host():
    """qwsg_gen_gauge_device draws the same random streams and applies the same
    smoothing as the host generator: the operators built on the two fields
    agree to rounding, and so do the plaquettes."""
    import qws_b200

    U, plaq = qws_b200.gen_gauge(L, 21, 5, 0.36)
    host = qws_b200.Lattice(L, (2, 2, 2, 2), tbc=-1, kappa=KAPPA)
    dev = qws_b200.Lattice(L, (2, 2, 2, 2), tbc=-1, kappa=KAPPA)
    try:
        host.load_gauge(U)
        p = dev.gen_gauge_device(21, 5, 0.36)
        assert abs(p - plaq) < 1e-12, (p, plaq)
        host.build_clover(CSW)
        dev.build_clover(CSW)
        b = qws_b200.gen_source(L, 4)
        assert rel(dev.to_host(dev.ddd(dev.to_device(b))),
                   host.to_host(host.ddd(host.to_device(b)))) < 1e-12
    finally:
        host.close()
        dev.close()
