"""Vector-level comparison of the CPU oracle with the reference's own
sources compiled by oracle/Makefile (oracle/_ref/<variant>/libqwsref.so).

Skipped where the prebuilt reference library is absent.  Tolerances: FP64
operators at 1e-13 relative (norm of the difference over the norm), FP32
single operators at a few units of FP32 roundoff, the SAP preconditioner
(about 15 Dirac applications in FP32) at 5e-6.
"""
import ctypes

import numpy as np
import pytest

from qwsref import Oracle, RefQWS, aligned_empty, gen_main_fields, ref_variant_path

VARIANT = "v8s16"
pytestmark = pytest.mark.skipif(not ref_variant_path(VARIANT).exists(),
                                reason="oracle/_ref not built (make -C oracle ref)")

L = (32, 6, 4, 3)
KAPPA = 0.05


def rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def setup():
    U, C, S = gen_main_fields(L, (1, 1, 1, 1), 2)
    o = Oracle(L, (2, 1, 1, 1), tbc=-1, kappa=KAPPA)
    o.set_fields(U, C)
    r = RefQWS(VARIANT, L, tbc=-1)
    r.set_kappa(KAPPA)
    r.set_fields(U, C)
    return o, r, S[0]


def test_ddd_d_and_s(setup):
    o, r, b = setup
    out = aligned_empty(b.size, np.float64)
    r.call("ddd_d_", out, r.to_d(b))
    assert rel(r.from_d(out), o.ddd_d(b)) < 1e-13
    bs = b.astype(np.float32)
    out = aligned_empty(b.size, np.float32)
    r.call("ddd_s_", out, r.to_s(bs))
    assert rel(r.from_s(out), o.ddd_s(bs)) < 5e-7


def test_sap_preconditioner(setup):
    o, r, b = setup
    bs = b.astype(np.float32)
    nsap, nm = ctypes.c_int(4), ctypes.c_int(2)
    out = aligned_empty(b.size, np.float32)
    r.call("prec_ddd_s_", out, r.to_s(bs), ctypes.byref(nsap), ctypes.byref(nm))
    assert rel(r.from_s(out), o.prec_ddd_s(bs, 4, 2)) < 5e-6
    out = aligned_empty(b.size, np.float32)
    r.call("prec_s_", out, r.to_s(bs), ctypes.byref(nsap), ctypes.byref(nm))
    assert rel(r.from_s(out), o.prec_s(bs, 4, 2)) < 5e-6


def test_jinv(setup):
    o, r, b = setup
    bs = b.astype(np.float32)
    xo = aligned_empty(b.size, np.float32)
    xo[:] = 0
    r.call("jinv_ddd_in_s_", xo, r.to_s(bs), ctypes.byref(ctypes.c_int(0)),
           ctypes.byref(ctypes.c_int(2)))
    mask = (np.arange(o.V) % L[0]) < L[0] // 2  # domain 0 = x-half 0
    assert rel(r.from_s(xo)[mask], o.jinv_s(bs, 0, 2)[mask]) < 1e-6


def test_mixed_solver(setup):
    o, r, b = setup
    x0 = np.zeros_like(b)
    xr, bb = r.to_d(x0), r.to_d(b)
    conv = ctypes.c_int(0)
    r.call("bicgstab_dd_mix_", xr, bb, ctypes.byref(ctypes.c_double(1e-12)), ctypes.byref(conv),
           ctypes.byref(ctypes.c_int(20)), ctypes.byref(ctypes.c_double(1e-6)),
           ctypes.byref(ctypes.c_int(50)), ctypes.byref(ctypes.c_int(4)),
           ctypes.byref(ctypes.c_int(2)))
    xo, stats, _ = o.bicgstab_dd_mix(b, x0, 1e-12, 20, 1e-6, 50, 4, 2)
    assert abs(conv.value - stats[0]) <= 1
    assert rel(r.from_d(xr), xo) < 1e-11


def test_bqcd_loaders_match_reference(setup):
    """The reference's own loaders (qws_bqcd.cc:66-642) on arrays made by
    qwsref's nat_to_bqcd_* helpers: the DD loaders give the DD layout of the
    natural fields; the even-odd loaders give the layout whose even-odd
    reading (eo_perm) is the natural field.  This pins the BQCD-format
    helpers the drop-in tests feed to this library's loaders."""
    from qwsref import (eo_perm, nat_to_bqcd_clover, nat_to_bqcd_gauge, nat_to_bqcd_spinor,
                        nat_to_qws_clover, nat_to_qws_gauge, nat_to_qws_spinor)

    o, r, b = setup
    U, C, _ = gen_main_fields(L, (1, 1, 1, 1), 2)
    V = int(np.prod(L))
    volh = ctypes.c_int(V // 2)
    kap = ctypes.c_double(KAPPA)
    u, c = nat_to_bqcd_gauge(U, L), nat_to_bqcd_clover(C, L)

    def glob(name, dt):
        ct = ctypes.c_double if dt == np.float64 else ctypes.c_float
        return np.ctypeslib.as_array((ct * (72 * V)).from_address(r._global_ptr(name))).copy()

    def expect(Un, Cn):
        return {"glud": nat_to_qws_gauge(Un, L, r.vlend), "clvd": nat_to_qws_clover(Cn, L, r.vlend),
                "glus": nat_to_qws_gauge(Un, L, r.vlens).astype(np.float32),
                "clvs": nat_to_qws_clover(Cn, L, r.vlens).astype(np.float32)}

    try:
        r.lib.qws_loadg_dd_(ctypes.c_void_p(u.ctypes.data), ctypes.byref(volh), ctypes.byref(kap))
        r.lib.qws_loadc_dd_(ctypes.c_void_p(c.ctypes.data), ctypes.byref(volh))
        for name, want in expect(U, C).items():
            np.testing.assert_array_equal(glob(name, want.dtype), want, err_msg=name)
        P = eo_perm(L)
        Ud, Cd = np.zeros_like(U), np.zeros_like(C)
        Ud[:, P], Cd[P] = U, C
        r.lib.qws_loadg_bqcd_(ctypes.c_void_p(u.ctypes.data), ctypes.byref(volh),
                              ctypes.byref(kap))
        r.lib.qws_loadc_bqcd_(ctypes.c_void_p(c.ctypes.data), ctypes.byref(volh))
        for name, want in expect(Ud, Cd).items():
            np.testing.assert_array_equal(glob(name, want.dtype), want, err_msg=name)
        # spinors: the DD pair loader, and the even sites into a half array
        e, od = nat_to_bqcd_spinor(b, L)
        q = aligned_empty(24 * V, np.float64)
        r.lib.qws_loadfd_dd_(ctypes.c_void_p(q.ctypes.data), ctypes.c_void_p(e.ctypes.data),
                             ctypes.c_void_p(od.ctypes.data))
        np.testing.assert_array_equal(q, nat_to_qws_spinor(b, L, r.vlend))
        q[:] = 0
        r.lib.qws_loadfd_bqcd_(ctypes.c_void_p(q.ctypes.data), ctypes.c_void_p(e.ctypes.data))
        bd = np.zeros_like(b)
        bd[P] = b
        np.testing.assert_array_equal(q[:12 * V], nat_to_qws_spinor(bd, L, r.vlend)[:12 * V])
    finally:
        r.set_kappa(KAPPA)
        r.set_fields(U, C)


def test_cg_solvers_match_reference(setup):
    """cg_vm_ (cg.cc:65) and mcg_vm_ (mcg.cc:65) of the reference against
    the oracle's restatements, driven as main.cc drives the even-odd family:
    the DD arrays are read with the parity split (eo_perm), the source is the
    first half array read as a parity-0 field.  Solutions agree to 1e-11
    relative on the even sites (both stop at |r|/|b| < 1e-14)."""
    from qwsref import eo_perm, parity_mask

    o, r, _ = setup
    U, C, S = gen_main_fields(L, (1, 1, 1, 1), 2)
    P, m0 = eo_perm(L), parity_mask(L, 0)
    oe = Oracle(L, (2, 1, 1, 1), tbc=-1, kappa=KAPPA)
    oe.set_fields(U[:, P], C[P])
    V = int(np.prod(L))
    half = 12 * V  # reals of one half array
    bfull = r.to_d(S[0])
    be = S[0][P] * m0[:, None]

    def eo_field(h):
        q = aligned_empty(24 * V, np.float64)
        q[:] = 0
        q[:half] = h
        return r.from_d(q)[P] * m0[:, None]

    x = aligned_empty(half, np.float64)
    x[:] = 0
    # main.cc's links are not unitary: CG on mtdagmt needs about 1100 iterations
    r.call("cg_vm_", x, bfull, ctypes.byref(ctypes.c_int(0)), ctypes.byref(ctypes.c_int(2000)))
    xo, it = oe.cg_vm(be, np.zeros_like(be), 2000)
    assert 1 < it < 1999
    assert rel(eo_field(x)[m0], xo[m0]) < 1e-11

    sigma = np.array([0.0, 0.01, 0.2, 1.5])
    xx = aligned_empty(len(sigma) * half, np.float64)
    xx[:] = 0
    r.call("mcg_vm_", xx, bfull, ctypes.byref(ctypes.c_int(len(sigma))),
           sigma.ctypes.data_as(ctypes.c_void_p), ctypes.byref(ctypes.c_int(2000)))
    Xo, it = oe.mcg_vm(be, sigma, 2000)
    assert 1 < it < 1999
    # shifts 0 and 0.01 run to the end in the reference too; the larger ones
    # converge early, after which the reference's zeta underflows (0/0 = NaN)
    # while the oracle has stopped updating them
    finite = [bool(np.isfinite(xx[k * half:(k + 1) * half]).all()) for k in range(len(sigma))]
    assert finite[0] and finite[1]
    for k in range(len(sigma)):
        if finite[k]:
            assert rel(eo_field(xx[k * half:(k + 1) * half])[m0], Xo[k][m0]) < 1e-11, k
    # the shifted systems are solved: (mtdagmt + sigma) x_k = b on the even sites
    for k, s in enumerate(sigma):
        assert rel((oe.mtdagmt(Xo[k]) + s * Xo[k])[m0], be[m0]) < 1e-10, k
