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
