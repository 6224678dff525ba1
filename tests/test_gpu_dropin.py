"""The drop-in C ABI (include/qws_dropin.h) driven the way the reference's
main.cc drives QWS: qws_init_, then the host globals glud/glus/clvd/clvs and
kappa written directly in QWS's SIMD-lane layout (main.cc:168-175, 416-518),
then the reference-named entry points on host arrays.  Results are compared
with the CPU oracle and with the reference's CASE0 golden norms.
"""
import ctypes
import json
from pathlib import Path

import numpy as np
import pytest

from qwsref import (Oracle, aligned_empty, check_sh_ok, gen_main_fields, nat_to_qws_clover,
                    nat_to_qws_gauge, nat_to_qws_spinor, qws_to_nat_spinor)

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parents[1]
GOLD = json.loads((REPO / "tests" / "golden" / "case_norms.json").read_text())
L = (32, 6, 4, 3)
VLEND, VLENS = 8, 16
KAPPA = 0.05


def rel(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def qws():
    import qws_b200

    lib = qws_b200.load_library()
    U, C, S = gen_main_fields(L, (1, 1, 1, 1), 2)
    args = [ctypes.byref(ctypes.c_int(v)) for v in L]
    npe = (ctypes.c_int * 4)(1, 1, 1, 1)
    fbc = (ctypes.c_int * 4)(1, 1, 1, -1)
    pce, pco = ctypes.c_int(0), ctypes.c_int(1)
    bs = (ctypes.c_int * 4)(1, 2, 2, 2)
    assert lib.qwsg_set_host_vlen(VLEND, VLENS) == 0
    lib.qws_init_(*args, npe, fbc, ctypes.byref(pce), ctypes.byref(pco), bs)
    ctypes.c_double.in_dll(lib, "kappa").value = KAPPA
    ctypes.c_double.in_dll(lib, "mkappa").value = -KAPPA
    ctypes.c_double.in_dll(lib, "kappa2").value = KAPPA * KAPPA
    for name, arr in (("glud", nat_to_qws_gauge(U, L, VLEND)),
                      ("clvd", nat_to_qws_clover(C, L, VLEND)),
                      ("glus", nat_to_qws_gauge(U, L, VLENS).astype(np.float32)),
                      ("clvs", nat_to_qws_clover(C, L, VLENS).astype(np.float32))):
        ptr = ctypes.c_void_p.in_dll(lib, name).value
        ctypes.memmove(ptr, arr.ctypes.data, arr.nbytes)
    lib.qwsg_mark_fields_dirty()
    o = Oracle(L, (2, 1, 1, 1), tbc=-1, kappa=KAPPA)
    o.set_fields(U, C)
    yield lib, o, S[0], S[1]
    lib.qws_finalize_()


def to_d(v):
    q = nat_to_qws_spinor(v, L, VLEND)
    a = aligned_empty(q.size, np.float64)
    a[:] = q
    return a


def to_s(v):
    q = nat_to_qws_spinor(np.asarray(v, np.float32), L, VLENS)
    a = aligned_empty(q.size, np.float32)
    a[:] = q
    return a


def P(a):
    """The address of `a` for a C call.  The pointer object holds a
    reference to `a`, so a temporary argument stays alive through the call
    (a bare c_void_p(a.ctypes.data) of a temporary points at memory Python
    frees as soon as this function returns)."""
    return a.ctypes.data_as(ctypes.c_void_p)


def test_globals(qws):
    lib, o, b, _ = qws
    assert ctypes.c_int.in_dll(lib, "vold").value == 16 // VLEND * 6 * 4 * 3
    assert ctypes.c_int.in_dll(lib, "vols").value == 16 // VLENS * 6 * 4 * 3
    assert ctypes.c_int.in_dll(lib, "nxh").value == 16


def test_ddd(qws):
    lib, o, b, _ = qws
    out = aligned_empty(b.size, np.float64)
    bd = to_d(b)
    lib.ddd_d_(P(out), P(bd))
    assert rel(qws_to_nat_spinor(out, L, VLEND), o.ddd_d(b)) < 1e-13
    bs = b.astype(np.float32)
    out = aligned_empty(b.size, np.float32)
    bq = to_s(bs)
    lib.ddd_s_(P(out), P(bq))
    assert rel(qws_to_nat_spinor(out, L, VLENS), o.ddd_s(bs)) < 1e-6


def test_ddd_in_out_domain0(qws):
    """main.cc:775-784: ddd_in_d_/ddd_out_pre|pos_d_ with DEO = 0 on full arrays."""
    lib, o, b, _ = qws
    deo = ctypes.byref(ctypes.c_int(0))
    out = aligned_empty(b.size, np.float64)
    out[:] = 0
    bd = to_d(b)
    lib.ddd_in_d_(P(out), P(bd), deo)
    g = GOLD["CASE0"]["norms"]
    val = float(np.sum(out.astype(np.float64) ** 2))
    assert check_sh_ok("ddd_in_d_", val, dict(g)["ddd_in_d_"])
    out[:] = 0
    bq = to_d(b)
    lib.ddd_out_pre_d_(P(bq), deo)
    lib.ddd_out_pos_d_(P(out), P(bq), deo)
    val = float(np.sum(out ** 2))
    assert check_sh_ok("ddd_out_pre|pos_d_", val, dict(g)["ddd_out_pre|pos_d_"])


def test_sap(qws):
    lib, o, b, _ = qws
    bs = b.astype(np.float32)
    nsap, nm = ctypes.c_int(4), ctypes.c_int(2)
    out = aligned_empty(b.size, np.float32)
    bq = to_s(bs)
    lib.prec_ddd_s_(P(out), P(bq), ctypes.byref(nsap), ctypes.byref(nm))
    assert rel(qws_to_nat_spinor(out, L, VLENS), o.prec_ddd_s(bs, 4, 2)) < 5e-6
    lib.prec_s_(P(out), P(bq), ctypes.byref(nsap), ctypes.byref(nm))
    assert rel(qws_to_nat_spinor(out, L, VLENS), o.prec_s(bs, 4, 2)) < 5e-6


def test_case0_dd_solve(qws):
    """The DD solve of main.cc:258-313 through bicgstab_dd_mix_, checked
    against data/CASE0 with check.sh's tolerances."""
    lib, o, b, x0 = qws
    x, bq = to_d(x0), to_d(b)
    it = ctypes.c_int(0)
    lib.bicgstab_dd_mix_(P(x), P(bq), ctypes.byref(ctypes.c_double(-1.0)), ctypes.byref(it),
                         ctypes.byref(ctypes.c_int(6)), ctypes.byref(ctypes.c_double(-1.0)),
                         ctypes.byref(ctypes.c_int(50)), ctypes.byref(ctypes.c_int(4)),
                         ctypes.byref(ctypes.c_int(2)))
    assert it.value == 6
    r = aligned_empty(b.size, np.float64)
    lib.ddd_d_(P(r), P(x))
    res = bq - r
    vals = [v for k, v in GOLD["CASE0"]["norms"] if k in ("bnorm^2", "rnorm^2", "xnorm^2")][-3:]
    for name, val, ref in zip(("bnorm^2", "rnorm^2", "xnorm^2"),
                              (np.sum(bq * bq), np.sum(res * res), np.sum(x * x)), vals):
        assert check_sh_ok(name, float(val), ref), (name, val, ref)


def test_loaders_roundtrip(qws):
    """qws_loadfd_dd_/qws_storefd_dd_ (qws_bqcd.cc:500-570) invert each other."""
    lib, o, b, _ = qws
    V = int(np.prod(L))
    rng = np.random.default_rng(3)
    ine, ino = rng.standard_normal(12 * V), rng.standard_normal(12 * V)
    q = aligned_empty(24 * V, np.float64)
    lib.qws_loadfd_dd_(P(q), P(ine), P(ino))
    oe, oo = np.zeros_like(ine), np.zeros_like(ino)
    lib.qws_storefd_dd_(P(oe), P(oo), P(q))
    np.testing.assert_array_equal(oe, ine)
    np.testing.assert_array_equal(oo, ino)
