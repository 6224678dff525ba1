"""Pin the CPU oracle against the reference's own golden files (data/CASE*,
extracted into tests/golden/case_norms.json by tests/golden/make_golden.py)
under check.sh's tolerances (check.sh:17-26).

Multi-rank goldens (CASE1-9) are reproduced on one lattice: every rank seeds
mt19937(12345) identically (main.cc:129), so the global field is the local
field tiled over the rank grid, and the reference's SAP blocks are the
x-halves of each rank's local volume (block grid NB = (2*px, py, pz, pt)).
"""
import json
from pathlib import Path

import numpy as np
import pytest

from qwsref import Oracle, check_sh_ok, gen_main_fields

GOLD = json.loads((Path(__file__).parent / "golden" / "case_norms.json").read_text())
KAPPA = 0.05  # main.cc:173


def _setup(case):
    g = GOLD[case]
    lloc, npe = g["lloc"], g["npe"]
    U, C, S = gen_main_fields(lloc, npe, 2)
    L = [a * b for a, b in zip(lloc, npe)]
    NB = (2 * npe[0], npe[1], npe[2], npe[3])
    o = Oracle(L, NB, tbc=-1, kappa=KAPPA)
    o.set_fields(U, C)
    return g, o, S[0], S[1]


def _golden(g, name, which=-1):
    vals = [v for k, v in g["norms"] if k == name]
    return vals[which]


def _dd_operator_norms(o, b):
    bs = b.astype(np.float32)
    n2 = lambda a: float(np.sum(np.asarray(a, np.float64) ** 2))
    return {
        "ddd_out_pre|pos_d_": n2(o.ddd_out_d(b, 1, 0, -KAPPA)),
        "ddd_in_d_": n2(o.ddd_in_d(b, 1, 0)),
        "ddd_d_": n2(o.ddd_d(b)),
        # kind 2: the FP32 face packer's x-half pairing with a fixed domain
        "ddd_out_pre|pos_s_": n2(o.ddd_out_s(bs, 2, 0, np.float32(-KAPPA))),
        "ddd_in_s_": n2(o.ddd_in_s(bs, 1, 0)),
        "ddd_s_": n2(o.ddd_s(bs)),
    }


@pytest.mark.parametrize("case", ["CASE0", "CASE_4111_1111", "CASE1", "CASE2", "CASE3",
                                  "CASE4", "CASE5", "CASE6", "CASE7", "CASE8", "CASE9"])
def test_dd_operator_norms(case):
    g, o, b, _ = _setup(case)
    assert check_sh_ok("input", float(np.sum(b * b)), _golden(g, "input"))
    for name, val in _dd_operator_norms(o, b).items():
        ref = _golden(g, name)
        assert check_sh_ok(name, val, ref), (name, val, ref)


@pytest.mark.parametrize("case", ["CASE0", "CASE_4111_1111"])
def test_dd_solve_norms(case):
    """bicgstab_dd_mix_ with tol<0: 5 outer x 2 inner solves x 50 iterations,
    nsap=4, nm=2 (main.cc:258-313), then the true residual with ddd_d_."""
    g, o, b, x0 = _setup(case)
    a = g["args"]
    x, stats, hist = o.bicgstab_dd_mix(b, x0, a["tol"], a["maxiter"], a["tol_s"],
                                       a["maxiter_s"], a["nsap"], a["nm"])
    assert stats[0] == a["maxiter"]       # loop runs iter=1..maxiter-1
    assert stats[1] == 10 * a["maxiter_s"]  # 10 inner solves x 50 (data/CASE0:67-83)
    r = b - o.ddd_d(x)
    got = {"bnorm^2": float(np.sum(b * b)), "rnorm^2": float(np.sum(r * r)),
           "xnorm^2": float(np.sum(x * x))}
    for name, val in got.items():
        assert check_sh_ok(name, val, _golden(g, name)), (name, val, _golden(g, name))


@pytest.mark.slow
@pytest.mark.parametrize("case", ["CASE1", "CASE7"])
def test_dd_solve_norms_rank_grid(case):
    g, o, b, x0 = _setup(case)
    a = g["args"]
    x, stats, _ = o.bicgstab_dd_mix(b, x0, a["tol"], a["maxiter"], a["tol_s"],
                                    a["maxiter_s"], a["nsap"], a["nm"])
    r = b - o.ddd_d(x)
    for name, val in (("bnorm^2", np.sum(b * b)), ("rnorm^2", np.sum(r * r)),
                      ("xnorm^2", np.sum(x * x))):
        assert check_sh_ok(name, float(val), _golden(g, name))


# ---------------------------------------------------------------------------
# even-odd family (deo_*, mtilde, bicgstab_vm_) on CASE0 (main.cc:584-721)
# ---------------------------------------------------------------------------
def _eo_setup():
    from qwsref import eo_partner, eo_perm, parity_mask

    g = GOLD["CASE0"]
    L = tuple(g["lloc"])
    U, C, S = gen_main_fields(L, (1, 1, 1, 1), 2)
    P, Q = eo_perm(L), eo_partner(L)
    o = Oracle(L, (2, 1, 1, 1), tbc=-1, kappa=KAPPA)
    o.set_fields(U[:, P], C[P])
    return g, o, S[0][P], Q, parity_mask(L, 0), parity_mask(L, 1)


def test_eo_operator_norms_case0():
    g, o, b, Q, m0, m1 = _eo_setup()
    fac = -KAPPA * KAPPA
    n2 = lambda a, m: float(np.sum(np.asarray(a, np.float64)[m] ** 2))
    in0 = b[Q]  # main.cc passes in0 = in: parity-1 outputs read the parity-0 half
    got = {
        "deo_in_vm_": n2(o.deo(b, 1, 1, 0, 0, 0), m1),
        "dee_deo_in_vm_": n2(o.deo(b, 1, 1, 0, 1, 0), m1),
        "deo_dag_in_vm_": n2(o.deo(b, 1, 1, 1, 0, 0), m1),
        "dee_deo_dag_in_vm_": n2(o.deo(b, 1, 1, 1, 1, 0), m1),
        "one_minus_dee_deo_in_vm_": n2(o.deo(b, 1, 1, 0, 1, 2, fac, in0), m1),
        "one_minus_deo_dag_in_vm_": n2(o.deo(b, 1, 1, 1, 0, 2, fac, in0), m1),
        "deo_out_pre|pos_vm_": n2(o.deo(b, 1, 2, 0, 0, 1, fac), m1),
        "deo_dag_out_pre|pos_vm_": n2(o.deo(b, 1, 2, 1, 0, 1, fac), m1),
        "dee_deo_out_pre|pos_vm_": n2(o.deo(b, 1, 2, 0, 1, 1, fac), m1),
        "dee_deo_dag_out_pre|pos_vm_": n2(o.deo(b, 1, 2, 1, 1, 1, fac), m1),
        "clvd_vm_": n2(o.clv(b, 0), m0),
        "deo_vm_": n2(o.deo(b, 1, 3, 0, 0, 0), m1),
        "dee_deo_vm_": n2(o.deo(b, 1, 3, 0, 1, 0), m1),
        "one_minus_dee_deo_vm_": n2(o.deo(b, 1, 3, 0, 1, 2, fac, in0), m1),
        "deo_dag_vm_": n2(o.deo(b, 1, 3, 1, 0, 0), m1),
        "dee_deo_dag_vm_": n2(o.deo(b, 1, 3, 1, 1, 0), m1),
        "one_minus_deo_dag_vm_": n2(o.deo(b, 1, 3, 1, 0, 2, fac, in0), m1),
        "mtilde_vm_": n2(o.mtilde(b), m0),
        "mtilde_dag_vm_": n2(o.mtilde(b, True), m0),
        "mtdagmt_vm_": n2(o.mtilde(o.mtilde(b), True), m0),
    }
    bs = b.astype(np.float32)
    fs = np.float32(fac)
    tmp = o.deo(bs, 1, 3, 0, 1, 0)  # dee_deo_s_(pco, pce, tmp, in)
    got.update({
        "deo_in_s_": n2(o.deo(bs, 1, 1, 0, 0, 0), m1),
        "dee_deo_in_s_": n2(o.deo(bs, 1, 1, 0, 1, 0), m1),
        "one_minus_dee_deo_in_s_": n2(o.deo(bs, 1, 1, 0, 1, 2, fs, bs[Q]), m1),
        "deo_out_pre|pos_s_": n2(o.deo(bs, 1, 2, 0, 0, 1, fs), m1),
        "dee_deo_out_pre|pos_s_": n2(o.deo(bs, 1, 2, 0, 1, 1, fs), m1),
        "clv_s_": n2(o.clv(bs, 0), m0),
        "deo_s_": n2(o.deo(bs, 1, 3, 0, 0, 0), m1),
        "dee_deo_s_": n2(o.deo(bs, 1, 3, 0, 1, 0), m1),
        "one_minus_dee_deo_s_": n2(o.deo(bs, 1, 3, 0, 1, 2, fs, bs[Q]), m1),
        "mtilde_s_": n2(o.deo(tmp, 0, 3, 0, 1, 2, fs, bs), m0),
    })
    for name, val in got.items():
        ref = _golden(g, name)
        assert check_sh_ok(name, val, ref), (name, val, ref)


def test_eo_solve_case0():
    """bicgstab_vm_ (bicgstab.cc:68): 91 iterations on CASE0 (the golden's
    timing table counts 91 bicgstab_iter_ calls), then the true residual."""
    g, o, b, Q, m0, m1 = _eo_setup()
    be = b * m0[:, None]
    x, it = o.bicgstab_vm(be, np.zeros_like(b), 100)
    assert it == 91
    r = be - o.mtilde(x)
    n2 = lambda a: float(np.sum(a[m0] ** 2))
    vals = [v for k, v in g["norms"] if k in ("bnorm^2", "rnorm^2", "xnorm^2")][:3]
    for name, val, ref in zip(("bnorm^2", "rnorm^2", "xnorm^2"), (n2(be), n2(r), n2(x)), vals):
        assert check_sh_ok(name, val, ref), (name, val, ref)
