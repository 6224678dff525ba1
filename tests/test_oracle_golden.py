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
                                  "CASE4", "CASE7", "CASE8", "CASE9"])
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
