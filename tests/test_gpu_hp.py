"""GPU precision form: the SAP preconditioner in FP16 storage with per-site
FP32 scales (FP32 arithmetic), the flexible inner solver and the FP64 outer
loop of the reference's half-precision pair (prec_ddd_s_h.h:63,
bicgstab_precdd_s_h.cc:83, bicgstab_dd_mix2_hf.cc:110).

Tolerances: the FP16 SAP against the oracle's FP32 SAP of the same sweep
count (nsap-1 sweeps + final stage) at 1e-2 relative -- a few hundred FP16
unit roundoffs (2^-11 = 4.9e-4) accumulated over ~13 Dirac applications;
the solvers must reach their stated residuals, and the outer solution must
match the oracle's FP64 solve to 1e-9.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from qwsref import Oracle, check_sh_ok, gen_main_fields

pytestmark = pytest.mark.gpu

GOLD = json.loads((Path(__file__).parent / "golden" / "case_norms.json").read_text())
KAPPA = 0.05
# main.cc's fields on the lattices of the DD goldens: SAP blocks 16x6x4x3
# (one rank, and rank grids (1,2,2,2) and (1,1,4,4)), 16x3x4x4 (an odd
# extent) and 16x6x6x2 (two sites across)
CASES = {
    "CASE0": ((32, 6, 4, 3), (1, 1, 1, 1)),
    "CASE2": ((32, 3, 4, 4), (1, 1, 1, 2)),
    "CASE4": ((32, 6, 6, 2), (1, 1, 1, 2)),
    "CASE7": ((32, 6, 4, 3), (1, 2, 2, 2)),
    "CASE9": ((32, 6, 4, 3), (1, 1, 4, 4)),
}


def rel(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module", params=list(CASES))
def case(request):
    import qws_b200

    lloc, npe = CASES[request.param]
    L = tuple(a * b for a, b in zip(lloc, npe))
    NB = (2 * npe[0], npe[1], npe[2], npe[3])
    U, C, S = gen_main_fields(lloc, npe, 2)
    o = Oracle(L, NB, tbc=-1, kappa=KAPPA)
    o.set_fields(U, C)
    lat = qws_b200.Lattice(L, NB, tbc=-1, kappa=KAPPA)
    lat.load_fields(U, C)
    yield request.param, o, lat, S[0], S[1]
    lat.close()


@pytest.mark.parametrize("nsap,nm", [(4, 2), (2, 1), (3, 3)])
def test_fp16_sap_against_fp32(case, nsap, nm):
    name, o, lat, b, _ = case
    bs = b.astype(np.float32)
    got = lat.to_host(lat.prec_h(lat.to_device(bs), nsap, nm))
    ref = o.prec_s(bs, nsap - 1, nm)
    err = rel(got, ref)
    assert err < 1e-2, err


def test_fp16_sap_input_scaling(case):
    """Per-site scales: the preconditioner is linear up to FP16 rounding for
    inputs spanning many orders of magnitude (the reference's single global
    scale would flush the small sites)."""
    name, o, lat, b, _ = case
    bs = b.astype(np.float32)
    scale = np.exp(np.linspace(-12, 0, len(bs))).astype(np.float32)[:, None]
    x = (bs * scale).astype(np.float32)
    got = lat.to_host(lat.prec_h(lat.to_device(x), 4, 2))
    ref = o.prec_s(x, 3, 2)
    assert rel(got, ref) < 1e-2


def test_flexible_inner_solver(case):
    name, o, lat, b, _ = case
    bs = (b / np.linalg.norm(b)).astype(np.float32)
    xo, it_o, _ = o.bicgstab_precdd_s_h(bs, 1e-6, 50, 4, 2)
    xg, it_g, rel_g = lat.bicgstab_precdd_h(lat.to_device(bs), 1e-6, 50, 4, 2)
    assert rel_g < 1e-6
    assert it_g <= it_o + 2
    assert rel(lat.to_host(xg), xo) < 1e-4


def test_outer_mixed_fp16(case):
    name, o, lat, b, _ = case
    xo, _, _ = o.bicgstab_dd_mix(b, np.zeros_like(b), 1e-12, 20, 1e-6, 50, 4, 2)
    xd, bd = lat.empty("f64"), lat.to_device(b)
    st = lat.bicgstab_dd_mix2_hf(xd, bd, 1e-12, 20, 1e-6, 50, 4, 2, reliable=3)
    assert st["rel_resid_true"] < 1e-12
    assert lat.true_residual(xd, bd) < 1e-12
    assert rel(lat.to_host(xd), xo) < 1e-9


def test_hp_golden():
    """data/CASE_4111_1111_HP: the reference's half-precision DD solve
    (tol < 0, 6 outer x 2 x 50 inner iterations from the random initial
    guess) -- final bnorm^2, rnorm^2, xnorm^2 under check.sh's tolerances."""
    import qws_b200

    g = GOLD["CASE_4111_1111_HP"]
    a = g["args"]
    L = tuple(g["lloc"])
    U, C, S = gen_main_fields(L, (1, 1, 1, 1), 2)
    o = Oracle(L, (2, 1, 1, 1), tbc=-1, kappa=KAPPA)
    o.set_fields(U, C)
    lat = qws_b200.Lattice(L, (2, 1, 1, 1), tbc=-1, kappa=KAPPA)
    lat.load_fields(U, C)
    b, x0 = S[0], S[1]
    xd, bd = lat.to_device(x0), lat.to_device(b)
    st = lat.bicgstab_dd_mix2_hf(xd, bd, a["tol"], a["maxiter"], a["tol_s"], a["maxiter_s"],
                                 a["nsap"], a["nm"])
    assert st["inner_iters"] == 2 * a["maxiter"] * a["maxiter_s"]
    x = lat.to_host(xd)
    r = b - o.ddd_d(x)
    vals = [v for k, v in g["norms"] if k in ("bnorm^2", "rnorm^2", "xnorm^2")][-3:]
    for nm_, val, ref in zip(("bnorm^2", "rnorm^2", "xnorm^2"),
                             (np.sum(b * b), np.sum(r * r), np.sum(x * x)), vals):
        assert check_sh_ok(nm_, float(val), ref), (nm_, val, ref)
    lat.close()


def test_fp16_storage_of_vanishing_sites():
    """Sites whose components are FP32 denormals (a point source's solution
    far from the source on a large lattice) are stored as zero, never as
    NaN: the FP16 SAP of such a field stays finite and matches the FP32 SAP
    of the same field (the tiny sites contribute nothing either way)."""
    import qws_b200

    L = (8, 8, 8, 16)
    U, _ = qws_b200.gen_gauge(L, 3, 5, 0.36)
    C = qws_b200.gen_clover(U, L, 1.7, 0.1365)
    lat = qws_b200.Lattice(L, (2, 2, 2, 2), tbc=-1, kappa=0.1365)
    try:
        lat.load_fields(U, C)
        v = np.full((int(np.prod(L)), 24), 1e-39, np.float32)  # denormal everywhere
        v[0] = 1.0
        x = lat.to_device(v)
        h = lat.to_host(lat.prec_h(x, 4, 2))
        f = lat.to_host(lat.prec(x, 3, 2))  # the same sweep count: nsap-1 sweeps + final
        assert np.all(np.isfinite(h))
        assert rel(h, f) < 1e-2
    finally:
        lat.close()


def test_graphs_updated_for_a_new_kappa_match_direct_launches():
    """The precision form's inner solve replays each half iteration as a
    captured CUDA graph with its scalars on the device; when kappa changes
    the graphs are captured again and updated in place.  After such a
    change the solve is bit-for-bit the one direct launches give, and the
    device-side iteration count equals the host-side one."""
    import qws_b200

    L, NB = (8, 8, 8, 8), (2, 2, 2, 2)
    U, _ = qws_b200.gen_gauge(L, 5, 2, 0.36)
    b = qws_b200.gen_source(L, 6)
    res = {}
    for graphs in (True, False):
        lat = qws_b200.Lattice(L, NB, tbc=-1, kappa=0.130)
        try:
            lat.load_gauge(U)
            lat.set_graphs(graphs)
            bd, x = lat.to_device(b), lat.empty("f64")
            for kappa in (0.130, 0.1345, 0.132):  # the second and third update the graphs
                lat.set_kappa(kappa)
                lat.build_clover(1.7)
                x.zero_()
                st = lat.bicgstab_dd_mix2_hf(x, bd, 1e-10, 50, 1e-6, 50, 4, 2, reliable=5)
            res[graphs] = (lat.to_host(x), st, lat.true_residual(x, bd))
        finally:
            lat.close()
    (xg, sg, tg), (xd, sd, td) = res[True], res[False]
    np.testing.assert_array_equal(xg, xd)
    assert sg["inner_iters"] == sd["inner_iters"] and sg["outer_iters"] == sd["outer_iters"]
    assert tg < 1e-10
