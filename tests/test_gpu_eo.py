"""GPU even-odd (site parity) family against the oracle (on the CASE0, 4 and 7
lattices) and the CASE0 golden.

main.cc fills its arrays with the DD generator and reads them with the
even-odd operators too; oracle/qwsref.py's eo_perm gives the field an
even-odd operator sees, eo_partner the aliasing of half-array arguments.
Tolerances: FP64 1e-13, FP32 1e-6 (relative norm of the difference).
"""
import json
from pathlib import Path

import numpy as np
import pytest

from qwsref import Oracle, check_sh_ok, eo_partner, eo_perm, gen_main_fields, parity_mask

pytestmark = pytest.mark.gpu

GOLD = json.loads((Path(__file__).parent / "golden" / "case_norms.json").read_text())
KAPPA = 0.05
FAC = -KAPPA * KAPPA
# (pe, which, dag, clov, mode) of the reference's entry points
COMBOS = [(1, 1, 0, 0, 0), (1, 1, 0, 1, 0), (1, 1, 1, 0, 0), (1, 1, 1, 1, 0), (1, 1, 0, 1, 2),
          (1, 1, 1, 0, 2), (1, 2, 0, 0, 1), (1, 2, 1, 0, 1), (1, 2, 0, 1, 1), (1, 2, 1, 1, 1),
          (1, 3, 0, 0, 0), (1, 3, 0, 1, 0), (1, 3, 1, 0, 0), (1, 3, 1, 1, 0), (1, 3, 0, 1, 2),
          (1, 3, 1, 0, 2), (0, 3, 0, 1, 2)]


def rel(a, b, m):
    a, b = np.asarray(a, np.float64)[m], np.asarray(b, np.float64)[m]
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


# golden lattices whose global extents are all even (site parity is then
# consistent across the periodic boundaries)
EO_CASES = {
    "CASE0": ((32, 6, 4, 3), (1, 1, 1, 1)),
    "CASE4": ((32, 6, 6, 2), (1, 1, 1, 2)),
    "CASE7": ((32, 6, 4, 3), (1, 2, 2, 2)),
}


@pytest.fixture(scope="module", params=list(EO_CASES))
def setup(request):
    import qws_b200

    lloc, npe = EO_CASES[request.param]
    L = tuple(a * b for a, b in zip(lloc, npe))
    NB = (2 * npe[0], npe[1], npe[2], npe[3])
    U, C, S = gen_main_fields(lloc, npe, 2)
    if request.param == "CASE0":  # the even-odd reading of main.cc's arrays
        P = eo_perm(L)
        U, C, b = U[:, P], C[P], S[0][P]
    else:
        b = S[0]
    o = Oracle(L, NB, tbc=-1, kappa=KAPPA)
    o.set_fields(U, C)
    lat = qws_b200.Lattice(L, NB, tbc=-1, kappa=KAPPA)
    lat.load_fields(U, C)
    yield request.param, L, o, lat, b
    lat.close()


@pytest.mark.parametrize("combo", COMBOS)
def test_deo_combos(setup, combo):
    name, L, o, lat, b = setup
    pe, which, dag, clov, mode = combo
    m = parity_mask(L, pe)
    in0 = b[eo_partner(L)]
    acc0 = np.random.default_rng(7).standard_normal(b.shape)
    for dt, tol in ((np.float64, 1e-13), (np.float32, 1e-6)):
        x, i0, a0 = b.astype(dt), in0.astype(dt), acc0.astype(dt)
        ref = o.deo(x, pe, which, dag, clov, mode, dt(FAC), i0 if mode == 2 else None,
                    out=a0.copy() if mode == 1 else None)
        got = lat.to_host(lat.deo(lat.to_device(x), pe, which, dag, clov, mode, FAC,
                                  in0=lat.to_device(i0) if mode == 2 else None,
                                  out=lat.to_device(a0) if mode == 1 else None))
        assert rel(got, ref, m) < tol, (dt, combo)


def test_mtilde_and_solver(setup):
    name, L, o, lat, b = setup
    m0 = parity_mask(L, 0)
    xd = lat.to_device(b)
    assert rel(lat.to_host(lat.mtilde(xd)), o.mtilde(b), m0) < 1e-13
    assert rel(lat.to_host(lat.mtilde(xd, dag=True)), o.mtilde(b, True), m0) < 1e-13
    be = b * m0[:, None]
    xo, it_o = o.bicgstab_vm(be, np.zeros_like(b), 100)
    x = lat.empty("f64")
    it = lat.bicgstab_vm(x, lat.to_device(be), 100)
    assert abs(it - it_o) <= 1
    assert rel(lat.to_host(x), xo, m0) < 1e-11
    if name == "CASE0":
        assert it == 91  # the golden's timing table: 91 bicgstab_iter_ calls
        r = be - o.mtilde(lat.to_host(x))
        n2 = lambda a: float(np.sum(a[m0] ** 2))
        vals = [v for k, v in GOLD["CASE0"]["norms"] if k in ("bnorm^2", "rnorm^2", "xnorm^2")][:3]
        for nm_, val, ref in zip(("bnorm^2", "rnorm^2", "xnorm^2"),
                                 (n2(be), n2(r), n2(lat.to_host(x))), vals):
            assert check_sh_ok(nm_, val, ref), (nm_, val, ref)


def test_cg_solvers(setup):
    """cg_vm_ (cg.cc:65) and mcg_vm_ (mcg.cc:65) on mtilde^dag mtilde against
    the oracle's restatements (which tests/test_oracle_vs_ref.py pins to the
    reference's own solvers): iteration counts within 2% (about a thousand
    iterations on an ill-conditioned operator, where the sums' rounding moves
    the count by a few), solutions to 1e-10 relative (both stop at
    |r|/|b| < 1e-14; the condition number is ~4e3), and every shifted
    system solved to 1e-10."""
    name, L, o, lat, b = setup
    m0 = parity_mask(L, 0)
    be = b * m0[:, None]
    bd = lat.to_device(be)
    xo, it_o = o.cg_vm(be, np.zeros_like(b), 3000)
    assert it_o < 2999
    x = lat.empty("f64")
    it = lat.cg_vm(x, bd, 3000)
    assert abs(it - it_o) <= max(1, it_o // 50)
    assert rel(lat.to_host(x), xo, m0) < 1e-10
    sigma = [0.0, 0.05, 0.5, 2.0]
    Xo, it_o = o.mcg_vm(be, sigma, 3000)
    X, it = lat.mcg_vm(bd, sigma, 3000)
    assert abs(it - it_o) <= max(1, it_o // 50)
    for k, s in enumerate(sigma):
        xk = lat.to_host(X[k])
        assert np.isfinite(xk).all(), k
        assert rel(xk, Xo[k], m0) < 1e-10, k
        ax = lat.to_host(lat.mtdagmt(X[k])) + s * xk
        assert rel(ax, be, m0) < 1e-10, k
