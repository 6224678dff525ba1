"""Properties of the synthetic benchmark fields (host code of the library,
no GPU needed).  The reference only loads fields built elsewhere, so these
conventions are checked by their properties rather than against it."""
import numpy as np
import pytest

import qws_b200
from qwsref import Oracle

L = (8, 4, 4, 8)


@pytest.fixture(scope="module")
def gauge():
    return qws_b200.gen_gauge(L, seed=5, n_smear=5, alpha=0.36)


def as_complex(U):
    u = U.reshape(4, -1, 3, 3, 2)
    return u[..., 0] + 1j * u[..., 1]


def test_su3(gauge):
    U, plaq = gauge
    u = as_complex(U)
    eye = np.einsum("...ij,...kj->...ik", u, u.conj())
    assert np.abs(eye - np.eye(3)).max() < 1e-12
    assert np.abs(np.linalg.det(u) - 1).max() < 1e-12


def test_plaquette_target(gauge):
    U, plaq = gauge
    assert abs(plaq - qws_b200.plaquette(U, L)) < 1e-12
    assert 0.50 < plaq < 0.60  # 5 APE steps at alpha 0.36 -> ~0.55
    U0, p0 = qws_b200.gen_gauge(L, seed=5, n_smear=0)
    assert abs(p0) < 0.05  # Haar-like random links


def test_deterministic(gauge):
    U, _ = gauge
    U2, _ = qws_b200.gen_gauge(L, seed=5, n_smear=5, alpha=0.36)
    np.testing.assert_array_equal(U, U2)


def test_clover_inverse_and_hermiticity(gauge):
    U, _ = gauge
    C, T = qws_b200.gen_clover(U, L, csw=1.7, kappa=0.1365, with_T=True)
    Tc = T[..., 0] + 1j * T[..., 1]
    assert np.abs(Tc - np.conj(np.swapaxes(Tc, 1, 2))).max() < 1e-14
    assert np.linalg.eigvalsh(Tc).min() > 0
    # QWS's packed-clover kernel (oracle, clover_def.h) applied to T v gives v
    V = int(np.prod(L))
    o = Oracle(L, (2, 1, 1, 1), tbc=1, kappa=0.1365)
    o.set_fields(U.reshape(4, V, 18), C)
    v = np.random.default_rng(0).standard_normal((V, 24))
    w = o.clover_d(v)
    vc, wc = v[:, 0::2] + 1j * v[:, 1::2], w[:, 0::2] + 1j * w[:, 1::2]
    assert np.abs(np.einsum("sij,sj->si", Tc, wc) - vc).max() < 1e-12


def test_free_field_limit():
    V = int(np.prod(L))
    U = np.zeros((4, V, 18))
    for a in range(3):
        U[:, :, 2 * (3 * a + a)] = 1
    C = qws_b200.gen_clover(U, L, csw=1.7, kappa=0.1365)
    assert np.allclose(C[:, :6], 0.5) and np.allclose(C[:, 36:42], 0.5)
    assert np.abs(C[:, 6:36]).max() == 0 and np.abs(C[:, 42:]).max() == 0


def test_sources():
    V = int(np.prod(L))
    g = qws_b200.gen_source(L, seed=3, kind="gauss")
    assert abs(np.mean(g ** 2) - 0.5) < 0.05
    p = qws_b200.gen_source(L, kind="point", arg=4 * 2 + 3)  # colour 2, spin 3
    assert p.sum() == 1 and p[0, 8 * 2 + 2 * 3] == 1
    z = qws_b200.gen_source(L, seed=4, kind="z2")
    assert np.allclose(np.abs(z), 1 / np.sqrt(2))
    assert z.shape == (V, 24)


@pytest.mark.parametrize("Lg,n_smear,csw,kappa", [
    ((8, 4, 4, 8), 5, 1.7, 0.1365),
    ((32, 6, 4, 3), 0, 1.0, 0.125),  # the plain CPU-runnable workload's fields
    ((6, 6, 4, 4), 2, 1.7, 0.1355),
])
def test_oracle_generator_bit_equal(Lg, n_smear, csw, kappa):
    """The reference arm builds its inputs with the oracle's restatement of
    the generator (oracle/fields_oracle.cc) so that it never loads the
    product library; both arms of a comparison must see identical arrays,
    so the two generators agree bit for bit (links, clover, every source kind)."""
    import qwsref

    bits = lambda a: np.ascontiguousarray(a).view(np.uint64)
    U, p = qws_b200.gen_gauge(Lg, seed=11, n_smear=n_smear, alpha=0.36)
    Uo, po = qwsref.gen_gauge(Lg, seed=11, n_smear=n_smear, alpha=0.36)
    np.testing.assert_array_equal(bits(U), bits(Uo))
    assert abs(p - po) < 1e-13  # reduction order of the threads may differ
    np.testing.assert_array_equal(bits(qws_b200.gen_clover(U, Lg, csw, kappa)),
                                  bits(qwsref.gen_clover(Uo, Lg, csw, kappa)))
    for kind, arg in (("gauss", 0), ("z2", 0), ("point", 7)):
        np.testing.assert_array_equal(bits(qws_b200.gen_source(Lg, 12, kind, arg)),
                                      bits(qwsref.gen_source(Lg, 12, kind, arg)))


def test_reference_solution_fixture():
    """tests/golden/ref_solutions_48c96.npz (made by make_ref_solutions.py from
    the reference's own 48^3x96 solves): both kappas, 1024 distinct sites in
    range, finite values, iteration counts and residuals of a converged
    1e-10 solve, and the same gauge field and source digests for both."""
    import json
    from pathlib import Path

    z = np.load(Path(__file__).parent / "golden" / "ref_solutions_48c96.npz")
    meta = json.loads(str(z["meta"]))
    V = 48 * 48 * 48 * 96
    sites = z["sites"]
    assert len(sites) == 1024 and len(set(sites.tolist())) == 1024
    assert sites.min() >= 0 and sites.max() < V and (np.diff(sites) > 0).all()
    assert set(meta) == {"0.1365", "0.1355"}
    for k, m in meta.items():
        x = z[f"x_{k}"]
        assert x.shape == (1024, 24) and np.isfinite(x).all()
        assert m["true_rel_resid"] < 1e-10 and m["outer_iters"] >= 1
        # the sample carries its share of |x|^2
        share = float(np.sum(x * x)) / float(z[f"xnorm2_{k}"])
        assert 0.2 * 1024 / V < share < 5 * 1024 / V
    a, b = meta["0.1365"]["field_sha256"], meta["0.1355"]["field_sha256"]
    assert a["gauge"] == b["gauge"] and a["source"] == b["source"] and a["clover"] != b["clover"]
