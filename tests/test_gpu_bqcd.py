"""BQCD-format arrays converted on the device (qwsg_load_{gauge,clover}_bqcd,
qwsg_spinor_{from,to}_bqcd_*): the planes they write are bit-equal to the
ones the natural-layout loaders write from the same field, with the default
numbering and with a caller's site map; spinors round-trip exactly.  The
BQCD arrays come from oracle/qwsref.py's nat_to_bqcd_* helpers, which
tests/test_oracle_vs_ref.py pins to the reference's own loaders
(qws_bqcd.cc:66-642)."""
import numpy as np
import pytest

from qwsref import BQCD_CLV_PERM, nat_to_bqcd_clover, nat_to_bqcd_gauge, nat_to_bqcd_spinor

pytestmark = pytest.mark.gpu

L = (8, 4, 4, 8)
V = int(np.prod(L))


def parity(L):
    n = np.arange(int(np.prod(L)))
    x, y = n % L[0], (n // L[0]) % L[1]
    z, t = (n // (L[0] * L[1])) % L[2], n // (L[0] * L[1] * L[2])
    return (x + y + z + t) % 2


def random_map(seed):
    """each parity's sites sent to a random order of that parity's slots"""
    rng = np.random.default_rng(seed)
    eo = parity(L)
    m = np.empty(V, np.int32)
    for p in (0, 1):
        sites = np.flatnonzero(eo == p)
        m[sites] = p * (V // 2) + rng.permutation(V // 2)
    return m


# the BQCD arrays for a given site map (slot of natural site n = m[n])
def bqcd_gauge(U, m):
    out = np.zeros((4, V, 3, 3, 2))  # mu, slot, col, row, ri
    out[:, m] = np.asarray(U).reshape(4, V, 3, 3, 2).transpose(0, 1, 3, 2, 4)
    return out.reshape(-1)


def bqcd_clover(C, m):
    blk = np.zeros((V, 2, 36))
    blk[:, :, BQCD_CLV_PERM] = np.asarray(C).reshape(V, 2, 36)
    out = np.zeros((V, 2, 36))
    out[m] = blk
    return out.reshape(-1)


def bqcd_spinor(v, m):
    out = np.zeros((V, 24))
    out[m] = np.asarray(v).reshape(V, 24)
    return out[:V // 2].reshape(-1), out[V // 2:].reshape(-1)


@pytest.fixture(scope="module")
def fields():
    import qws_b200

    U, _ = qws_b200.gen_gauge(L, 5, 2, 0.36)
    C = qws_b200.gen_clover(U, L, 1.7, 0.13)
    b = qws_b200.gen_source(L, 9, "gauss")
    ref = qws_b200.Lattice(L, (2, 2, 2, 2), tbc=-1, kappa=0.13)
    ref.load_fields(U, C)
    yield U, C, b, ref
    ref.close()


def apply_all(lat, b):
    d, s = lat.to_device(b), lat.to_device(b.astype(np.float32))
    return {"ddd_d": lat.to_host(lat.ddd(d)), "ddd_s": lat.to_host(lat.ddd(s)),
            "prec": lat.to_host(lat.prec(s, 4, 2))}


@pytest.mark.parametrize("mapped", [False, True], ids=["default", "site_map"])
def test_fields_bit_equal(fields, mapped):
    import qws_b200

    U, C, b, ref = fields
    m = random_map(1) if mapped else None
    u = bqcd_gauge(U, m) if mapped else nat_to_bqcd_gauge(U, L)
    c = bqcd_clover(C, m) if mapped else nat_to_bqcd_clover(C, L)
    lat = qws_b200.Lattice(L, (2, 2, 2, 2), tbc=-1, kappa=0.13)
    try:
        lat.load_fields_bqcd(u, c, site_map=m)
        want, got = apply_all(ref, b), apply_all(lat, b)
        for k in want:
            assert np.array_equal(got[k], want[k]), k
    finally:
        lat.close()


@pytest.mark.parametrize("mapped", [False, True], ids=["default", "site_map"])
def test_spinors(fields, mapped):
    U, C, b, ref = fields
    m = random_map(2) if mapped else None
    e, o = bqcd_spinor(b, m) if mapped else nat_to_bqcd_spinor(b, L)
    d = ref.from_bqcd(e, o, "f64", site_map=m)
    assert ref.torch.equal(d, ref.to_device(b))
    s = ref.from_bqcd(e, o, "f32", site_map=m)
    assert ref.torch.equal(s, ref.to_device(b.astype(np.float32)))
    e2, o2 = ref.to_bqcd(d, site_map=m)
    assert np.array_equal(e2, e) and np.array_equal(o2, o)
    e3, o3 = ref.to_bqcd(s, site_map=m)
    assert np.array_equal(e3, e.astype(np.float32).astype(np.float64))
    # a batch handle takes nrhs arrays back to back
    B = ref.batch(2)
    try:
        b2 = np.stack([b, 2 * b])
        pairs = [bqcd_spinor(v, m) if mapped else nat_to_bqcd_spinor(v, L) for v in b2]
        db = B.from_bqcd(np.concatenate([p[0] for p in pairs]),
                         np.concatenate([p[1] for p in pairs]), "f64", site_map=m)
        assert B.torch.equal(db, B.to_device(b2))
    finally:
        B.close()


def test_bad_site_map(fields):
    import qws_b200

    U, C, b, ref = fields
    m = np.arange(V, dtype=np.int32)  # slots ignore the parity split
    e, o = nat_to_bqcd_spinor(b, L)
    with pytest.raises(qws_b200.QwsgError):
        ref.from_bqcd(e, o, "f64", site_map=m)
