"""qwsg_jinv_s_noalloc: the block-Richardson solve for callers that cannot
let the library allocate device memory (it uses a fixed array compiled into
the library instead of lazily allocated scratch).

Called through the C ABI and compared with qwsg_jinv_s, the allocating entry
point, on two calls in a row: the shared scratch keeps the previous call's
contents, so the second call checks that nothing depends on them.  On SU(3)
fields it is also compared with the CPU oracle's jinv.  This file
is collected last so a failure here never hides the other tests.
"""
import ctypes

import numpy as np
import pytest

from qwsref import gen_main_fields

pytestmark = pytest.mark.gpu

L = (32, 6, 4, 3)
KAPPA = 0.05


def rel(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def lat():
    import qws_b200

    lib = qws_b200.load_library()
    lib.qwsg_jinv_s_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int, ctypes.c_int]
    lib.qwsg_jinv_s_noalloc.restype = ctypes.c_int
    U, C, S = gen_main_fields(L, (1, 1, 1, 1), 2)
    lt = qws_b200.Lattice(L, (2, 1, 1, 1), tbc=-1, kappa=KAPPA)
    lt.load_fields(U, C)
    yield lib, lt, S
    lt.close()


@pytest.mark.parametrize("nm", [1, 2, 3])
def test_matches_allocating_entry_point_twice(lat, nm):
    lib, lt, S = lat
    for call, src in enumerate(S):  # two calls in a row, different inputs
        b = lt.to_device(src.astype(np.float32))
        for colour in (0, 1):
            ref = lt.to_host(lt.jinv(b, colour, nm))
            x = lt.empty("f32")
            rc = lib.qwsg_jinv_s_noalloc(lt.h, ctypes.c_void_p(x.data_ptr()),
                                         ctypes.c_void_p(b.data_ptr()), colour, nm)
            assert rc == 0, lib.qwsg_last_error().decode()
            got = lt.to_host(x)
            # both leave the other colour's sites untouched (zero here)
            assert rel(got, ref) < 1e-6, (call, colour)


def test_su3_fields_against_oracle_twice():
    """On SU(3) fields, after qwsg_jinv_s has switched the handle to its
    12-real links, the fixed-scratch path reads the same links and matches
    both the allocating entry point and the CPU oracle, on two calls in a row."""
    import qws_b200
    from qwsref import Oracle

    lib = qws_b200.load_library()
    Ls = (8, 8, 8, 16)
    U, _ = qws_b200.gen_gauge(Ls, seed=7, n_smear=2, alpha=0.36)
    C = qws_b200.gen_clover(U, Ls, 1.7, 0.1365)
    o = Oracle(Ls, (2, 1, 1, 1), tbc=-1, kappa=0.1365)
    o.set_fields(U, C)
    lt = qws_b200.Lattice(Ls, (2, 1, 1, 1), tbc=-1, kappa=0.1365)
    try:
        lt.load_fields(U, C)
        rng = np.random.default_rng(3)
        for call in range(2):
            src = rng.standard_normal((lt.V, 24)).astype(np.float32)
            b = lt.to_device(src)
            for colour in (0, 1):
                ref = lt.to_host(lt.jinv(b, colour, 2))
                assert lt.link_compression()
                x = lt.empty("f32")
                rc = lib.qwsg_jinv_s_noalloc(lt.h, ctypes.c_void_p(x.data_ptr()),
                                             ctypes.c_void_p(b.data_ptr()), colour, 2)
                assert rc == 0, lib.qwsg_last_error().decode()
                got = lt.to_host(x)
                np.testing.assert_array_equal(got, ref)  # same kernel, same links
                m = np.zeros(lt.V, bool)
                orc = o.jinv_s(src, colour, 2)
                m[np.abs(ref).sum(axis=1) > 0] = True
                assert rel(got[m], orc[m]) < 1e-6, (call, colour)
    finally:
        lt.close()


def test_rejects_batch_handle(lat):
    """A handle made by qwsg_create_batch (even with one RHS) reads its
    parent's fields through a stream synchronisation this path does not do:
    it is refused with code 1."""
    lib, lt, _ = lat
    B = lt.batch(1)
    try:
        x = B.empty("f32")
        b = B.empty("f32")
        rc = lib.qwsg_jinv_s_noalloc(B.h, ctypes.c_void_p(x.data_ptr()),
                                     ctypes.c_void_p(b.data_ptr()), 0, 2)
        assert rc == 1
        assert b"qwsg_create_batch" in lib.qwsg_last_error()
    finally:
        B.close()


def test_rejects_lattice_beyond_scratch(lat):
    import qws_b200

    lib, _, _ = lat
    big = qws_b200.Lattice((32, 32, 32, 64), (2, 1, 1, 1), tbc=-1, kappa=KAPPA)
    x = big.torch.empty(1, device="cuda")
    rc = lib.qwsg_jinv_s_noalloc(big.h, ctypes.c_void_p(x.data_ptr()),
                                 ctypes.c_void_p(x.data_ptr() + 4), 0, 2)
    assert rc == 2
    assert b"exceeds the fixed scratch" in lib.qwsg_last_error()
    big.close()
