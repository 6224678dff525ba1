"""qwsg_jinv_s_noalloc: the block-Richardson solve for callers that cannot
let the library allocate device memory (it uses a fixed array compiled into
the library instead of lazily allocated scratch).

Called through the C ABI and compared with qwsg_jinv_s, the allocating entry
point, on two calls in a row: the shared scratch keeps the previous call's
contents, so the second call checks that nothing depends on them.  This file
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
