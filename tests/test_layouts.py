"""qws_b200.layouts (the QWS host-layout converters the package ships)
agree with the test harness's converters, which the oracle tests pin to
the reference's own arrays (main.cc's layout and the reference's loaders)."""
import numpy as np

from qws_b200 import layouts
from qwsref import nat_to_qws_clover, nat_to_qws_gauge, nat_to_qws_spinor, qws_to_nat_spinor


def test_layouts_match_harness():
    rng = np.random.default_rng(0)
    for L, vlen in (((32, 6, 4, 3), 8), ((32, 6, 4, 3), 16), ((8, 4, 4, 8), 2)):
        V = int(np.prod(L))
        v = rng.standard_normal((V, 24))
        U = rng.standard_normal((4, V, 3, 3, 2))
        C = rng.standard_normal((V, 72))
        q = layouts.nat_to_qws_spinor(v, L, vlen)
        assert np.array_equal(q, nat_to_qws_spinor(v, L, vlen))
        out = layouts.aligned_empty(q.size, np.float64)
        layouts.nat_to_qws_spinor(v, L, vlen, out=out)
        assert np.array_equal(out, q) and out.ctypes.data % 256 == 0
        assert np.array_equal(layouts.qws_to_nat_spinor(q, L, vlen), qws_to_nat_spinor(q, L, vlen))
        assert np.array_equal(layouts.qws_to_nat_spinor(q, L, vlen), v)
        assert np.array_equal(layouts.nat_to_qws_gauge(U, L, vlen), nat_to_qws_gauge(U, L, vlen))
        assert np.array_equal(layouts.nat_to_qws_clover(C, L, vlen), nat_to_qws_clover(C, L, vlen))
