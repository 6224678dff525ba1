"""qwsg_batch_set_parent: a multi-RHS handle re-attached to another lattice of
the same extents and block grid serves that lattice's fields and kappa with
its own buffers (the solve service moves idle work buffers between the
gauge fields of one volume this way).  The bar is bitwise equality with a
handle made on that lattice: the same geometry, fields and kernels.  Per-RHS
kappas must be set again after the move; a handle whose old parent was
already destroyed can still move; other geometries are refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L, NB, CSW = (8, 8, 8, 16), (2, 1, 1, 1), 1.7
ARGS = (1e-10, 100, 1e-6, 50, 4, 2)


def lattice(seed, kappa):
    import qws_b200

    lat = qws_b200.Lattice(L, NB, tbc=-1, kappa=kappa)
    lat.load_gauge(qws_b200.gen_gauge(L, seed)[0])
    lat.build_clover(CSW)
    return lat


def solve(h, b):
    x = h.empty("f64")
    st = h.bicgstab_dd_mix2_hf(x, h.to_device(b), *ARGS, reliable=2)
    return x, st


def test_moved_handle_solves_the_new_lattice_bitwise():
    import qws_b200
    import torch

    A, B = lattice(1, 0.130), lattice(2, 0.125)
    b = qws_b200.gen_source(L, 3)
    h = A.batch(1)
    xa, _ = solve(h, b)  # graphs and buffers made on A
    h.set_parent(B)
    x1, s1 = solve(h, b)
    fresh = B.batch(1)
    x2, s2 = solve(fresh, b)
    torch.cuda.synchronize()
    assert torch.equal(x1, x2) and s1 == s2
    assert not torch.equal(x1, xa)
    assert B.true_residual(x1, B.to_device(b)) < 1e-9
    for o in (h, fresh, A, B):
        o.close()


def test_moved_batch_with_kappas_per_rhs():
    import qws_b200
    import torch

    A, B = lattice(4, 0.130), lattice(5, 0.130)
    b = np.stack([qws_b200.gen_source(L, 6), qws_b200.gen_source(L, 7)])
    h = A.batch(2)
    h.set_kappas([0.130, 0.125], CSW)
    solve(h, b)
    h.set_parent(B)
    h.set_kappas([0.128, 0.131], CSW)
    x1, _ = solve(h, b)
    fresh = B.batch(2)
    fresh.set_kappas([0.128, 0.131], CSW)
    x2, _ = solve(fresh, b)
    torch.cuda.synchronize()
    assert torch.equal(x1, x2)
    for o in (h, fresh, A, B):
        o.close()


def test_move_after_the_old_parent_is_gone_and_refusals():
    import qws_b200
    import torch

    A, B = lattice(8, 0.13), lattice(9, 0.13)
    b = qws_b200.gen_source(L, 10)
    h = A.batch(1)
    solve(h, b)
    A.close()  # the handle's old parent no longer exists
    h.set_parent(B)
    x1, _ = solve(h, b)
    fresh = B.batch(1)
    x2, _ = solve(fresh, b)
    torch.cuda.synchronize()
    assert torch.equal(x1, x2)
    other = qws_b200.Lattice((8, 8, 8, 8), NB, tbc=-1, kappa=0.13)
    with pytest.raises(qws_b200.QwsgError, match="same extents"):
        h.set_parent(other)
    with pytest.raises(qws_b200.QwsgError, match="not a multi-RHS handle"):
        qws_b200._check(B.lib.qwsg_batch_set_parent(B.h, other.h))
    for o in (h, fresh, B, other):
        o.close()
