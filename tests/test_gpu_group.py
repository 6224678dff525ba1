"""Group solves (qwsg_group_bicgstab_dd_mix2_hf): lattices of different
volumes, block grids, kappas and tolerances solved together, each kernel
step one launch over all of them.

The merged kernels run, for every lattice, the blocks of that lattice's own
launch with its own arguments (reductions included: the same block count,
partials and final sum), so the bar is bitwise equality of every solution
and of its statistics with the lattice's own qwsg_bicgstab_dd_mix2_hf call.
A lattice whose solve fails (a non-finite source) reports its error while
the others finish with the same bitwise results.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CSW = 1.7
# (L, NB, kappa, seed, tol, nsap, nm, reliable): four volumes, three block
# grids, two (nsap, nm) pairs -- lattices with other parameters run other
# launch sequences, merged among themselves
LATS = [
    ((8, 8, 8, 8), (2, 2, 2, 2), 0.1365, 11, 1e-10, 4, 2, 0),
    ((12, 12, 12, 24), (2, 2, 2, 2), 0.130, 12, 1e-8, 4, 2, 0),
    ((8, 8, 8, 16), (2, 1, 1, 1), 0.125, 13, 1e-12, 4, 2, 2),
    ((16, 16, 16, 32), (2, 2, 2, 4), 0.1365, 14, 1e-10, 4, 2, 2),
    ((8, 8, 8, 8), (2, 2, 2, 2), 0.132, 15, 1e-10, 3, 3, 0),
]


def solve_args(p):
    L, NB, kappa, seed, tol, nsap, nm, rel = p
    return dict(tol=tol, maxiter=50, tol_s=1e-2, maxiter_s=50, nsap=nsap, nm=nm, reliable=rel)


@pytest.fixture(scope="module")
def lattices():
    import qws_b200

    out = []
    for p in LATS:
        L, NB, kappa, seed = p[:4]
        lat = qws_b200.Lattice(L, NB, tbc=-1, kappa=kappa)
        lat.load_gauge(qws_b200.gen_gauge(L, seed)[0])
        lat.build_clover(CSW)
        b = lat.to_device(qws_b200.gen_source(L, seed + 100))
        out.append((p, lat, b))
    yield out
    for _, lat, _ in out:
        lat.close()


def own_solves(lattices):
    res = []
    for p, lat, b in lattices:
        x = lat.empty("f64")
        st = lat.bicgstab_dd_mix2_hf(x, b, **solve_args(p))
        res.append((x, st))
    return res


def group(lattices, xs=None):
    import qws_b200

    if xs is None:
        xs = [lat.empty("f64") for _, lat, _ in lattices]
    solves = [dict(lattice=lat, x=x, b=b, **solve_args(p))
              for (p, lat, b), x in zip(lattices, xs)]
    st, gs = qws_b200.group_solve(solves, check=False)
    return xs, st, gs


def test_group_bitwise_equal_to_own_solves(lattices):
    import torch

    own = own_solves(lattices)
    for rep in range(2):  # two group calls in a row
        xs, st, gs = group(lattices)
        torch.cuda.synchronize()
        for (x0, s0), x, s, (p, lat, b) in zip(own, xs, st, lattices):
            assert s["status"] == 0, (p, s)
            assert torch.equal(x, x0), p
            for k in ("outer_iters", "inner_iters", "rel_resid_recursive", "rel_resid_true"):
                assert s[k] == s0[k], (p, k, s[k], s0[k])
            assert lat.true_residual(x, b) < p[4] * 10
        assert gs["merged_launches"] < gs["member_launches"], gs
        assert gs["rounds"] > 0


def test_group_merges_lattices_at_the_same_step(lattices):
    """Three volumes with the same solver parameters: the lattices stay in
    step (a group one step ahead waits a round for the others), so one
    launch serves all three most of the time."""
    import torch

    same = [(p[:4] + (1e-10, 4, 2, 0), lat, b) for p, lat, b in
            (lattices[0], lattices[1], lattices[3])]
    own = own_solves(same)
    xs, st, gs = group(same)
    torch.cuda.synchronize()
    for (x0, s0), x, s in zip(own, xs, st):
        assert s["status"] == 0 and torch.equal(x, x0)
    assert gs["merged_launches"] * 2 < gs["member_launches"], gs


def test_group_with_initial_guess(lattices):
    """x holds the initial guess on entry, as in the one-lattice call."""
    import torch

    xs0 = []
    for p, lat, b in lattices:
        x = lat.empty("f64")
        lat.bicgstab_dd_mix2_hf(x, b, **dict(solve_args(p), tol=1e-4, reliable=0))
        xs0.append(x)
    own = []
    for (p, lat, b), x0 in zip(lattices, xs0):
        x = x0.clone()
        own.append((x, lat.bicgstab_dd_mix2_hf(x, b, **solve_args(p))))
    xs, st, _ = group(lattices, [x0.clone() for x0 in xs0])
    torch.cuda.synchronize()
    for (x1, s1), x, s in zip(own, xs, st):
        assert s["status"] == 0
        assert torch.equal(x, x1)
        assert s["inner_iters"] == s1["inner_iters"]


def test_group_failed_member_leaves_others_intact(lattices):
    import qws_b200
    import torch

    own = own_solves(lattices)
    p_bad, lat_bad, b_bad = lattices[1]
    bad = b_bad.clone()
    bad[7] = float("nan")
    mixed = list(lattices)
    mixed[1] = (p_bad, lat_bad, bad)
    xs, st, _ = group(mixed)
    torch.cuda.synchronize()
    assert st[1]["status"] == 3, st[1]
    for i, ((x0, s0), x, s) in enumerate(zip(own, xs, st)):
        if i == 1:
            continue
        assert s["status"] == 0
        assert torch.equal(x, x0)
    with pytest.raises(qws_b200.QwsgError, match="item 1"):
        qws_b200.group_solve([dict(lattice=lat, x=x, b=b, **solve_args(p))
                              for (p, lat, b), x in zip(mixed, xs)])


def test_group_rejects_bad_items(lattices):
    import qws_b200

    p, lat, b = lattices[0]
    x = lat.empty("f64")
    one = dict(lattice=lat, x=x, b=b, **solve_args(p))
    with pytest.raises(qws_b200.QwsgError, match="twice"):
        qws_b200.group_solve([one, dict(one)])
    with pytest.raises(qws_b200.QwsgError, match="nsap and nm"):
        qws_b200.group_solve([dict(one, nsap=11)])
    batch = lat.batch(2)
    try:
        with pytest.raises(qws_b200.QwsgError):
            qws_b200.group_solve([dict(one, lattice=batch)])
    finally:
        batch.close()
    # an empty group is a no-op
    st, gs = qws_b200.group_solve([])
    assert st == [] and gs["rounds"] == 0 and gs["merged_launches"] == 0
