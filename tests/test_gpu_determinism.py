"""Checks that stand in for a race detector and a bounds checker (the pool
runs no compute-sanitizer):

* reproducibility: a solve gives bit-identical solutions and statistics run
  after run, with its CUDA graphs replayed or off, and with the Dirac
  kernels launched in CTAs of 64, 128 or 256 threads.  Every site is one
  thread's work and every reduction sums its block partials in a fixed
  order (blas.cu), so nothing may depend on timing or on the launch shape;
  a race or an order-dependent sum would show up as a difference here.
* padding canaries: on a lattice whose site count is not a multiple of the
  128-site plane padding, NaN is planted in the padding entries of every
  input field; no operator or solver may read them (their results must be
  finite and bit-identical to the results without canaries) nor write
  them.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CSW, KAPPA = 1.7, 0.1365


def lattice(L, NB, seed):
    import qws_b200

    lat = qws_b200.Lattice(L, NB, tbc=-1, kappa=KAPPA)
    lat.load_gauge(qws_b200.gen_gauge(L, seed)[0])
    lat.build_clover(CSW)
    return lat


def test_solves_reproducible_across_runs_graphs_and_cta_sizes():
    import qws_b200
    import torch

    L, NB = (8, 8, 8, 16), (2, 2, 2, 2)
    lat = lattice(L, NB, 21)
    bd = lat.to_device(qws_b200.gen_source(L, 22))

    def solves():
        x1, x2 = lat.empty("f64"), lat.empty("f64")
        s1 = lat.bicgstab_dd_mix(x1, bd, 1e-10, 100, 1e-6, 50, 4, 2)
        s2 = lat.bicgstab_dd_mix2_hf(x2, bd, 1e-10, 100, 1e-6, 50, 4, 3, reliable=3)
        torch.cuda.synchronize()
        return (x1, s1), (x2, s2)

    ref = solves()
    runs = [solves()]                       # again, graphs replayed
    lat.set_graphs(False)
    runs.append(solves())                   # launch by launch
    lat.set_graphs(True)
    for t in (64, 256, 128):
        lat.set_hop_threads(t)
        runs.append(solves())
    for run in runs:
        for (x0, s0), (x, s) in zip(ref, run):
            assert torch.equal(x, x0)
            assert s == s0
    lat.close()


def plant(x, lat):
    """NaN in the padding entries [V, pad) of every plane of a spinor field."""
    if x.dtype.itemsize == 4:  # six float4 planes
        x.view(6, lat.pad, 4)[:, lat.V:, :] = float("nan")
    else:                      # twelve double2 planes
        x.view(12, lat.pad, 2)[:, lat.V:, :] = float("nan")


def valid(x, lat):
    if x.dtype.itemsize == 4:
        return x.view(6, lat.pad, 4)[:, :lat.V, :]
    return x.view(12, lat.pad, 2)[:, :lat.V, :]


def padding(x, lat):
    if x.dtype.itemsize == 4:
        return x.view(6, lat.pad, 4)[:, lat.V:, :]
    return x.view(12, lat.pad, 2)[:, lat.V:, :]


def test_padding_canaries():
    import qws_b200
    import torch

    L, NB = (12, 6, 4, 6), (2, 1, 1, 1)   # 1728 sites, planes of 1792
    lat = lattice(L, NB, 31)
    assert lat.pad > lat.V
    b = qws_b200.gen_source(L, 32)
    ops = {
        "ddd_s": lambda x, o: lat.ddd(x, out=o),
        "ddd_in_s": lambda x, o: lat.ddd_in(x, 1, out=o),
        "ddd_out_s": lambda x, o: lat.ddd_out(x, 0, 0.3, out=o),
        "jinv_s": lambda x, o: lat.jinv(x, 0, 3, out=o),
        "prec_ddd_s": lambda x, o: lat.prec_ddd(x, 4, 2, out=o),
        "prec_s": lambda x, o: lat.prec(x, 4, 2, out=o),
        "prec_h": lambda x, o: lat.prec_h(x, 4, 2, out=o),
    }
    xs = lat.to_device(b.astype(np.float32))
    for name, op in ops.items():
        clean = op(xs.clone(), torch.zeros_like(xs))
        x = xs.clone()
        plant(x, lat)
        o = torch.zeros_like(xs)
        plant(o, lat)
        op(x, o)
        torch.cuda.synchronize()
        assert torch.isfinite(valid(o, lat)).all(), name
        assert torch.equal(valid(o, lat), valid(clean, lat)), name
        assert torch.isnan(padding(o, lat)).all(), name  # not written
    xd = lat.to_device(b)
    clean = lat.ddd(xd.clone())
    x = xd.clone()
    plant(x, lat)
    o = torch.zeros_like(xd)
    plant(o, lat)
    lat.ddd(x, out=o)
    torch.cuda.synchronize()
    assert torch.equal(valid(o, lat), valid(clean, lat))
    assert torch.isnan(padding(o, lat)).all()
    # whole solves: b and the initial guess with canaries
    for solve in (lambda x, bb: lat.bicgstab_dd_mix(x, bb, 1e-10, 100, 1e-6, 50, 4, 2),
                  lambda x, bb: lat.bicgstab_dd_mix2_hf(x, bb, 1e-10, 100, 1e-6, 50, 4, 2,
                                                        reliable=2)):
        x0 = lat.empty("f64")
        s0 = solve(x0, xd.clone())
        x, bb = lat.empty("f64"), xd.clone()
        plant(x, lat)
        plant(bb, lat)
        s = solve(x, bb)
        torch.cuda.synchronize()
        assert s == s0
        assert torch.equal(valid(x, lat), valid(x0, lat))
    lat.close()
