"""The autotuner (qws_b200.autotune): the block grids it may choose are the
ones the library accepts (NB[0] even, NB[1..3] 1 or even, even block
extents of at least min_block sites), its greedy step doubles one
direction's block count at a time, and the cache round-trips per (GPU,
lattice, solver, RHS tile).  On the GPU: every CTA size of the Dirac
kernels gives bit-equal operators, and a tuning run on a small lattice
returns a configuration whose solve meets the tolerance."""
import json

import numpy as np
import pytest

from qws_b200 import autotune


def test_valid_grid():
    L = (32, 32, 32, 64)
    assert autotune.valid_grid(L, (2, 1, 1, 1))
    assert autotune.valid_grid(L, (4, 2, 2, 8))
    assert not autotune.valid_grid(L, (1, 1, 1, 1))      # NB[0] odd
    assert not autotune.valid_grid(L, (2, 3, 1, 1))      # NB[1] odd and not 1
    assert not autotune.valid_grid(L, (16, 1, 1, 1))     # block extent 2 < 4
    assert not autotune.valid_grid((24, 24, 24, 48), (2, 1, 1, 16))  # extent 3 is odd
    assert not autotune.valid_grid((32, 6, 4, 3), (2, 1, 1, 1))      # t extent 3 is odd


def test_neighbours():
    L = (48, 48, 48, 96)
    assert autotune.neighbours(L, (2, 1, 1, 1)) == [(4, 1, 1, 1), (2, 2, 1, 1), (2, 1, 2, 1),
                                                    (2, 1, 1, 2)]
    # 48/8 = 6 sites: one more doubling of x would give 3 (odd)
    assert (16, 1, 1, 1) not in autotune.neighbours(L, (8, 1, 1, 1))
    for n in autotune.neighbours(L, (4, 4, 4, 4)):
        assert autotune.valid_grid(L, n)
        assert sum(a != b for a, b in zip(n, (4, 4, 4, 4))) == 1


def test_cache_roundtrip(tmp_path):
    p = tmp_path / "tuning.json"
    e = {"gpu": "NVIDIA B200", "lattice": [32, 32, 32, 64], "solver": "hf", "nrhs": 1,
         "NB": [2, 2, 2, 4], "nsap": 4, "nm": 3, "hop_threads": 128, "rhs_tile": 1}
    autotune.store(e, p)
    autotune.store(dict(e, solver="plain", NB=[2, 2, 2, 2]), p)
    assert autotune.lookup((32, 32, 32, 64), "hf", 1, p, gpu="NVIDIA B200")["NB"] == [2, 2, 2, 4]
    assert autotune.lookup((32, 32, 32, 64), "plain", 1, p, gpu="NVIDIA B200")["NB"] == [2, 2, 2, 2]
    assert autotune.lookup((32, 32, 32, 64), "hf", 16, p, gpu="NVIDIA B200") is None
    assert autotune.lookup((32, 32, 32, 64), "hf", 1, p, gpu="other") is None
    assert len(json.loads(p.read_text())) == 2


def test_shipped_cache_is_valid():
    """Every committed tuning entry names a block grid the library accepts."""
    if not autotune.DEFAULT_CACHE.exists():
        pytest.skip("no tuning cache shipped")
    for key, e in json.loads(autotune.DEFAULT_CACHE.read_text()).items():
        assert autotune.valid_grid(tuple(e["lattice"]), tuple(e["NB"])), key
        assert e["hop_threads"] in (64, 128, 256) and e["nsap"] >= 1 and e["nm"] >= 1, key


@pytest.mark.gpu
@pytest.mark.parametrize("threads", [64, 256])
def test_hop_threads_bit_equal(threads):
    import qws_b200

    L = (8, 8, 8, 16)
    U, _ = qws_b200.gen_gauge(L, 7, 5, 0.36)
    C = qws_b200.gen_clover(U, L, 1.7, 0.1365)
    lat = qws_b200.Lattice(L, (2, 2, 2, 2), tbc=-1, kappa=0.1365)
    try:
        lat.load_fields(U, C)
        s = qws_b200.gen_source(L, 3, "gauss")
        d, f = lat.to_device(s), lat.to_device(s.astype(np.float32))
        B = lat.batch(4)
        S4 = np.stack([s] * 4).astype(np.float32)
        f4 = B.to_device(S4)

        def run():
            return {"ddd_d": lat.to_host(lat.ddd(d)), "ddd_s": lat.to_host(lat.ddd(f)),
                    "prec": lat.to_host(lat.prec(f, 4, 2)), "prec_h": lat.to_host(lat.prec_h(f, 4, 2)),
                    "prec4": B.to_host(B.prec(f4, 4, 2))}

        want = run()
        lat.set_hop_threads(threads)
        B.set_hop_threads(threads)
        got = run()
        for k in want:
            assert np.array_equal(got[k], want[k]), k
        B.close()
        with pytest.raises(qws_b200.QwsgError):
            lat.set_hop_threads(96)
    finally:
        lat.close()


@pytest.mark.gpu
def test_tuning_run_small(tmp_path):
    L = (8, 8, 8, 16)
    cache = tmp_path / "tuning.json"
    entry, table = autotune.autotune(L, "hf", 2, cache=cache, reps=1,
                                     sweeps=((4, 2), (3, 2)), kappa=0.1300)
    assert entry["source"] == "tuned" and table
    assert autotune.valid_grid(L, tuple(entry["NB"]))
    assert entry["rhs_tile"] in (1, 2)
    chosen = [r for r in table if r["NB"] == entry["NB"] and r["nsap"] == entry["nsap"]
              and r["nm"] == entry["nm"] and r["hop_threads"] == entry["hop_threads"]]
    assert chosen and all(r["ok"] and r["true_rel_resid"] < 1e-10 for r in chosen)
    again, table2 = autotune.autotune(L, "hf", 2, cache=cache)
    assert again["source"] == "cache" and not table2 and again["NB"] == entry["NB"]
