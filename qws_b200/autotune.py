"""Autotuner for the DD solver's launch configuration on one GPU.

What it chooses, per (GPU, lattice, solver):

* the SAP block grid NB -- how the lattice is cut into Schwarz blocks.  The
  reference's blocks are the two x-halves of each MPI rank's sub-lattice
  (NB = (2*npe0, npe1, npe2, npe3), qws.cc:224-225); on one GPU any grid
  that divides the lattice into even-extent blocks is available, and the
  grid trades block-solve quality (outer/inner iterations) against the work
  of one sweep;
* the sweep counts (nsap SAP sweeps, nm Richardson steps per block solve);
* threads per CTA of the Dirac-operator kernels (64/128/256);
* the RHS tile -- how many right-hand sides one multi-RHS handle solves at
  once (1..16), by solves/s per RHS.

Every candidate is timed as real solves to the target tolerance on seeded
synthetic fields generated on the device (SU(3) + APE smearing, clover
built on the GPU) with CUDA events on a private stream, one warm-up solve
first; a candidate whose FP64 true residual misses the tolerance is
rejected.  The block grid is searched greedily: from the reference's
one-rank partition (2,1,1,1), double the block count along each direction
in turn and move to the fastest neighbour while it improves the time by
more than `min_gain`.  Results are cached in a JSON file (default: the
`tuning.json` beside this module) keyed by GPU name, lattice, solver and
number of RHS; `lookup` reads the cache without touching the GPU.

    python -m qws_b200.autotune --lattice 32x32x32x64 --solver hf --rhs-tile 16
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

DEFAULT_CACHE = Path(__file__).with_name("tuning.json")
REFERENCE_NB = (2, 1, 1, 1)
DEFAULTS = {"NB": list(REFERENCE_NB), "nsap": 4, "nm": 2, "hop_threads": 128, "rhs_tile": 1}
SWEEPS = ((4, 2), (3, 2), (4, 3), (3, 3), (2, 4), (5, 2))


def gpu_name():
    import torch

    return torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"


def cache_key(gpu, L, solver, nrhs):
    return f"{gpu}|{'x'.join(map(str, L))}|{solver}|nrhs{nrhs}"


def valid_grid(L, NB, min_block=4):
    """NB[0] even, NB[1..3] 1 or even, every block extent even and >= min_block."""
    if NB[0] % 2:
        return False
    for mu in range(4):
        if NB[mu] < 1 or L[mu] % NB[mu]:
            return False
        if mu > 0 and NB[mu] != 1 and NB[mu] % 2:
            return False
        B = L[mu] // NB[mu]
        if B < min_block or B % 2:
            return False
    return True


def neighbours(L, NB, min_block=4):
    """Grids with the block count doubled along one direction."""
    out = []
    for mu in range(4):
        n = list(NB)
        n[mu] = 2 if n[mu] == 1 else 2 * n[mu]
        if valid_grid(L, n, min_block):
            out.append(tuple(n))
    return out


def lookup(L, solver="hf", nrhs=1, cache=DEFAULT_CACHE, gpu=None):
    """The cached choice for this GPU and lattice, or None."""
    p = Path(cache)
    if not p.exists():
        return None
    known = json.loads(p.read_text())
    return known.get(cache_key(gpu or gpu_name(), tuple(L), solver, nrhs))


def store(entry, cache=DEFAULT_CACHE):
    p = Path(cache)
    known = json.loads(p.read_text()) if p.exists() else {}
    known[cache_key(entry["gpu"], tuple(entry["lattice"]), entry["solver"], entry["nrhs"])] = entry
    p.write_text(json.dumps(known, indent=1, sort_keys=True) + "\n")


class Tuner:
    """Times candidate configurations of one lattice size and solver.

    solver: "hf" (bicgstab_dd_mix2_hf, the precision form) or "plain"
    (bicgstab_dd_mix)."""

    def __init__(self, L, solver="hf", kappa=0.1365, csw=1.7, tol=1e-10, tol_s=1e-6,
                 maxiter=200, maxiter_s=50, reliable=5, seed=11, reps=2, min_block=4,
                 min_gain=0.02, log=None):
        import torch

        import qws_b200

        self.q, self.torch = qws_b200, torch
        self.L, self.solver = tuple(int(v) for v in L), solver
        self.kappa, self.csw, self.tol, self.tol_s = kappa, csw, tol, tol_s
        self.maxiter, self.maxiter_s, self.reliable = maxiter, maxiter_s, reliable
        self.seed, self.reps, self.min_block, self.min_gain = seed, reps, min_block, min_gain
        self.log = log or (lambda msg: None)
        self.stream = torch.cuda.Stream()
        self.table = []
        self._lat = None
        self._src = [qws_b200.gen_source(self.L, seed + 1 + k, "gauss") for k in range(2)]

    # ---- fields ---------------------------------------------------------------
    def lattice(self, NB):
        """A lattice on block grid NB with the seeded fields (one kept at a time)."""
        NB = tuple(NB)
        if self._lat is not None and self._lat.NB == NB:
            return self._lat
        self.close()
        lat = self.q.Lattice(self.L, NB, tbc=-1, kappa=self.kappa, stream=self.stream)
        lat.gen_gauge_device(self.seed, 5, 0.36)
        lat.build_clover(self.csw)
        self._lat = lat
        return lat

    def close(self):
        if self._lat is not None:
            self._lat.close()
            self._lat = None
            self.torch.cuda.empty_cache()

    # ---- one measurement --------------------------------------------------------
    def measure(self, NB, nsap, nm, hop_threads=128, nrhs=1):
        torch = self.torch
        lat = self.lattice(NB)
        lat.set_hop_threads(hop_threads)
        h = None
        row = {"NB": list(NB), "nsap": nsap, "nm": nm, "hop_threads": hop_threads, "nrhs": nrhs}
        try:
            h = lat.batch(nrhs, stream=self.stream) if nrhs > 1 else lat
            with torch.cuda.stream(self.stream):
                src = self._src[0] if nrhs == 1 else \
                    np.stack([self._src[k % 2] for k in range(nrhs)])
                b = h.to_device(src)
                x = h.empty("f64")

                def solve():
                    x.zero_()
                    if self.solver == "plain":
                        return h.bicgstab_dd_mix(x, b, self.tol, self.maxiter, self.tol_s,
                                                 self.maxiter_s, nsap, nm)
                    return h.bicgstab_dd_mix2_hf(x, b, self.tol, self.maxiter, self.tol_s,
                                                 self.maxiter_s, nsap, nm, reliable=self.reliable)

                solve()
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(self.stream)
                for _ in range(self.reps):
                    st = solve()
                e1.record(self.stream)
                torch.cuda.synchronize()
                true = h.true_residual(x, b)
                true = max(true) if nrhs > 1 else true
                ms = e0.elapsed_time(e1) / self.reps
            row.update(ms=round(ms, 3), ms_per_rhs=round(ms / nrhs, 3),
                       outer_iters=st["outer_iters"], inner_iters=st["inner_iters"],
                       true_rel_resid=true, ok=bool(true < self.tol))
        except Exception as e:  # noqa: BLE001 -- e.g. out of memory: the candidate is out
            row.update(ms=None, ok=False, error=f"{type(e).__name__}: {str(e)[-200:]}")
        finally:
            if h is not None and h is not lat:
                h.close()
            lat.set_hop_threads(128)
            torch.cuda.empty_cache()
        self.table.append(row)
        self.log(f"tune {row}")
        return row

    # ---- the search -------------------------------------------------------------
    def _better(self, a, b):
        """a beats b by more than min_gain (per RHS)."""
        return a["ok"] and (b is None or not b["ok"] or
                            a["ms_per_rhs"] < (1.0 - self.min_gain) * b["ms_per_rhs"])

    def run(self, rhs_tile_max=1, sweeps=SWEEPS, threads=(64, 128, 256)):
        t0 = time.time()
        try:
            best = self.measure(REFERENCE_NB, 4, 2)
            # block grid: greedy descent from the reference partition
            while True:
                cand = [self.measure(n, best["nsap"], best["nm"])
                        for n in neighbours(self.L, tuple(best["NB"]), self.min_block)]
                cand = [c for c in cand if c["ok"]]
                top = min(cand, key=lambda c: c["ms_per_rhs"]) if cand else None
                if top is None or not self._better(top, best):
                    break
                best = top
            # sweep counts on that grid
            for nsap, nm in sweeps:
                if (nsap, nm) == (best["nsap"], best["nm"]):
                    continue
                r = self.measure(best["NB"], nsap, nm)
                if self._better(r, best):
                    best = r
            # CTA size of the Dirac-operator kernels
            for th in threads:
                if th == best["hop_threads"]:
                    continue
                r = self.measure(best["NB"], best["nsap"], best["nm"], th)
                if self._better(r, best):
                    best = r
            # RHS tile: solves per second per RHS on a multi-RHS handle
            tile = best
            nr = 2
            while nr <= rhs_tile_max:
                r = self.measure(best["NB"], best["nsap"], best["nm"], best["hop_threads"], nr)
                if not r["ok"]:
                    break
                if self._better(r, tile):
                    tile = r
                nr *= 2
        finally:
            self.close()
        ref = self.table[0]
        return {
            "gpu": gpu_name(), "lattice": list(self.L), "solver": self.solver,
            "nrhs": rhs_tile_max, "NB": best["NB"], "nsap": best["nsap"], "nm": best["nm"],
            "hop_threads": best["hop_threads"], "rhs_tile": tile["nrhs"],
            "ms": best["ms"], "ms_per_rhs_at_tile": tile["ms_per_rhs"],
            "reference_partition_ms": ref["ms"] if ref["ok"] else None,
            "kappa": self.kappa, "csw": self.csw, "tol": self.tol,
            "candidates": len(self.table), "tuning_s": round(time.time() - t0, 1),
        }


def autotune(L, solver="hf", rhs_tile_max=1, cache=DEFAULT_CACHE, retune=False, log=None,
             write=True, sweeps=SWEEPS, **kw):
    """The cached choice, or a fresh tuning run (stored in the cache when
    `write`).  Returns (entry, table); table is empty for a cache hit."""
    if not retune and cache is not None:
        hit = lookup(L, solver, rhs_tile_max, cache)
        if hit is not None:
            return dict(hit, source="cache"), []
    t = Tuner(L, solver, log=log, **kw)
    entry = t.run(rhs_tile_max, sweeps)
    if cache is not None and write:
        store(entry, cache)
    return dict(entry, source="tuned"), t.table


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--lattice", action="append", required=True, help="e.g. 32x32x32x64")
    ap.add_argument("--solver", default="hf", choices=["hf", "plain"])
    ap.add_argument("--rhs-tile", type=int, default=1, help="largest RHS tile to try")
    ap.add_argument("--cache", default=str(DEFAULT_CACHE))
    ap.add_argument("--table", default=None, help="append every timed candidate to this JSONL file")
    ap.add_argument("--retune", action="store_true")
    a = ap.parse_args()
    for s in a.lattice:
        L = tuple(int(v) for v in s.split("x"))
        entry, table = autotune(L, a.solver, a.rhs_tile, a.cache, a.retune,
                                log=lambda m: print(m, flush=True))
        print(json.dumps(entry), flush=True)
        if a.table and table:
            with open(a.table, "a") as f:
                for row in table:
                    f.write(json.dumps(dict(row, lattice=s, solver=a.solver)) + "\n")


if __name__ == "__main__":
    main()
