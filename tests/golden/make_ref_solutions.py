"""Reference solutions of the 48^3x96 precision-form workload, as a small
fixture for comparing the GPU's solutions with the reference's.

One complete solve per kappa of the reference's own bicgstab_dd_mix_
(oracle/_ref, the generic VLENS = 8 build: nx/2 = 24 is not a multiple of
the AVX-512 build's 16) on the workload's fields from the oracle's
generator (bit-equal to the product's host generator): 48^3x96, seeded SU(3)
links (seed 11) after 5 smoothing steps at alpha 0.36, clover-leaf clover at
csw 1.7, Gaussian source (seed 12), antiperiodic in t, the reference's
one-rank partition, tol 1e-10, inner 1e-6 / 50, nsap 4, nm 2.  A full
solution is 2 GB, so the fixture keeps what a comparison needs: the
iteration counts, the true residual, |x|^2, and the solution on 1024 sites
drawn with a fixed seed (the relative error on that sample estimates the
relative error of the whole vector).

    python tests/golden/make_ref_solutions.py [threads]
        -> tests/golden/ref_solutions_48c96.npz  (about 200 KB)

Takes about 10-20 minutes per kappa on 8 host threads and ~40 GB of host memory.
"""
import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
L = (48, 48, 48, 96)
KAPPAS = (0.1365, 0.1355)
N_SAMPLE = 1024


def sample_sites(V, n=N_SAMPLE, seed=0):
    return np.sort(np.random.default_rng(seed).choice(V, n, replace=False))


def main():
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else len(os.sched_getaffinity(0))
    V = int(np.prod(L))
    sites = sample_sites(V)
    out = {"sites": sites, "lattice": np.array(L)}
    meta = {}
    for kappa in KAPPAS:
        spec = dict(L=list(L), tbc=-1, seed=11, n_smear=5, alpha=0.36, csw=1.7, kappa=kappa,
                    src="gauss", tol=1e-10, maxiter=200, tol_s=1e-6, maxiter_s=50, nsap=4,
                    nm=2, warmup=0, steps=1)
        with tempfile.TemporaryDirectory() as td:
            spec["solution_out"] = os.path.join(td, "x.npy")
            env = dict(os.environ, OMP_NUM_THREADS=str(threads), CUDA_VISIBLE_DEVICES="")
            res = subprocess.run([sys.executable, str(ROOT / "oracle" / "refbench.py"),
                                  json.dumps(spec)], capture_output=True, text=True, env=env)
            if res.returncode != 0:
                raise RuntimeError(res.stderr[-2000:])
            r = json.loads(res.stdout.strip().splitlines()[-1])
            x = np.load(spec["solution_out"], mmap_mode="r")
            key = f"{kappa:.4f}"
            out[f"x_{key}"] = np.array(x[sites])
            out[f"xnorm2_{key}"] = np.array(float(np.einsum("ij,ij->", x, x)))
            meta[key] = {k: r[k] for k in ("outer_iters", "inner_iters_per_solve",
                                           "inner_solves_per_solve", "true_rel_resid",
                                           "variant", "threads", "solve_s", "field_sha256",
                                           "plaquette")}
            del x
        print(key, meta[key], flush=True)
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(HERE / "ref_solutions_48c96.npz", **out)


if __name__ == "__main__":
    main()
