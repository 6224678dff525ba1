"""Parity with the reference itself on the benchmark's own workloads.

The reference's solver (oracle/_ref, compiled from its sources) runs in a
subprocess through oracle/refbench.py -- the same harness as the benchmark's
reference arm -- on inputs from the oracle's generator; the GPU solves the
same arrays (the product's generator is bit-equal to the oracle's,
tests/test_fields.py; here the SHA-256 digests are compared as well).

* The plain CPU-runnable workload exactly: 32x6x4x3, random SU(3) links
  (no smoothing), csw 1.0, kappa 0.125, periodic in every direction, tol < 0
  so both run a fixed 5 outer (iter = 1..maxiter-1 with maxiter 6,
  bicgstab_dd_mix.cc:170) x 2 inner solves x 50 iterations, nsap 4, nm 2,
  the reference's one-rank partition.  The outer solve reaches the FP64
  floor, so the solutions agree to roundoff (1e-13 relative).
* A 16^3x32 stand-in for the 32^3x64 GPU-scale workload (same generator
  settings: 5 smoothing steps, csw 1.7, kappa 0.1365, tol 1e-10 outer / 1e-6
  inner, 50 inner iterations at most): solution within 1e-10 relative of
  the reference's, outer count within +-1, inner count within +-1 per inner
  solve.
"""
import hashlib
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import qws_b200
from qwsref import REF_DIR

ROOT = Path(__file__).resolve().parents[1]
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not any(REF_DIR.glob("*/libqwsref.so")),
                                 reason="oracle/_ref not built (make -C oracle ref)")]

CONFIG1 = dict(L=(32, 6, 4, 3), tbc=1, seed=1, n_smear=0, alpha=0.36, csw=1.0, kappa=0.125,
               src="gauss", tol=-1.0, maxiter=6, tol_s=-1.0, maxiter_s=50, nsap=4, nm=2)
STANDIN2 = dict(L=(16, 16, 16, 32), tbc=-1, seed=11, n_smear=5, alpha=0.36, csw=1.7,
                kappa=0.1365, src="gauss", tol=1e-10, maxiter=200, tol_s=1e-6, maxiter_s=50,
                nsap=4, nm=2)


def reference_solve(w, tmp_path):
    spec = {k: (list(v) if isinstance(v, tuple) else v) for k, v in w.items()}
    spec.update(warmup=0, steps=1, solution_out=str(tmp_path / "x_ref.npy"))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    env.setdefault("OMP_NUM_THREADS", str(len(os.sched_getaffinity(0))))
    res = subprocess.run([sys.executable, str(ROOT / "oracle" / "refbench.py"), json.dumps(spec)],
                         capture_output=True, text=True, env=env, timeout=1200)
    assert res.returncode == 0, res.stderr[-2000:]
    out = json.loads(res.stdout.strip().splitlines()[-1])
    return out, np.load(tmp_path / "x_ref.npy")


def gpu_solve(w):
    L = w["L"]
    U, _ = qws_b200.gen_gauge(L, w["seed"], w["n_smear"], w["alpha"])
    C = qws_b200.gen_clover(U, L, w["csw"], w["kappa"])
    b = qws_b200.gen_source(L, w["seed"] + 1, w["src"])
    h = lambda a: hashlib.sha256(memoryview(np.ascontiguousarray(a)).cast("B")).hexdigest()
    digests = {"gauge": h(U), "clover": h(C), "source": h(b)}
    lat = qws_b200.Lattice(L, (2, 1, 1, 1), tbc=w["tbc"], kappa=w["kappa"])
    try:
        lat.load_fields(U, C)
        bd, x = lat.to_device(b), lat.empty("f64")
        st = lat.bicgstab_dd_mix(x, bd, w["tol"], w["maxiter"], w["tol_s"], w["maxiter_s"],
                                 w["nsap"], w["nm"])
        return lat.to_host(x), st, lat.true_residual(x, bd), digests
    finally:
        lat.close()


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_plain_cpu_workload_matches_reference(tmp_path):
    ref, x_ref = reference_solve(CONFIG1, tmp_path)
    x, st, true_rel, digests = gpu_solve(CONFIG1)
    assert digests == ref["field_sha256"]
    assert np.isfinite(x).all() and np.isfinite(x_ref).all()
    # fixed iteration counts: 5 outer, 2 x 50 inner each
    assert st["outer_iters"] == ref["outer_iters"] == 6
    assert st["inner_iters"] == ref["inner_iters_per_solve"] == 500
    assert rel(x, x_ref) < 1e-13
    assert true_rel < 1e-14 and ref["true_rel_resid"] < 1e-14


def test_gpu_scale_standin_matches_reference(tmp_path):
    ref, x_ref = reference_solve(STANDIN2, tmp_path)
    x, st, true_rel, digests = gpu_solve(STANDIN2)
    assert digests == ref["field_sha256"]
    assert abs(st["outer_iters"] - ref["outer_iters"]) <= 1
    assert abs(st["inner_iters"] - ref["inner_iters_per_solve"]) <= ref["inner_solves_per_solve"]
    assert true_rel < 1e-10 and ref["true_rel_resid"] < 1e-10
    assert rel(x, x_ref) < 1e-10
