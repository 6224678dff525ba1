"""Time the reference's own CPU solver (oracle/_ref, built from its sources)
on a bounded sample of a workload, and scale it to solves per second.

Test / baseline infrastructure: run by bench.py's cpu_baseline leg and by
`bench.py --impl reference`, always as a separate process (the reference
prints to stdout and keeps process-global state).  The last stdout line is
one JSON object.

What is timed (all on the same seeded fields and source as the GPU arm):
  t_iter   one inner BiCGStab iteration: bicgstab_precdd_s_ with tol < 0 and
           maxiter = SAMPLE_ITERS, divided by SAMPLE_ITERS (two prec_ddd_s_
           calls plus the reductions and updates, bicgstab_precdd_s.cc:213-545)
  t_prec_s one prec_s_ call (the final M application of approx_inv_dirac_op)
  t_ddd_d  one ddd_d_ call (FP64 D of the outer loop)
A solve is then  inner_iters * t_iter + n_approx * t_prec_s + n_ddd_d * t_ddd_d,
with the iteration counts of a full solve of this workload passed in by
the caller (they are a property of the algorithm: the reference and the GPU
path run the same iterations, see tests/test_gpu_dd.py).

Usage: python oracle/refbench.py '<json spec>'
"""
from __future__ import annotations

import ctypes
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent))

SAMPLE_ITERS = 2


def cpu_has(flag):
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                return flag in line.split()
    except OSError:
        pass
    return False


def pick_variant(L):
    nxh = L[0] // 2
    isa = "avx512" if cpu_has("avx512f") else "avx2"
    if nxh % 16 == 0:
        return f"v8s16_{isa}"
    if nxh % 8 == 0:
        return f"v8s8_{isa}"
    raise ValueError(f"no reference build for nx/2 = {nxh}")


def main():
    spec = json.loads(sys.argv[1])
    from qwsref import RefQWS, aligned_empty

    import qws_b200

    L = tuple(spec["L"])
    variant = spec.get("variant") or pick_variant(L)
    t0 = time.time()
    U, plaq = qws_b200.gen_gauge(L, spec["seed"], spec["n_smear"], spec["alpha"])
    C = qws_b200.gen_clover(U, L, spec["csw"], spec["kappa"])
    b = qws_b200.gen_source(L, spec["seed"] + 1, spec.get("src", "gauss"))
    t_gen = time.time() - t0

    r = RefQWS(variant, L, tbc=spec["tbc"])
    r.set_kappa(spec["kappa"])
    r.set_fields(U, C)
    del U, C
    nsap, nm = ctypes.c_int(spec["nsap"]), ctypes.c_int(spec["nm"])
    bd = r.to_d(b)
    bs = r.to_s((b / np.linalg.norm(b)).astype(np.float32))
    outd = aligned_empty(bd.size, np.float64)
    outs = aligned_empty(bs.size, np.float32)

    warm = set()

    def timed(fn, reps=1, key=None):
        if key not in warm:  # first-touch of the reference's static scratch
            fn()
            warm.add(key)
        t = time.perf_counter()
        for _ in range(reps):
            fn()
        return (time.perf_counter() - t) / reps

    tol = ctypes.c_double(-1.0)
    it = ctypes.c_int(0)
    mx = ctypes.c_int(SAMPLE_ITERS)
    counts = spec["counts"]
    samples = []
    # repeats > 1: the first `warmup` samples are discarded by the caller
    for _ in range(int(spec.get("repeats", 1))):
        t_iter = timed(lambda: r.call("bicgstab_precdd_s_", outs, bs, ctypes.byref(tol),
                                      ctypes.byref(it), ctypes.byref(mx), ctypes.byref(nsap),
                                      ctypes.byref(nm)), key="iter") / SAMPLE_ITERS
        t_prec_s = timed(lambda: r.call("prec_s_", outs, bs, ctypes.byref(nsap),
                                        ctypes.byref(nm)), key="prec")
        t_ddd_d = timed(lambda: r.call("ddd_d_", outd, bd), key="ddd")
        samples.append(counts["inner_iters"] * t_iter + counts["n_approx"] * t_prec_s +
                       counts["n_ddd_d"] * t_ddd_d)
    t_solve = samples[-1]
    threads = int(os.environ.get("OMP_NUM_THREADS", "0") or 0) or len(os.sched_getaffinity(0))
    out = {
        "variant": variant,
        "threads": threads,
        "t_inner_iter_s": t_iter,
        "t_prec_s_s": t_prec_s,
        "t_ddd_d_s": t_ddd_d,
        "t_solve_s": t_solve,
        "solves_per_s": 1.0 / t_solve,
        "solves_per_s_samples": [1.0 / t for t in samples],
        "plaquette": plaq,
        "t_fieldgen_s": t_gen,
        "sample": (f"reference {variant} on {threads} threads: bicgstab_precdd_s_ "
                   f"{SAMPLE_ITERS} iterations + 1 prec_s_ + 1 ddd_d_ on the full "
                   f"{'x'.join(map(str, L))} lattice, scaled by the iteration counts of a "
                   f"1e-10 solve ({counts['inner_iters']} inner iterations, "
                   f"{counts['n_approx']} approx_inv, {counts['n_ddd_d']} ddd_d_)"),
    }
    sys.stdout.write("\n" + json.dumps(out) + "\n")
    sys.stdout.flush()


if __name__ == "__main__":
    main()
