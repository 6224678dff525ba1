"""Time complete solves of the reference's own CPU solver (oracle/_ref, built
from its sources by oracle/Makefile) on a benchmark workload.

Test / baseline infrastructure: run by bench.py's cpu_baseline leg and by
`bench.py --impl reference`, always as a separate process (the reference
prints to stdout and keeps process-global state).  The last stdout line is
one JSON object.  Nothing here loads the product library: the inputs come
from the oracle's restatement of the benchmark's field generator
(oracle/fields_oracle.cc, bit-equal to the product's, tests/test_fields.py),
and their SHA-256 digests are reported so the GPU arm can show that it
solved the same arrays.

What is timed: `warmup` + `steps` calls of the reference's
bicgstab_dd_mix_(x, b, tol, conviter, maxiter, tol_s, maxiter_s, nsap, nm)
(bicgstab_dd_mix.cc:105-388), x zeroed before each call, exactly as main.cc
calls it (main.cc:258-313), each one a full solve to `tol`; host clock
around each call.  The outer iteration count is the reference's conviter;
the inner counts come from the reference's own call counters (timing.c,
read once at the end: ref_timing_dump in oracle/ref_glue.cc) divided by the
number of solves.  The true relative residual |b - D x| / |b| of the last
solution uses the reference's own ddd_d_.  With "solution_out" the last
solution is saved (natural layout [V, 24], FP64) for the GPU arm to compare.

Usage: python oracle/refbench.py '<json spec>'
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))


def cpu_has(flag):
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                return flag in line.split()
    except OSError:
        pass
    return False


def pick_variant(L):
    """QWS needs nx/2 to be a multiple of its single-precision lane width
    VLENS (qws.cc:143-146): VLENS 16 (the AVX-512 intrinsics build) where it
    is, else the generic build with VLENS 8."""
    nxh = L[0] // 2
    isa = "avx512" if cpu_has("avx512f") else "avx2"
    if nxh % 16 == 0:
        return f"v8s16_{isa}"
    if nxh % 8 == 0:
        return f"v8s8_{isa}"
    raise ValueError(f"no reference build for nx/2 = {nxh}")


def sha256(a):
    return hashlib.sha256(memoryview(np.ascontiguousarray(a)).cast("B")).hexdigest()


def read_counts(path):
    """routine -> calls, from the reference's timing table"""
    out = {}
    for line in Path(path).read_text().splitlines():
        parts = line.split()
        if len(parts) == 5 and parts[0].isdigit():
            out[parts[1]] = int(parts[2])
    return out


def main():
    spec = json.loads(sys.argv[1])
    import qwsref
    from qwsref import RefQWS, aligned_empty

    L = tuple(spec["L"])
    variant = spec.get("variant") or pick_variant(L)
    t0 = time.time()
    U, plaq = qwsref.gen_gauge(L, spec["seed"], spec["n_smear"], spec["alpha"])
    C = qwsref.gen_clover(U, L, spec["csw"], spec["kappa"])
    b = qwsref.gen_source(L, spec["seed"] + 1, spec.get("src", "gauss"))
    digests = {"gauge": sha256(U), "clover": sha256(C), "source": sha256(b)}
    t_gen = time.time() - t0

    r = RefQWS(variant, L, tbc=spec["tbc"])
    r.set_kappa(spec["kappa"])
    r.set_fields(U, C)
    del U, C
    bq = r.to_d(b)
    x = aligned_empty(bq.size, np.float64)
    I = lambda v: ctypes.byref(ctypes.c_int(int(v)))
    D = lambda v: ctypes.byref(ctypes.c_double(float(v)))
    conv = ctypes.c_int(0)

    def solve():
        x[:] = 0.0
        r.lib.bicgstab_dd_mix_(ctypes.c_void_p(x.ctypes.data), ctypes.c_void_p(bq.ctypes.data),
                               D(spec["tol"]), ctypes.byref(conv), I(spec["maxiter"]),
                               D(spec["tol_s"]), I(spec["maxiter_s"]), I(spec["nsap"]),
                               I(spec["nm"]))

    warm, timed = [], []
    outer = []
    for k in range(int(spec.get("warmup", 0)) + int(spec.get("steps", 1))):
        t = time.perf_counter()
        solve()
        dt = time.perf_counter() - t
        (warm if k < int(spec.get("warmup", 0)) else timed).append(dt)
        outer.append(conv.value)
    n_solves = len(warm) + len(timed)

    # true relative residual of the last solution with the reference's own D
    dx = aligned_empty(bq.size, np.float64)
    r.call("ddd_d_", dx, x)
    true_rel = float(np.linalg.norm(bq - dx) / np.linalg.norm(bq))
    if spec.get("solution_out"):
        np.save(spec["solution_out"], r.from_d(x))

    with tempfile.TemporaryDirectory() as td:
        tf = os.path.join(td, "timing.txt")
        r.lib.ref_timing_dump(tf.encode())
        calls = read_counts(tf)
    per = lambda name: calls.get(name, 0) / n_solves
    threads = int(os.environ.get("OMP_NUM_THREADS", "0") or 0) or len(os.sched_getaffinity(0))
    out = {
        "variant": variant,
        "threads": threads,
        "solve_s": timed,
        "warmup_solve_s": warm,
        "solves_per_s": len(timed) / sum(timed),
        "outer_iters": outer[-1],
        "outer_iters_all": sorted(set(outer)),
        "inner_solves_per_solve": per("bicgstab_precdd_s_"),
        "inner_iters_per_solve": per("bicgstab_precdd_s_iter_"),
        "prec_ddd_s_per_solve": per("prec_ddd_s_"),
        "true_rel_resid": true_rel,
        "plaquette": plaq,
        "field_sha256": digests,
        "t_fieldgen_s": t_gen,
        "sample": (f"reference {variant} (built from its sources) on {threads} host threads: "
                   f"{len(timed)} complete bicgstab_dd_mix_ solves of the "
                   f"{'x'.join(map(str, L))} lattice to tol {spec['tol']:g} after "
                   f"{len(warm)} untimed, x = 0 start, host clock per call"),
    }
    sys.stdout.write("\n" + json.dumps(out) + "\n")
    sys.stdout.flush()


if __name__ == "__main__":
    main()
