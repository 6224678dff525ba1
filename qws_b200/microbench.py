"""Per-kernel microbenchmark of the DD operator kernels on one GPU.

    python -m qws_b200.microbench --lattice 32,32,32,64 --kernel jinv --iters 20

Builds seeded synthetic fields of the given lattice (SU(3) + 5 APE steps,
clover-leaf clover), then times `iters` launches of one operator with CUDA
events on the library's stream and prints one JSON line with the average
launch time and the algorithmic HBM bandwidth (bytes each launch must move:
spinors read and written once, links and clover once per site).

Kernels: jinv (one Richardson step on one colour), dslash_s / dslash_d (full
D in FP32 / FP64), block_s (block-interior D on one colour), update_s (the SAP
half-sweep update s += in - D_blk a on one colour), face_s (face hops of one
colour), block_d (block-interior D in FP64), jinv_h / face_h / update_h (the
FP16-storage Richardson step, face hops and SAP update through the
single-operator entry points, conversions included), prec
(the whole SAP preconditioner prec_ddd_s_), prec_h (the FP16-storage SAP),
solve_hf (a whole precision-form solve to 1e-10; --new-kappa rebuilds the
clover term for another kappa before each, as a serving loop sees them).  --nrhs N runs the launch on a multi-RHS handle (N
right-hand sides per launch; spinor bytes count N times, links and clover
once).

    python -m qws_b200.microbench --kernel solve_group --count 48 \
        --volumes 8x8x8x8,12x12x12x24,16x16x16x32,24x24x24x48

solve_group: `count` precision-form solves to 1e-10 on lattices drawn from
`volumes` (each its own seeded gauge field, generated on the GPU; block grid
and sweep counts from the autotuner's cache for the volume), all fields and
sources resident: the solves one after another on one stream, then the same
solves as one group solve (qws_b200.group_solve), each timed with CUDA
events over `iters` repetitions.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def main():
    import torch

    import qws_b200

    ap = argparse.ArgumentParser()
    ap.add_argument("--lattice", default="32,32,32,64")
    ap.add_argument("--blocks", default="2,1,1,1")
    ap.add_argument("--kernel", default="jinv")
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--kappa", type=float, default=0.1365)
    ap.add_argument("--csw", type=float, default=1.7)
    ap.add_argument("--nrhs", type=int, default=1)
    ap.add_argument("--new-kappa", action="store_true",
                    help="solve_hf: a different kappa (clover rebuilt on the GPU) before every "
                         "solve, as a serving loop sees them")
    ap.add_argument("--links18", action="store_true",
                    help="FP32 kernels read 18-real links even for SU(3) fields")
    ap.add_argument("--count", type=int, default=48, help="solve_group: number of solves")
    ap.add_argument("--volumes", default="8x8x8x8,12x12x12x24,16x16x16x32,24x24x24x48",
                    help="solve_group: lattice volumes drawn uniformly")
    a = ap.parse_args()
    if a.kernel == "solve_group":
        return solve_group(a)
    L = tuple(int(v) for v in a.lattice.split(","))
    NB = tuple(int(v) for v in a.blocks.split(","))
    U, plaq = qws_b200.gen_gauge(L, 11, 5, 0.36)
    C = qws_b200.gen_clover(U, L, a.csw, a.kappa)
    b = qws_b200.gen_source(L, 12)
    st = torch.cuda.Stream()
    base = qws_b200.Lattice(L, NB, tbc=-1, kappa=a.kappa, stream=st)
    if a.links18:
        base.set_link_compression(0)
    base.load_fields(U, C)
    links12 = base.link_compression()
    del U, C
    V, nr = base.V, a.nrhs
    lat = base if nr == 1 else base.batch(nr, stream=st)
    if nr > 1:
        b = np.stack([b] * nr)
    # algorithmic bytes per site: spinor streams per RHS + links + clover
    # (FP32 links: 48 instead of 72 B per direction in 12-real form)
    sp32, sp64, lc32, lc64 = 96 * nr, 192 * nr, (192 if links12 else 288) + 288, 1152
    with torch.cuda.stream(st):
        bs = lat.to_device(b.astype(np.float32))
        bd = lat.to_device(b)
        out_s = lat.empty("f32")
        out_d = lat.empty("f64")
        k = a.kernel
        if k == "jinv":
            fn, nbytes = (lambda: lat.jinv(bs, 0, 1, out=out_s)), (V // 2) * (3 * sp32 + lc32)
        elif k == "dslash_s":
            fn, nbytes = (lambda: lat.ddd(bs, out=out_s)), V * (2 * sp32 + lc32)
        elif k == "dslash_d":
            fn, nbytes = (lambda: lat.ddd(bd, out=out_d)), V * (2 * sp64 + lc64)
        elif k == "block_s":
            fn, nbytes = (lambda: lat.ddd_in(bs, 0, out=out_s)), (V // 2) * (2 * sp32 + lc32)
        elif k == "update_s":  # one SAP half-sweep update on one colour: s += in - D_blk a
            rhs = lat.to_device(np.roll(b, 1, axis=-2).astype(np.float32))  # its own stream
            fn = lambda: lat.sap_update(out_s, bs, rhs, 0)
            nbytes = (V // 2) * (4 * sp32 + lc32)  # a, in, s read + written; links, clover
        elif k == "update_h":  # the same update with the FP16-storage kernel (conversions included)
            rhs = lat.to_device(np.roll(b, 1, axis=-2).astype(np.float32))
            fn, nbytes = (lambda: lat.sap_update(out_s, bs, rhs, 0, half=True)), None
        elif k == "block_d":
            fn, nbytes = (lambda: lat.ddd_in(bd, 0, out=out_d)), (V // 2) * (2 * sp64 + lc64)
        elif k == "face_s":
            fn, nbytes = (lambda: lat.ddd_out(bs, 0, 0.1, out=out_s)), None
        elif k == "jinv_h":  # FP16 storage: with the conversions of the single-op entry point
            fn, nbytes = (lambda: lat.jinv_h(bs, 0, 1, out=out_s)), None
        elif k == "face_h":
            fn, nbytes = (lambda: lat.ddd_out_h(bs, 0, 0.1, out=out_s)), None
        elif k == "solve_hf":  # one precision-form solve to 1e-10 from x = 0
            xs = lat.empty("f64")
            state = {"n": 0}

            def fn():
                if a.new_kappa:
                    state["n"] += 1
                    lat.set_kappa(a.kappa - 1e-4 * (state["n"] % 50))
                    lat.build_clover(a.csw)
                xs.zero_()
                lat.bicgstab_dd_mix2_hf(xs, bd, 1e-10, 100, 1e-6, 50, 4, 2, reliable=5)
            nbytes = None
        elif k == "prec":
            fn, nbytes = (lambda: lat.prec_ddd(bs, 4, 2, out=out_s)), None
        elif k == "prec_h":
            fn, nbytes = (lambda: lat.prec_h(bs, 4, 2, out=out_s)), None
        else:
            raise SystemExit(f"unknown kernel {k}")
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(a.iters):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
    us = e0.elapsed_time(e1) * 1e3 / a.iters
    res = {"kernel": k, "lattice": "x".join(map(str, L)), "blocks": list(NB), "nrhs": nr,
           "fp32_links": 12 if links12 else 18,
           "us_per_launch": us, "us_per_rhs": us / nr, "plaquette": plaq}
    if nbytes:
        res["bytes_per_launch"] = nbytes
        res["GBps"] = nbytes / (us * 1e-6) / 1e9
        # 1872 flops per site (1320 hops + 504 clover + 48 axpy), per RHS
        sites = (V if k in ("dslash_s", "dslash_d") else V // 2) * nr
        res["GFLOPs"] = 1872 * sites / (us * 1e-6) / 1e9
    print(json.dumps(res), flush=True)
    lat.close()
    if lat is not base:
        base.close()


def solve_group(a):
    import torch

    import qws_b200
    from qws_b200 import autotune

    vols = [tuple(int(v) for v in s.split("x")) for s in a.volumes.split(",")]
    rng = np.random.default_rng(4)
    picks = [vols[int(rng.integers(len(vols)))] for _ in range(a.count)]
    st = torch.cuda.Stream()
    solves = []
    for i, L in enumerate(picks):
        hit = autotune.lookup(L, "hf", 1) or {}
        NB = tuple(hit.get("NB", autotune.REFERENCE_NB))
        lat = qws_b200.Lattice(L, NB, tbc=-1, kappa=a.kappa, stream=st)
        lat.set_hop_threads(hit.get("hop_threads", 128))
        lat.gen_gauge_device(1000 + 7919 * i + sum(L), 5, 0.36)
        lat.build_clover(a.csw)
        with torch.cuda.stream(st):
            b = lat.to_device(qws_b200.gen_source(L, 77))
            x = lat.empty("f64")
        solves.append(dict(lattice=lat, x=x, b=b, tol=1e-10, maxiter=100, tol_s=1e-6,
                           maxiter_s=50, nsap=hit.get("nsap", 4), nm=hit.get("nm", 2),
                           reliable=5))
    torch.cuda.synchronize()

    def solo():
        for s in solves:
            s["x"].zero_()
            s["lattice"].bicgstab_dd_mix2_hf(s["x"], s["b"], s["tol"], s["maxiter"], s["tol_s"],
                                             s["maxiter_s"], s["nsap"], s["nm"], s["reliable"])

    def group():
        for s in solves:
            s["x"].zero_()
        return qws_b200.group_solve(solves, stream=st)[1]

    def timed(fn):
        with torch.cuda.stream(st):
            for _ in range(a.warmup):
                fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            out = None
            for _ in range(a.iters):
                out = fn()
            e1.record(st)
            torch.cuda.synchronize()
        return e0.elapsed_time(e1) / a.iters, out

    t_solo, _ = timed(solo)
    x_solo = [s["x"].clone() for s in solves]
    t_group, gs = timed(group)
    same = all(torch.equal(s["x"], x0) for s, x0 in zip(solves, x_solo))
    res = {"kernel": "solve_group", "count": a.count,
           "volumes": {"x".join(map(str, L)): picks.count(L) for L in vols},
           "sites": int(sum(np.prod(L) for L in picks)),
           "solo_ms": t_solo, "group_ms": t_group,
           "solo_solves_per_s": a.count / (t_solo * 1e-3),
           "group_solves_per_s": a.count / (t_group * 1e-3),
           "group_bitwise_equal_solo": same, "group_stats": gs}
    print(json.dumps(res), flush=True)
    for s in solves:
        s["lattice"].close()


if __name__ == "__main__":
    main()
