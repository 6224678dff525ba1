"""Per-kernel microbenchmark of the DD operator kernels on one GPU.

    python -m qws_b200.microbench --lattice 32,32,32,64 --kernel jinv --iters 20

Builds seeded synthetic fields of the given lattice (SU(3) + 5 APE steps,
clover-leaf clover), then times `iters` launches of one operator with CUDA
events on the library's stream and prints one JSON line with the average
launch time and the algorithmic HBM bandwidth (bytes each launch must move:
spinors read and written once, links and clover once per site).

Kernels: jinv (one Richardson step on one colour), dslash_s / dslash_d (full
D in FP32 / FP64), block_s (block-interior D on one colour), face_s (face hops
of one colour), jinv_h / face_h (the FP16-storage Richardson step and face
hops through the single-operator entry points, conversions included), prec
(the whole SAP preconditioner prec_ddd_s_), prec_h (the FP16-storage SAP),
solve_hf (a whole precision-form solve to 1e-10; --new-kappa rebuilds the
clover term for another kappa before each, as a serving loop sees them).  --nrhs N runs the launch on a multi-RHS handle (N
right-hand sides per launch; spinor bytes count N times, links and clover
once).
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
    a = ap.parse_args()
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


if __name__ == "__main__":
    main()
