#!/usr/bin/env python3
"""Benchmark of the DD Wilson-clover solver on B200: solves per second.

One step = one complete solve D x = b to a 1e-10 relative residual with the
FP64-outer / FP32-SAP-inner DD BiCGStab (bicgstab_dd_mix_), x = 0 start,
on seeded synthetic fields (SU(3) links smoothed by 5 APE-style steps,
clover-leaf clover term, Gaussian complex FP64 source).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
    python bench.py --impl reference ...     # the reference's CPU solver

Prints one JSON line (rank 0).  Multi-GPU runs (torchrun) are independent
replicas (the single-GPU path holds the whole lattice; no data exchange):
value = total solves of all ranks / max over ranks of the timed device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # the plain method at GPU scale, single RHS (roofline figures):
    # 32^3x64, 5 APE steps, csw 1.7, kappa 0.1365, outer 1e-10, inner 1e-6 / 50
    "plain_32c64": dict(L=(32, 32, 32, 64), NB=(2, 1, 1, 1), csw=1.7, kappa=0.1365, tbc=-1,
                        seed=11, n_smear=5, alpha=0.36, tol=1e-10, maxiter=200, tol_s=1e-6,
                        maxiter_s=50, nsap=4, nm=2, src="gauss"),
    # small variant of the same for quick checks
    "plain_16c32": dict(L=(16, 16, 16, 32), NB=(2, 1, 1, 1), csw=1.7, kappa=0.1365, tbc=-1,
                        seed=11, n_smear=5, alpha=0.36, tol=1e-10, maxiter=200, tol_s=1e-6,
                        maxiter_s=50, nsap=4, nm=2, src="gauss"),
}
DEFAULT_WORKLOAD = "plain_32c64"
METRIC = "solves/s @1e-10 resid: mixed-prec vs plain FP64 on B200; Dslash GB/s; p99 ms"
METRIC_DETAIL = ("value: plain DD BiCGStab solves/s (FP64 outer / FP32 SAP inner, 1e-10 true "
                 "relative residual); precision_form: the mixed-precision solver on the same "
                 "workload; roofline: the dominant stencil kernel's HBM GB/s")
_T0 = time.time()


def progress(msg):
    """Phase markers on stderr (the JSON line alone goes to stdout)."""
    print(f"[bench {time.time() - _T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region.
    nvidia-smi runs on a pseudo-terminal (so it writes each sample as it
    takes it instead of buffering them) with its own timestamp per sample;
    the samples between mark() and stop() are the timed region's."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.t_mark = float("-inf")

    def start(self):
        try:
            import pty

            master, slave = pty.openpty()
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=slave, stderr=subprocess.DEVNULL, close_fds=True)
            os.close(slave)
            self.fd = master
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        buf = b""
        while True:
            try:
                chunk = os.read(self.fd, 4096)
            except OSError:  # the terminal closes when nvidia-smi exits
                break
            if not chunk:
                break
            buf += chunk
            *lines, buf = buf.split(b"\n")
            for line in lines:
                parts = [p.strip() for p in line.decode(errors="replace").split(",")]
                if len(parts) >= 10:
                    self.rows.append((self._stamp(parts[0]), parts[1:]))

    @staticmethod
    def _stamp(text):
        import datetime

        for fmt in ("%Y/%m/%d %H:%M:%S.%f", "%Y/%m/%d %H:%M:%S"):
            try:
                return datetime.datetime.strptime(text, fmt).timestamp()
            except ValueError:
                pass
        return time.time()

    def mark(self):
        """Start of the timed region: the sampler runs from before the
        warm-up (nvidia-smi takes a moment to emit its first sample)."""
        self.t_mark = time.time()

    def stop(self):
        t_end = time.time()
        if self.proc:
            time.sleep(0.3)  # the sample in flight
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)
            try:
                os.close(self.fd)
            except OSError:
                pass
        sm = []
        reasons = set()
        smax = None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, r in self.rows:
            if not self.t_mark <= t <= t_end:
                continue
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_fields(w):
    import qws_b200

    t0 = time.time()
    U, plaq = qws_b200.gen_gauge(w["L"], w["seed"], w["n_smear"], w["alpha"])
    C = qws_b200.gen_clover(U, w["L"], w["csw"], w["kappa"])
    b = qws_b200.gen_source(w["L"], w["seed"] + 1, w["src"])
    return U, C, b, plaq, time.time() - t0


def run_reference(w, warmup, steps, solution_out=None, threads=None):
    """Complete solves of the reference's own CPU solver on this host
    (oracle/refbench.py in a subprocess, all host threads): `warmup` untimed
    then `steps` timed bicgstab_dd_mix_ calls on the workload's fields, which
    the oracle generates bit-equal to the product's."""
    spec = {k: (list(v) if isinstance(v, tuple) else v) for k, v in w.items()}
    spec.update(warmup=int(warmup), steps=int(steps))
    if solution_out:
        spec["solution_out"] = str(solution_out)
    env = dict(os.environ)
    n = threads or len(os.sched_getaffinity(0))
    env["OMP_NUM_THREADS"] = str(n)
    env.setdefault("OMP_PROC_BIND", "close")
    env["CUDA_VISIBLE_DEVICES"] = ""
    res = subprocess.run([sys.executable, str(ROOT / "oracle" / "refbench.py"), json.dumps(spec)],
                         capture_output=True, text=True, env=env, timeout=3600)
    if res.returncode != 0:
        raise RuntimeError("reference run failed: " + res.stderr[-2000:])
    return json.loads(res.stdout.strip().splitlines()[-1])


def field_digests(U, C, b):
    """SHA-256 of the arrays a solve consumes (compared with the reference arm's)."""
    import hashlib

    h = lambda a: hashlib.sha256(memoryview(np.ascontiguousarray(a)).cast("B")).hexdigest()
    return {"gauge": h(U), "clover": h(C), "source": h(b)}


def config_of(w, name):
    """The `config` object of both arms' lines: the workload, nothing else."""
    return {"workload": name, "lattice": "x".join(map(str, w["L"])),
            "block_grid": list(w["NB"]), "kappa": w["kappa"], "csw": w["csw"],
            "tol": w["tol"], "tol_s": w["tol_s"], "maxiter_s": w["maxiter_s"],
            "nsap": w["nsap"], "nm": w["nm"],
            "l2": "inputs larger than L2 (one FP64 spinor = %.0f MB)"
                  % (int(np.prod(w["L"])) * 24 * 8 / 1e6)}


def dist_setup(n_gpus):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def allreduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def bench_ours(args, w, name):
    import torch

    import qws_b200

    world, rank, local = dist_setup(args.gpus)
    progress(f"fields for {name}")
    U, C, b, plaq, t_gen = make_fields(w)
    digests = field_digests(U, C, b) if rank == 0 and not args.no_cpu_baseline else None
    stream = torch.cuda.Stream()
    lat = qws_b200.Lattice(w["L"], w["NB"], tbc=w["tbc"], kappa=w["kappa"], stream=stream)
    lat.load_fields(U, C)
    with torch.cuda.stream(stream):
        bd = lat.to_device(b)
        xd = lat.empty("f64")
    V = lat.V

    def solve():
        xd.zero_()
        return lat.bicgstab_dd_mix(xd, bd, w["tol"], w["maxiter"], w["tol_s"], w["maxiter_s"],
                                   w["nsap"], w["nm"])

    clocks = ClockSampler(local)
    clocks.start()
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            st = solve()
        torch.cuda.synchronize()
        true_rel = lat.true_residual(xd, bd)
        c0 = lat.counters()

        progress("warm-up done; timed plain solves")
        # ---- device-resident timed region (production configuration: the
        #      SAP launch sequences replayed from CUDA graphs) ------------------
        barrier(world)
        torch.cuda.synchronize()
        clocks.mark()
        n_launch0 = qws_b200.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        stats = []
        for _ in range(args.steps):
            stats.append(solve())
        e1.record(stream)
        torch.cuda.synchronize()
        n_launches = qws_b200.launch_count() - n_launch0
        clk = clocks.stop()
        barrier(world)
        ms = e0.elapsed_time(e1)
        c1 = lat.counters()
        ms_max = allreduce_max(ms, world)

        # ---- per-kernel CUDA-event timing of the same solves (events between
        #      launches, so graphs are off for this pass) --------------------
        lat.kernel_timing(True)
        for _ in range(args.steps):
            solve()
        torch.cuda.synchronize()
        kstats = lat.kernel_stats()
        lat.kernel_timing(False)
        # the plain solver's solution, checked against the reference's below
        x_gpu = lat.to_host(xd) if rank == 0 and world == 1 and not args.no_cpu_baseline else None

        progress("end-to-end solves")
        # ---- end to end through the public API with host buffers --------------
        pinned = torch.from_numpy(b).pin_memory()
        host_b = pinned.numpy()
        host_x = torch.empty_like(pinned).pin_memory().numpy()
        xh = lat.empty("f64")
        bh = lat.empty("f64")
        torch.cuda.synchronize()
        barrier(world)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            lat.to_device(host_b, out=bh)
            xh.zero_()
            lat.bicgstab_dd_mix(xh, bh, w["tol"], w["maxiter"], w["tol_s"], w["maxiter_s"],
                                w["nsap"], w["nm"])
            lat.to_host(xh, out=host_x)
        f1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = allreduce_max(f0.elapsed_time(f1), world)

        # ---- the precision form on the same workload: FP16-storage SAP with
        #      per-site scales, flexible FP32 inner, FP64 outer with reliable
        #      restarts from the true residual --------------------------------
        def solve_hf():
            xd.zero_()
            return lat.bicgstab_dd_mix2_hf(xd, bd, w["tol"], w["maxiter"], w["tol_s"],
                                           w["maxiter_s"], w["nsap"], w["nm"], reliable=5)

        for _ in range(max(1, args.warmup)):
            solve_hf()
        torch.cuda.synchronize()
        barrier(world)
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record(stream)
        hstats = [solve_hf() for _ in range(args.steps)]
        h1.record(stream)
        torch.cuda.synchronize()
        hf_ref_ms = allreduce_max(h0.elapsed_time(h1), world)
        hf_ref_true = lat.true_residual(xd, bd)
        hf_ref_iters = (sum(s["outer_iters"] for s in hstats) / len(hstats),
                        sum(s["inner_iters"] for s in hstats) / len(hstats))
    e2e_true = lat.true_residual(xh, bh)
    del xh, bh
    progress("end-to-end through the drop-in entry point")
    try:
        e2e_ref_api = e2e_dropin(w, U, C, b, args.steps, lat)
    except Exception as e:  # noqa: BLE001 -- reported in the line
        e2e_ref_api = {"error": f"{type(e).__name__}: {str(e)[-300:]}"}

    # sub-results: a failure is reported in the line, it does not lose the line
    def sub(fn, *a):
        try:
            return fn(*a)
        except Exception as e:  # noqa: BLE001
            return {"error": f"{type(e).__name__}: {str(e)[-400:]}"}

    # ---- the precision form in its tuned configuration (SAP block grid,
    #      sweep counts, CTA size chosen by qws_b200.autotune for this
    #      lattice), on the same fields and source -----------------------------
    progress("autotune")
    tuned = sub(tuned_config, args, w["L"], rank)
    tl = lat
    if "NB" in tuned and tuple(tuned["NB"]) != tuple(w["NB"]):
        tl = qws_b200.Lattice(w["L"], tuned["NB"], tbc=w["tbc"], kappa=w["kappa"], stream=stream)
        tl.load_fields(U, C)
    # the plain solver in the autotuner's configuration for it, on the same
    # fields: the precision form's gain at equal footing (both tuned)
    progress("plain solver, tuned")
    plain_tuned = sub(bench_plain_tuned, args, w, U, C, b, stream, world)
    del U, C
    cfg = {k: tuned.get(k, w.get(k, d)) for k, d in
           (("nsap", 4), ("nm", 2), ("hop_threads", 128))}
    tl.set_hop_threads(cfg["hop_threads"])
    with torch.cuda.stream(stream):
        bt = tl.to_device(b) if tl is not lat else bd
        xt = tl.empty("f64")

        def solve_tuned():
            xt.zero_()
            return tl.bicgstab_dd_mix2_hf(xt, bt, w["tol"], w["maxiter"], w["tol_s"],
                                          w["maxiter_s"], cfg["nsap"], cfg["nm"], reliable=5)

        progress("precision form, tuned")
        for _ in range(max(1, args.warmup)):
            solve_tuned()
        torch.cuda.synchronize()
        barrier(world)
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record(stream)
        hstats = [solve_tuned() for _ in range(args.steps)]
        h1.record(stream)
        torch.cuda.synchronize()
        hf_ms = allreduce_max(h0.elapsed_time(h1), world)
        hf_true = tl.true_residual(xt, bt)
        # per-kernel device times of the same solves (graphs off in this pass)
        tl.kernel_timing(True)
        for _ in range(args.steps):
            solve_tuned()
        torch.cuda.synchronize()
        hf_kstats = tl.kernel_stats()
        tl.kernel_timing(False)

    progress("batched")
    batched = sub(bench_batched, args, w, tl, stream, world, cfg) if args.batch > 1 else None
    serving = None
    precision_48 = None
    uneven = None
    if world == 1 and (args.serve_rate > 0 or args.config3 or args.uneven_workers > 0):
        lat.close()  # the later parts get the HBM to themselves
        if tl is not lat:
            tl.close()
        del xd, bd, xt, bt
        torch.cuda.empty_cache()
    if args.serve_rate > 0 and world == 1:
        progress("serving window")
        serving = sub(bench_serving, args)
    if args.uneven_workers > 0 and world == 1:
        progress("48 solves of uneven volume")
        uneven = sub(bench_uneven, args)
    if args.config3 and world == 1:
        progress("48^3x96 precision comparison")
        precision_48 = sub(bench_precision_48, args, world)
    progress("done with GPU parts")

    per_solve = {k: (c1[k] - c0[k]) / args.steps for k in c1}
    inner_iters = sum(s["inner_iters"] for s in stats) / len(stats)
    outer_iters = sum(s["outer_iters"] for s in stats) / len(stats)
    counts = {"inner_iters": int(round(inner_iters)),
              "n_approx": int(round(per_solve["prec_s"])),
              "n_ddd_d": int(round(per_solve["ddd_d"])) + 1}

    peak, peak_kind = measured_peaks()
    dom = max(kstats.items(), key=lambda kv: kv[1][1]) if kstats else None
    roofline = None
    if dom:
        kname, (nl, kms, kbytes) = dom
        achieved = kbytes / (kms * 1e-3) / 1e9
        traffic = None
        tp = ROOT / "profiles" / "traffic.json"
        if tp.exists():
            t = json.loads(tp.read_text())
            ent = t.get(name, {}).get(kname)
            if ent:
                traffic = ent["bytes_per_launch"]
        roofline = {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1),
                    "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                    "peak_source": peak_kind, "traffic": traffic,
                    "bytes_per_launch": kbytes / nl, "avg_launch_us": kms / nl * 1e3,
                    "launches": nl,
                    "share_of_kernel_time": round(kms / sum(v[1] for v in kstats.values()), 4)}
    kernels = kernel_table(kstats, peak, w["L"], w["NB"])
    if roofline and "GFLOPs" in kernels.get(roofline["kernel"], {}):
        roofline["gflops"] = kernels[roofline["kernel"]]["GFLOPs"]
        roofline["flop_convention"] = "1872 per site (1320 hops + 504 clover + 48 axpy)"

    line = {
        "metric": METRIC,
        "metric_detail": METRIC_DETAIL,
        "value": world * args.steps / (ms_max * 1e-3),
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 outer / f32 inner",
        "data": "synthetic: seeded SU(3) links + 5 APE steps (plaquette %.4f), clover-leaf "
                "clover, Gaussian source" % plaq,
        "config": dict(config_of(w, name), parallelism=f"replicas x{world}"),
        "solve": {"outer_iters": outer_iters, "inner_iters": inner_iters,
                  "true_rel_resid": true_rel, "recursive_rel_resid": stats[-1]["rel_resid_recursive"]},
        "e2e": (dict(e2e_ref_api, value=world * e2e_ref_api["value"])
                if "value" in e2e_ref_api else
                {"value": world * args.steps / (e2e_ms * 1e-3), "unit": "solves/s",
                 "h2d_bytes_per_step": int(b.nbytes), "d2h_bytes_per_step": int(b.nbytes),
                 "fallback_from_dropin": e2e_ref_api}),
        "e2e_native_api": {"value": world * args.steps / (e2e_ms * 1e-3), "unit": "solves/s",
                           "h2d_bytes_per_step": int(b.nbytes), "d2h_bytes_per_step": int(b.nbytes),
                           "true_rel_resid": e2e_true,
                           "path": "qws_b200.Lattice host arrays (pinned) -> qwsg_spinor_to_device_d "
                                   "-> qwsg_bicgstab_dd_mix -> qwsg_spinor_to_host_d"},
        "precision_form": {
            "value": world * args.steps / (hf_ms * 1e-3), "unit": "solves/s",
            "ms_per_step": hf_ms / args.steps,
            "speedup_vs_plain": ms_max / hf_ms,
            "speedup_vs_plain_tuned": (plain_tuned["value"] and
                                       (args.steps / (hf_ms * 1e-3)) / plain_tuned["value"])
                                      if "value" in plain_tuned else None,
            "plain_tuned": plain_tuned,
            "true_rel_resid": hf_true,
            "outer_iters": sum(s["outer_iters"] for s in hstats) / len(hstats),
            "inner_iters": sum(s["inner_iters"] for s in hstats) / len(hstats),
            "config": {"block_grid": list(tl.NB), **cfg},
            "tuning": tuned,
            "kernels": kernel_table(hf_kstats, peak, w["L"], tl.NB),
            "at_reference_partition": {
                "block_grid": list(w["NB"]), "nsap": w["nsap"], "nm": w["nm"],
                "value": world * args.steps / (hf_ref_ms * 1e-3),
                "speedup_vs_plain": ms_max / hf_ref_ms, "true_rel_resid": hf_ref_true,
                "outer_iters": hf_ref_iters[0], "inner_iters": hf_ref_iters[1]},
            "method": "bicgstab_dd_mix2_hf: FP64 outer (reliable restarts) / flexible FP32 "
                      "inner / SAP in FP16 storage with per-site FP32 scales (nsap-1 sweeps)"},
        "batched": batched,
        "uneven_volumes": uneven,
        "serving": serving,
        "precision_48c96": precision_48,
        "gpu_launches": int(n_launches),
        "roofline": roofline,
        "kernels": kernels,
        "clocks": clk,
        "counts_per_solve": counts,
        "field_gen_s": round(t_gen, 2),
    }
    if batched and "value" in batched:
        batched["speedup_vs_plain"] = batched["value"] / line["value"]
        batched["speedup_vs_precision_single"] = batched["value"] / line["precision_form"]["value"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        progress("cpu baseline: complete reference solves")
        line["cpu_baseline"] = sub(cpu_baseline, w, x_gpu, digests, line["solve"])
    del x_gpu
    lat.close()
    if tl is not lat:
        tl.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


# flops per handled site, the convention of the Wilson-clover D: 1320 for
# the eight hops (165 each: projection, SU(3) x half-spinor, reconstruction),
# 504 for the packed-Hermitian clover product, 48 for the axpy epilogue;
# a block or Richardson application counts as a whole site, a face site as
# its 1.1 face hops (average at the reference partition) + clover + axpy
FLOPS_PER_SITE = {"dslash_full": 1872, "dslash_block": 1872, "jinv_step": 1872,
                  "sap_update": 1872 + 48, "dslash_face": round(1.1 * 165) + 504 + 48}


def sites_per_launch(kind, L, NB, nr):
    """sites one launch of kernel kind handles (times the RHS count)"""
    V = int(np.prod(L))
    if kind.startswith("dslash_full"):
        return V * nr
    if kind.startswith("dslash_face"):
        B = [L[m] // NB[m] for m in range(4)]
        inner = int(np.prod([b - 2 if b > 2 else 0 for b in B]))
        return int(np.prod(NB)) // 2 * (int(np.prod(B)) - inner) * nr
    return V // 2 * nr


def kernel_table(kstats, peak, L=None, NB=None, nr=1):
    """{kernel: launches, device ms, share of the solve's kernel time,
    algorithmic GB/s and its fraction of the measured HBM peak, and GFLOP/s
    in the 1872-flop-per-site convention (FLOPS_PER_SITE)}"""
    total = sum(v[1] for v in kstats.values()) or 1.0
    out = {}
    for k, (n, ms, by) in sorted(kstats.items(), key=lambda kv: -kv[1][1]):
        gbs = by / (ms * 1e-3) / 1e9 if ms else None
        out[k] = {"launches": n, "ms": round(ms, 3), "share": round(ms / total, 4),
                  "GBps": round(gbs, 1) if gbs else None,
                  "frac_of_peak": round(gbs / peak, 4) if gbs else None}
        base = k.rsplit("_", 1)[0]
        if L is not None and base in FLOPS_PER_SITE and ms:
            fl = FLOPS_PER_SITE[base] * sites_per_launch(k, L, NB, nr) * n
            out[k]["GFLOPs"] = round(fl / (ms * 1e-3) / 1e9, 1)
    return out


def e2e_dropin(w, U, C, b, steps, lat):
    """End to end through the reference-facing C ABI: QWS's own
    `bicgstab_dd_mix_(x, b, ...)` on QWS-layout host arrays (pinned), as
    main.cc or BQCD call it after qws_init_ and loading glud/glus/clvd/clvs.
    Each call uploads b and the initial guess x (zero), solves and writes x
    back, so both transfers are inside the timed region.  Timed with the
    host clock: the call is synchronous.  The returned x's true residual
    is checked with the native handle `lat` (same fields)."""
    import ctypes

    import torch

    import qws_b200
    from qws_b200 import layouts

    os.environ["QWSG_NO_EXIT"] = "1"  # a failing call reports instead of ending the bench
    lib = qws_b200.load_library()
    L = tuple(w["L"])
    vd = 8
    vs = 16 if (L[0] // 2) % 16 == 0 else 8
    I = lambda v: ctypes.byref(ctypes.c_int(v))
    D = lambda v: ctypes.byref(ctypes.c_double(v))
    if lib.qwsg_set_host_vlen(vd, vs) != 0:
        raise RuntimeError("qwsg_set_host_vlen failed")
    npe = (ctypes.c_int * 4)(1, 1, 1, 1)
    fbc = (ctypes.c_int * 4)(1, 1, 1, int(w["tbc"]))
    blk = (ctypes.c_int * 4)(1, 1, 1, 1)
    lib.qws_init_(I(L[0]), I(L[1]), I(L[2]), I(L[3]), npe, fbc, I(0), I(1), blk)
    try:
        for name, val in (("kappa", w["kappa"]), ("mkappa", -w["kappa"]),
                          ("kappa2", w["kappa"] ** 2)):
            ctypes.c_double.in_dll(lib, name).value = val
        for name, arr in (("glud", layouts.nat_to_qws_gauge(U, L, vd)),
                          ("glus", layouts.nat_to_qws_gauge(U, L, vs).astype(np.float32)),
                          ("clvd", layouts.nat_to_qws_clover(C, L, vd)),
                          ("clvs", layouts.nat_to_qws_clover(C, L, vs).astype(np.float32))):
            ctypes.memmove(ctypes.c_void_p.in_dll(lib, name).value, arr.ctypes.data, arr.nbytes)
            del arr
        lib.qwsg_mark_fields_dirty()
        n = 24 * int(np.prod(L))

        def pinned():
            return torch.zeros(n, dtype=torch.float64, pin_memory=True).numpy()

        bq = pinned()
        layouts.nat_to_qws_spinor(b, L, vd, out=bq)
        xs = [pinned() for _ in range(steps + 1)]
        it = ctypes.c_int()

        def call(x):
            it.value = -1
            lib.bicgstab_dd_mix_(ctypes.c_void_p(x.ctypes.data), ctypes.c_void_p(bq.ctypes.data),
                                 D(w["tol"]), ctypes.byref(it), I(w["maxiter"]), D(w["tol_s"]),
                                 I(w["maxiter_s"]), I(w["nsap"]), I(w["nm"]))
            if it.value < 0:
                err = lib.qwsg_last_error()
                raise RuntimeError("bicgstab_dd_mix_ failed: " + (err.decode() if err else "?"))

        call(xs[0])  # warm-up: field upload, graph capture
        t0 = time.perf_counter()
        for k in range(steps):
            call(xs[k + 1])
        dt = time.perf_counter() - t0
        with torch.cuda.stream(torch.cuda.current_stream()):
            xn = layouts.qws_to_nat_spinor(xs[steps], L, vd)
            true = lat.true_residual(lat.to_device(xn), lat.to_device(b))
    finally:
        lib.qws_finalize_()
    return {"value": steps / dt, "unit": "solves/s", "h2d_bytes_per_step": 2 * n * 8,
            "d2h_bytes_per_step": n * 8, "true_rel_resid": true, "outer_iters": it.value,
            "path": "drop-in bicgstab_dd_mix_(x, b, ...) on QWS-layout (scd_t, VLEND=%d) pinned "
                    "host arrays after qws_init_ and glud/glus/clvd/clvs; b and the zero initial "
                    "guess x uploaded, x downloaded, in every call; host clock" % vd}


def tuned_config(args, L, rank):
    """The autotuner's choice for the precision form on lattice L (the
    cached entry for this GPU, else a tuning run; --retune forces one)."""
    from qws_b200 import autotune

    if args.tune == "off":
        return {"source": "off"}
    # every rank reads the cache; only rank 0 writes a new entry
    entry, _ = autotune.autotune(L, "hf", 1, retune=args.tune == "retune", log=progress,
                                 write=rank == 0)
    return entry


def bench_batched(args, w, lat, stream, world, cfg):
    """Multi-RHS form on the same gauge field: 12 point sources (one per spin x
    colour at the origin) + 4 Z2-noise sources solved together by the
    precision-form solver on one multi-RHS handle (every operator launch
    serves all of them); FP64 outer to the workload's tolerance."""
    import torch

    import qws_b200

    nr = args.batch
    L = w["L"]
    src = [qws_b200.gen_source(L, 0, "point", k) for k in range(min(nr, 12))]
    src += [qws_b200.gen_source(L, w["seed"] + 100 + k, "z2") for k in range(nr - len(src))]
    S = np.stack(src)
    del src
    B = lat.batch(nr, stream=stream)
    with torch.cuda.stream(stream):
        bb = B.to_device(S)
        del S
        xb = B.empty("f64")

        def solve():
            xb.zero_()
            return B.bicgstab_dd_mix2_hf(xb, bb, w["tol"], w["maxiter"], w["tol_s"],
                                         w["maxiter_s"], cfg["nsap"], cfg["nm"], reliable=5)

        for _ in range(max(1, min(args.warmup, 2))):
            solve()
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            st = solve()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = allreduce_max(e0.elapsed_time(e1), world)
        per, _ = B.batch_stats()
        truer = B.true_residual(xb, bb)
    B.close()
    del xb, bb
    torch.cuda.empty_cache()
    return {"value": world * args.steps * nr / (ms * 1e-3), "unit": "solves/s",
            "nrhs": nr, "ms_per_batch": ms / args.steps,
            "max_true_rel_resid": max(truer), "outer_iters": [p["outer_iters"] for p in per],
            "inner_iters": st["inner_iters"],
            "sources": f"{min(nr, 12)} point (spin x colour at the origin) + "
                       f"{max(0, nr - 12)} Z2 noise",
            "config": {"block_grid": list(lat.NB), **cfg},
            "method": "bicgstab_dd_mix2_hf on a multi-RHS handle: one launch per operator for "
                      "all RHS, per-RHS scalars and convergence"}


def rep_times(fn, reps, stream):
    """Device time (ms) of each of `reps` calls of fn after one untimed call,
    CUDA events on `stream`; returns (times, the last call's result)."""
    import torch

    fn()
    torch.cuda.synchronize()
    out, st = [], None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return out, st


def spread(ms, per=1):
    """solves/s from the median of repeated timings, with min/median/max (ms)"""
    med = statistics.median(ms)
    return {"solves_per_s": per * 1e3 / med, "median_ms": round(med, 2),
            "min_ms": round(min(ms), 2), "max_ms": round(max(ms), 2), "reps": len(ms)}


def reference_samples_48():
    """The reference's own 48^3x96 solutions on a fixed sample of sites
    (tests/golden/make_ref_solutions.py), if the fixture is present."""
    p = ROOT / "tests" / "golden" / "ref_solutions_48c96.npz"
    if not p.exists():
        return None
    z = np.load(p)
    meta = json.loads(str(z["meta"]))
    return {"sites": z["sites"], "meta": meta,
            "x": {float(k): z[f"x_{k}"] for k in meta}}


def bench_precision_48(args, world):
    """48^3x96 (the precision-form workload), seeded SU(3) + 5 APE steps
    (generated on the GPU), csw 1.7, kappa 0.1365 and 0.1355, Gaussian
    source, 1e-10.  Per kappa, each timed over `reps` solves (median, min,
    max):
      plain      the plain solver (FP64 outer / FP32 SAP inner) at the
                 reference's one-rank partition, and in the autotuner's
                 configuration for the plain solver;
      precision  the precision form (FP16-storage SAP, FP64 outer with
                 reliable restarts) at the reference partition, in its own
                 tuned configuration on one RHS, and on a --batch48-RHS handle;
    and the speed-ups at an equal partition and with both solvers tuned.
    Every solution has its true residual and its error against a 1e-13 solve
    of the same system, and the reference's own solution on a sample of
    sites where tests/golden/ref_solutions_48c96.npz holds it.  The block
    grids run one after the other (their work buffers do not fit in HBM
    together); the fields are generated from the same seeds on each."""
    import torch

    import qws_b200
    from qws_b200 import autotune

    L, NB = (48, 48, 48, 96), (2, 1, 1, 1)
    kappas = (0.1365, 0.1355)
    reps = max(5, int(args.reps48))
    stream = torch.cuda.Stream()
    b = qws_b200.gen_source(L, 12, "gauss")
    nrb = max(1, int(args.batch48))
    bn = np.stack([b] + [qws_b200.gen_source(L, 12 + k, "gauss") for k in range(1, nrb)])
    tuned = tuned_config(args, L, 0)
    cfg = {k: tuned.get(k, d) for k, d in (("nsap", 4), ("nm", 2), ("hop_threads", 128))}
    NBt = tuple(tuned.get("NB", NB))
    ptuned = autotune.lookup(L, "plain", 1) or {}
    pcfg = {k: ptuned.get(k, d) for k, d in (("nsap", 4), ("nm", 2), ("hop_threads", 128))}
    NBp = tuple(ptuned.get("NB", NB))
    ref = reference_samples_48()
    out = {"lattice": "48x48x48x96", "tol": 1e-10, "reps": reps,
           "reference_partition": list(NB),
           "precision_tuned": {"block_grid": list(NBt), **cfg, "tuning": tuned},
           "plain_tuned": {"block_grid": list(NBp), **pcfg,
                           "tuning": ptuned or "no cached plain tuning: reference partition"},
           "fields": "gauge generated and clover built on the GPU (equal to the host "
                     "generator's to rounding); the reference solved the host generator's",
           "per_kappa": []}
    per = {k: {"kappa": k} for k in kappas}
    xref = {}

    def errors(lat, x, kappa):
        xh = lat.to_host(x)
        e = {"rel_error_vs_fp64_solve": float(np.linalg.norm(xh - xref[kappa]) /
                                                np.linalg.norm(xref[kappa]))}
        if ref is not None and kappa in ref["x"]:
            xs, rs = xh[ref["sites"]], ref["x"][kappa]
            e["rel_error_vs_reference_sample"] = float(np.linalg.norm(xs - rs) / np.linalg.norm(rs))
        return e

    def plain_run(lat, nsap, nm, kappa):
        with torch.cuda.stream(stream):
            bd, x = lat.to_device(b), lat.empty("f64")

            def solve():
                x.zero_()
                return lat.bicgstab_dd_mix(x, bd, 1e-10, 200, 1e-6, 50, nsap, nm)

            ms, st = rep_times(solve, reps, stream)
            res = dict(spread(ms), true_rel_resid=lat.true_residual(x, bd),
                       outer_iters=st["outer_iters"], inner_iters=st["inner_iters"],
                       **errors(lat, x, kappa))
            del x, bd
            torch.cuda.empty_cache()
        return res

    def precision_run(lat, nsap, nm, kappa):
        with torch.cuda.stream(stream):
            bd, x = lat.to_device(b), lat.empty("f64")

            def solve():
                x.zero_()
                return lat.bicgstab_dd_mix2_hf(x, bd, 1e-10, 200, 1e-6, 50, nsap, nm, reliable=5)

            ms, st = rep_times(solve, reps, stream)
            res = dict(spread(ms), true_rel_resid=lat.true_residual(x, bd),
                       outer_iters=st["outer_iters"], inner_iters=st["inner_iters"],
                       **errors(lat, x, kappa))
            del x, bd
            torch.cuda.empty_cache()
        return res

    def batched_run(lat, nsap, nm, kappa):
        B = lat.batch(nrb, stream=stream)
        try:
            with torch.cuda.stream(stream):
                bb, xb = B.to_device(bn[:nrb]), B.empty("f64")

                def solve():
                    xb.zero_()
                    return B.bicgstab_dd_mix2_hf(xb, bb, 1e-10, 200, 1e-6, 50, nsap, nm,
                                                 reliable=5)

                ms, _ = rep_times(solve, reps, stream)
                xh = B.to_host(xb)[0]
                res = dict(spread(ms, nrb), nrhs=nrb,
                           max_true_rel_resid=max(B.true_residual(xb, bb)),
                           rel_error_vs_fp64_solve=float(np.linalg.norm(xh - xref[kappa]) /
                                                         np.linalg.norm(xref[kappa])))
                del xb, bb
        finally:
            B.close()
            torch.cuda.empty_cache()
        return res

    def lattice(NBx, threads):
        lat = qws_b200.Lattice(L, NBx, tbc=-1, kappa=kappas[0], stream=stream)
        plaq = lat.gen_gauge_device(11, 5, 0.36)
        lat.set_hop_threads(threads)
        return lat, plaq

    # ---- reference partition: the 1e-13 solution, plain, precision form -----
    lat, out["plaquette"] = lattice(NB, 128)
    try:
        for kappa in kappas:
            lat.set_kappa(kappa)
            lat.build_clover(1.7)
            with torch.cuda.stream(stream):
                bd, x = lat.to_device(b), lat.empty("f64")
                lat.bicgstab_dd_mix(x, bd, 1e-13, 200, 1e-6, 50)
                xref[kappa] = lat.to_host(x)
                del x, bd
            per[kappa]["plain_reference_partition"] = plain_run(lat, 4, 2, kappa)
            per[kappa]["precision_reference_partition"] = precision_run(lat, 4, 2, kappa)
    finally:
        lat.close()
        torch.cuda.empty_cache()
    # ---- the plain solver in its tuned configuration ------------------------
    if (NBp, pcfg["nsap"], pcfg["nm"], pcfg["hop_threads"]) != (NB, 4, 2, 128):
        lat, _ = lattice(NBp, pcfg["hop_threads"])
        try:
            for kappa in kappas:
                lat.set_kappa(kappa)
                lat.build_clover(1.7)
                per[kappa]["plain_tuned"] = plain_run(lat, pcfg["nsap"], pcfg["nm"], kappa)
        finally:
            lat.close()
            torch.cuda.empty_cache()
    else:
        for kappa in kappas:
            per[kappa]["plain_tuned"] = per[kappa]["plain_reference_partition"]
    # ---- the precision form in its tuned configuration ----------------------
    lat, _ = lattice(NBt, cfg["hop_threads"])
    try:
        # the multi-RHS runs first: the lattice's own single-RHS work buffers
        # (kept until the lattice closes) and an nr-RHS handle's do not fit
        # in HBM together at 48^3x96
        for kappa in kappas:
            lat.set_kappa(kappa)
            lat.build_clover(1.7)
            per[kappa]["precision_tuned_batched"] = batched_run(lat, cfg["nsap"], cfg["nm"], kappa)
        for kappa in kappas:
            lat.set_kappa(kappa)
            lat.build_clover(1.7)
            per[kappa]["precision_tuned"] = precision_run(lat, cfg["nsap"], cfg["nm"], kappa)
    finally:
        lat.close()
        torch.cuda.empty_cache()
    for kappa in kappas:
        p = per[kappa]
        sps = lambda k: p[k]["solves_per_s"]
        p["speedups"] = {
            "precision_vs_plain_same_partition":
                sps("precision_reference_partition") / sps("plain_reference_partition"),
            "precision_tuned_vs_plain_tuned": sps("precision_tuned") / sps("plain_tuned"),
            "batched_tuned_vs_plain_tuned": sps("precision_tuned_batched") / sps("plain_tuned"),
            "precision_tuned_vs_plain_reference_partition":
                sps("precision_tuned") / sps("plain_reference_partition"),
        }
        if ref is not None and f"{kappa:.4f}" in ref["meta"]:
            m = ref["meta"][f"{kappa:.4f}"]
            p["reference_solve"] = {"outer_iters": m["outer_iters"],
                                    "inner_iters": m["inner_iters_per_solve"],
                                    "true_rel_resid": m["true_rel_resid"],
                                    "variant": m["variant"], "sample_sites": len(ref["sites"])}
    out["per_kappa"] = [per[k] for k in kappas]
    return out


def _uneven_pass(args, picks, vols, modes):
    """Each mode: a service solving the requests for `picks` (one seeded
    gauge field each) submitted at once; a cold pass makes the fields
    resident, the timed warm pass solves the same requests again."""
    import qws_b200
    from qws_b200 import serve

    src = {L: qws_b200.gen_source(L, 77, "gauss") for L in vols}
    out = {"solves": len(picks), "volumes": {"x".join(map(str, L)): picks.count(L) for L in vols}}
    for name, workers, group, gmax in modes:
        svc = serve.Service(serve.seeded_gauge(), budget_bytes=150e9, workers=workers,
                            max_batch=1, group=group, group_max_sites=gmax)
        try:
            def run():
                t0 = time.monotonic()
                reqs = svc.submit_all([serve.Request(L=L, gauge=i, kappa=0.1365, csw=1.7,
                                                     tol=1e-10, source=src[L])
                                       for i, L in enumerate(picks)])
                for q in reqs:
                    q.wait(600)
                t1 = time.monotonic()
                st = serve.summarize(reqs, t0, t1)
                return st, t1 - t0, reqs

            cold, cold_s, _ = run()
            rounds0, launches0 = svc.group_rounds, list(svc.group_launches)
            phase0, host0 = list(svc.group_phase_s), dict(svc.group_host_s)
            warm, warm_s, reqs = run()
        finally:
            svc.close()
        out[name] = {
            "solves_per_s": warm["solves_per_s"], "wall_s": warm_s, "cold_wall_s": cold_s,
            "p50_ms": warm["p50_ms"], "max_true_rel_resid": warm["max_true_rel_resid"],
            "errors": warm["errors"] + cold["errors"], "above_tol": warm["above_tol"]}
        if group > 1:
            out[name]["group_sizes"] = sorted({q.group for q in reqs if q.error is None})
            out[name]["group_max_sites"] = gmax
            out[name]["host_rounds"] = svc.group_rounds - rounds0
            out[name]["launches"] = svc.group_launches[0] - launches0[0]
            out[name]["launches_if_alone"] = svc.group_launches[1] - launches0[1]
            out[name]["phases_s"] = {k: round(svc.group_phase_s[i] - phase0[i], 4) for i, k in
                                     enumerate(("setup", "group_solve", "results"))}
            out[name]["group_solve_host_s"] = {k[2:]: round(v - host0[k], 4)
                                               for k, v in svc.group_host_s.items()}
    return out


def bench_uneven(args):
    """48 independent solves, volumes drawn uniformly from 8^4, 12^3x24,
    16^3x32 and 24^3x48, each on its own seeded gauge field (generated on the
    GPU), csw 1.7, kappa 0.1365, Gaussian sources, 1e-10, precision form.
    All 48 are submitted at once to the solve service, run four ways:
    `workers_N`, N workers solving concurrently on separate CUDA streams
    (the small lattices fill a fraction of the SMs each); `workers_1`, one
    after another; `group`, one worker running all 48 as one group solve
    (qws_b200.group_solve: every kernel step one launch over all lattices at
    that step); `group_small`, N workers where the lattices of at most
    300,000 sites (whose own launches underfill the GPU) form one group solve
    and the larger ones run on their own streams beside it.  `small_volumes`
    repeats streams / one at a time / group for 48 solves drawn from 8^4 and
    12^3x24 only, the launch-bound case."""
    vols = [(8, 8, 8, 8), (12, 12, 12, 24), (16, 16, 16, 32), (24, 24, 24, 48)]
    rng = np.random.default_rng(4)
    picks = [vols[int(rng.integers(len(vols)))] for _ in range(48)]
    w = args.uneven_workers
    out = _uneven_pass(args, picks, vols,
                       [(f"workers_{w}", w, 1, None), ("workers_1", 1, 1, None),
                        ("group", 1, 48, None), ("group_small", w, 48, 300000)])
    c, one = out[f"workers_{w}"], out["workers_1"]
    g, gs = out["group"], out["group_small"]
    out["value"] = max(c["solves_per_s"], g["solves_per_s"], gs["solves_per_s"])
    out["unit"] = "solves/s"
    out["speedup_vs_one_at_a_time"] = c["solves_per_s"] / one["solves_per_s"]
    out["group_vs_streams"] = g["solves_per_s"] / c["solves_per_s"]
    out["group_small_vs_streams"] = gs["solves_per_s"] / c["solves_per_s"]
    svols = vols[:2]
    rng = np.random.default_rng(5)
    spicks = [svols[int(rng.integers(len(svols)))] for _ in range(48)]
    small = _uneven_pass(args, spicks, svols, [(f"workers_{w}", w, 1, None),
                                               ("workers_1", 1, 1, None), ("group", 1, 48, None)])
    small["group_vs_streams"] = small["group"]["solves_per_s"] / small[f"workers_{w}"]["solves_per_s"]
    small["group_vs_one_at_a_time"] = (small["group"]["solves_per_s"] /
                                       small["workers_1"]["solves_per_s"])
    out["small_volumes"] = small
    out["method"] = ("qws_b200.serve.Service: one resident field per gauge, clover built on the "
                     "GPU, bicgstab_dd_mix2_hf per request (workers_N: on the worker's stream; "
                     "group: the requests of the pass in one group solve); the wall-clock span "
                     "from submission to the last result, host sources and solutions included")
    return out


def bench_serving(args):
    """A short window of the serving workload: Poisson arrivals, volumes
    16^3x32 / 24^3x48 / 32^3x64 / 48^3x96 (weights .4/.3/.2/.1), kappa uniform
    in [0.130, 0.137], csw 1.7, Gaussian or point sources, tolerance in
    {1e-8, 1e-10, 1e-12}, against a 150 GB HBM budget (qws_b200.serve).
    The service is warmed first: one request per (volume, gauge field) makes
    every field resident, so the window measures the steady state of a
    long-running service (field generation on first use is reported as
    `warmup_s`)."""
    import qws_b200
    from qws_b200 import serve

    vols = [(16, 16, 16, 32), (24, 24, 24, 48), (32, 32, 32, 64), (48, 48, 48, 96)]
    svc = serve.Service(serve.seeded_gauge(), budget_bytes=150e9, workers=3, max_batch=16)
    try:
        t0 = time.monotonic()
        warm = [svc.submit(serve.Request(L=L, gauge=gid, kappa=0.1335, csw=1.7, tol=1e-8,
                                         source=qws_b200.gen_source(L, 4000 + gid, "gauss")))
                for L in vols for gid in range(args.serve_gauges)]
        for q in warm:
            q.wait(600)
        warmup_s = time.monotonic() - t0
        reqs = serve.poisson_workload(svc, args.serve_rate, args.serve_window, vols,
                                      [0.4, 0.3, 0.2, 0.1], args.serve_gauges, seed=1)
        for q in reqs:
            q.wait(600)
        out = serve.summarize(reqs)
    finally:
        svc.close()
    out.update({"rate_per_s": args.serve_rate, "window_s": args.serve_window,
                "warmup_s": round(warmup_s, 2), "warmup_errors": sum(q.error is not None for q in warm),
                "warmup_error_kinds": serve.summarize(warm).get("error_kinds", {}),
                "requests": len(reqs), "merged": svc.merged, "fields_evicted": svc.evicted,
                "work_handles_moved": svc.handles_moved,
                "gauges_per_volume": args.serve_gauges, "workers": 3, "budget_gb": 150,
                "solver": "bicgstab_dd_mix2_hf (reliable 5), clover built on the GPU per kappa"})
    return out


def bench_plain_tuned(args, w, U, C, b, stream, world):
    """The plain solver (bicgstab_dd_mix) in the autotuner's configuration
    for it (block grid, sweep counts, CTA size; qws_b200/tuning.json), on the
    workload's fields and source: `steps` timed solves after `warmup`."""
    import torch

    import qws_b200
    from qws_b200 import autotune

    t = autotune.lookup(w["L"], "plain", 1)
    if not t:
        return {"value": None, "note": "no cached plain tuning for this lattice"}
    lat = qws_b200.Lattice(w["L"], t["NB"], tbc=w["tbc"], kappa=w["kappa"], stream=stream)
    try:
        lat.load_fields(U, C)
        lat.set_hop_threads(t["hop_threads"])
        with torch.cuda.stream(stream):
            bd, x = lat.to_device(b), lat.empty("f64")

            def solve():
                x.zero_()
                return lat.bicgstab_dd_mix(x, bd, w["tol"], w["maxiter"], w["tol_s"],
                                           w["maxiter_s"], t["nsap"], t["nm"])

            for _ in range(max(1, args.warmup)):
                solve()
            torch.cuda.synchronize()
            barrier(world)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                st = solve()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = allreduce_max(e0.elapsed_time(e1), world)
            true = lat.true_residual(x, bd)
    finally:
        lat.close()
        torch.cuda.empty_cache()
    return {"value": world * args.steps / (ms * 1e-3), "unit": "solves/s",
            "config": {"block_grid": t["NB"], "nsap": t["nsap"], "nm": t["nm"],
                       "hop_threads": t["hop_threads"]},
            "true_rel_resid": true, "outer_iters": st["outer_iters"],
            "inner_iters": st["inner_iters"]}


def cpu_baseline(w, x_gpu, digests, gpu_solve):
    """The reference's CPU solver on this host, one untimed and one timed
    complete solve of the same workload (about 30 s of host work), and the
    GPU solution's distance to the reference's solution.  The reference's
    inputs come from the oracle's generator; their digests must equal the
    GPU arm's (the same arrays)."""
    import tempfile

    with tempfile.TemporaryDirectory() as td:
        sol = Path(td) / "x_ref.npy"
        ref = run_reference(w, 1, 1, solution_out=sol)
        x_ref = np.load(sol)
    err = float(np.linalg.norm(x_gpu - x_ref) / np.linalg.norm(x_ref))
    return {"value": ref["solves_per_s"], "unit": "solves/s", "cores": ref["threads"],
            "kind": "reference", "sample": ref["sample"],
            "reference_solve": {"outer_iters": ref["outer_iters"],
                                "inner_iters": ref["inner_iters_per_solve"],
                                "true_rel_resid": ref["true_rel_resid"]},
            "gpu_solve": {"outer_iters": gpu_solve["outer_iters"],
                          "inner_iters": gpu_solve["inner_iters"],
                          "true_rel_resid": gpu_solve["true_rel_resid"]},
            "rel_error_vs_reference": err,
            "same_fields": digests == ref["field_sha256"]}


def bench_reference(args, w, name):
    """The reference arm: the reference's own bicgstab_dd_mix_ (built from its
    sources, oracle/_ref) on this host's cores, `warmup` untimed and `steps`
    timed complete solves of the same workload, in one process."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ref = run_reference(w, args.warmup, args.steps)
    v = ref["solves_per_s"]
    line = {
        "impl": "reference",
        "metric": METRIC,
        "metric_detail": METRIC_DETAIL,
        "value": v, "unit": "solves/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 outer / f32 inner", "data": "synthetic: seeded SU(3) links + 5 APE steps "
        "(plaquette %.4f), clover-leaf clover, Gaussian source; arrays bit-equal to the GPU "
        "arm's (field_sha256)" % ref["plaquette"],
        "config": dict(config_of(w, name), parallelism="host threads x%d" % ref["threads"]),
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": ref["threads"],
                         "kind": "reference", "sample": ref["sample"]},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "solve": {"outer_iters": ref["outer_iters"], "inner_iters": ref["inner_iters_per_solve"],
                  "inner_solves": ref["inner_solves_per_solve"],
                  "true_rel_resid": ref["true_rel_resid"]},
        "solve_s": ref["solve_s"],
        "field_sha256": ref["field_sha256"],
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch", type=int, default=16,
                    help="right-hand sides of the multi-RHS sub-result (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=5.0,
                    help="arrival rate of the serving sub-result (0: skip)")
    ap.add_argument("--serve-window", type=float, default=30.0)
    ap.add_argument("--serve-gauges", type=int, default=4)
    ap.add_argument("--uneven-workers", type=int, default=8,
                    help="workers of the 48 uneven-volume solves sub-result (0: skip)")
    ap.add_argument("--batch48", type=int, default=4,
                    help="right-hand sides of the 48^3x96 multi-RHS precision-form run")
    ap.add_argument("--reps48", type=int, default=5,
                    help="timed solves per 48^3x96 measurement (at least 5)")
    ap.add_argument("--tune", default="cache", choices=["cache", "retune", "off"],
                    help="precision-form configuration: the autotuner's cached choice "
                         "(tuning on a miss), a fresh tuning run, or the reference partition")
    ap.add_argument("--config3", type=int, default=1,
                    help="run the 48^3x96 precision-form comparison (0: skip)")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        bench_reference(args, w, args.workload)
    else:
        bench_ours(args, w, args.workload)


if __name__ == "__main__":
    main()
