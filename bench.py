#!/usr/bin/env python
"""Credited solve TFLOP/s of the single-GPU HPL-MxP path.

One step = one whole solve of a freshly generated system: blocked no-pivot LU
with the tcgen05 Schur update plus FP64 iterative refinement to scaled
residual < 16.  Credited FLOPs are the reference's (2/3 N^3 + 3/2 N^2,
main.cpp:663); the time is LU + refinement with generation excluded, as in
main.cpp:617-657.  Default workload: N=122880, B=2560, seed 7.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--form fp16|bf16x2|fp8]
    python bench.py --impl reference      # CPU implementation of the path
Under torchrun each rank solves its own system (replicas: the path does not
shard); value = all ranks' credited FLOPs / max-over-ranks time.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solve TFLOP/s ((2/3N^3+3/2N^2)/t) at residual<16"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def hpl_flops(n: int) -> float:
    return 2.0 / 3.0 * n ** 3 + 1.5 * n ** 2


def schur_flops(n: int, b: int, kmul: int) -> float:
    """Tensor-core FLOPs of the Schur updates of one LU: sum_k 2 m_k^2 (kmul b)."""
    tot = 0.0
    for k in range(n // b):
        m = n - (k + 1) * b
        tot += 2.0 * m * m * b * kmul
    return tot


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


# ---------------------------------------------------------------------------
# multi-rank plumbing (replicas); exercised on CPU by tests/test_replicas_gloo.py
# ---------------------------------------------------------------------------
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(backend: str):
    import datetime

    import torch.distributed as dist
    ws, rank, _ = dist_env()
    if ws > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return dist if ws > 1 else None


def max_over_ranks(value: float, dist, device=None) -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist, device=None) -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU path (oracle restatement of the reference's CPU solve), timed on host cores
# ---------------------------------------------------------------------------
CPU_SAMPLE = {"n": 8192, "b": 256, "seed": 42}


def cpu_solve_once(form_id: int = 0):
    from oracle import oracle as O
    n, b, seed = CPU_SAMPLE["n"], CPU_SAMPLE["b"], CPU_SAMPLE["seed"]
    rc, x, st = O.solve(n, b, seed, 0, form_id, 50)
    t = st["t_lu"] + st["t_ir"]
    return hpl_flops(n) / t / 1e12, t, st, O.lib().orc_num_threads()


def cpu_baseline(samples: int = 1):
    vals = []
    for _ in range(samples):
        v, t, st, cores = cpu_solve_once()
        vals.append(v)
    return {"value": max(vals), "unit": "TFLOP/s", "cores": cores, "kind": "port",
            "sample": (f"whole solve (LU + classic IR, generation excluded) at N={CPU_SAMPLE['n']}, "
                       f"B={CPU_SAMPLE['b']}, seed {CPU_SAMPLE['seed']}, FP16-emulated Schur, on "
                       f"{cores} OpenMP threads of the oracle (oracle/mxp_oracle.c); the "
                       f"N=122880 solve would take hours on the host")}


def run_reference(args):
    ws, rank, _ = dist_env()
    dist = init_dist("gloo") if ws > 1 else None
    if rank != 0:
        barrier(dist)
        return 0
    for _ in range(args.warmup):
        cpu_solve_once()
    vals, times = [], []
    for _ in range(args.steps):
        v, t, st, cores = cpu_solve_once()
        vals.append(v)
        times.append(t)
    tot = sum(times)
    value = hpl_flops(CPU_SAMPLE["n"]) * len(times) / tot / 1e12
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f16", "data": "synthetic (HPL-MxP LCG generator)",
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": cores, "kind": "port",
                         "sample": cpu_baseline_sample_text(cores)},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    barrier(dist)
    return 0


def cpu_baseline_sample_text(cores):
    return (f"CPU restatement of the reference's path (oracle/mxp_oracle.c) solving "
            f"N={CPU_SAMPLE['n']}, B={CPU_SAMPLE['b']}, seed {CPU_SAMPLE['seed']} per step on "
            f"{cores} host threads; a bounded stand-in for the N=122880 workload")


def workload_config(args):
    return {"workload": (f"HPL-MxP solve N={args.n} B={args.b} seed={args.seed} "
                         f"{args.form}-Schur + FP64 {args.ir} IR to scaled residual<16"),
            "n": args.n, "b": args.b, "seed": args.seed, "form": args.form,
            "diag_rule": "rowsum" if args.diag_rule == 0 else "0.55*rowsum+1",
            "ir": args.ir, "trsm": args.trsm,
            "parallelism": "replicas (one independent system per GPU)",
            "l2": f"inputs larger than L2 (A = {args.n * args.n * 4 / 1e9:.1f} GB per GPU)"}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu(args):
    import torch

    import openmxp_b200 as mxp

    ws_n, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = init_dist("nccl") if ws_n > 1 else None
    form = mxp.FORMS[args.form]
    kmul = 3 if form == mxp.FORM_BF16X2 else 1
    n, b = args.n, args.b
    seed = args.seed + (rank if args.distinct_seeds else 0)

    p = mxp.panel_matgen(n, seed, args.diag_rule)
    ws = mxp.Workspace(n, b, form, device=local, trsm_tensor=(args.trsm == "tensor"))
    method = mxp.IR_GMRES if args.ir == "gmres" else mxp.IR_CLASSIC
    x = torch.empty(n, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()

    def one_step():
        mxp.regenerate(p)
        torch.cuda.synchronize()
        barrier(dist)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, lst, ist = mxp.solve(p, b, ws, x=x, maxit=args.maxit, method=method)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(dist)
        return e0.elapsed_time(e1), lst, ist

    for _ in range(args.warmup):
        one_step()

    clocks = ClockSampler(local)
    clocks.start()
    step_ms, lus, irs = [], [], []
    mxp.reset_kernel_launches()
    for _ in range(args.steps):
        ms, lst, ist = one_step()
        step_ms.append(ms)
        lus.append(lst)
        irs.append(ist)
    launches = mxp.kernel_launches()
    clk = clocks.stop()

    local_total_ms = sum(step_ms)
    total_ms = max_over_ranks(local_total_ms, dist, dev)
    value = hpl_flops(n) * args.steps * ws_n / (total_ms / 1e3) / 1e12

    # dominant kernel: the tcgen05 Schur update, timed with events on its stream
    schur_ms = sum(l["ms_schur"] for l in lus) / len(lus)
    sflops = schur_flops(n, b, kmul)
    peaks, peak_kind = load_peaks()
    peak = peaks.get("bf16_tflops_sustained", PEAKS_FALLBACK["bf16_tflops_sustained"])
    achieved = sflops / (schur_ms / 1e3) / 1e12 if schur_ms > 0 else None
    roofline = {"bound": "tensor", "kernel": "schur_tc_f16_kernel",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if achieved else None,
                "peak_source": f"{peak_kind} bf16 dense, sustained (MEASURED_PEAKS.json)",
                "traffic": None,
                "algorithmic_per_launch": "2*m_k^2*K flops, m_k = N-(k+1)B, K = B (x3 for bf16x2)"}

    # end-to-end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        h_rhs = torch.empty(n, dtype=torch.float64).pin_memory()
        h_x = torch.empty(n, dtype=torch.float64).pin_memory()
        e2e_s = []
        for _ in range(args.e2e_steps):
            mxp.regenerate(p)
            h_rhs.copy_(p.rhs.cpu())
            torch.cuda.synchronize()
            barrier(dist)
            t0 = time.perf_counter()
            mxp.solve_host(p, b, ws, h_rhs, h_x, maxit=args.maxit, method=method)
            t1 = time.perf_counter()
            barrier(dist)
            e2e_s.append(t1 - t0)
        tot = max_over_ranks(sum(e2e_s), dist, dev)
        e2e = {"value": hpl_flops(n) * len(e2e_s) * ws_n / tot / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
               "api": "mxp_solve_host (C ABI), pinned host rhs in / x out"}

    line = None
    if rank == 0:
        cpu = None
        if ws_n == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(1)
        last_ir = irs[-1]
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": ws_n,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp16": "f16", "bf16x2": "bf16", "fp8": "e4m3"}[args.form],
            "data": "synthetic (HPL-MxP LCG generator; generation excluded from t)",
            "config": workload_config(args),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": launches,
            "ir": {"iterations": last_ir["iterations"], "inner": last_ir["inner_iterations"],
                   "hpl_harness": last_ir["hpl_harness"],
                   "residual": last_ir["residual"], "converged": last_ir["converged"]},
            "phases_ms": {k: sum(l[k] for l in lus) / len(lus)
                          for k in ("ms_total", "ms_diag_lu", "ms_trsm", "ms_trsm_inv", "ms_trsm_gemm",
                                    "ms_cast", "ms_schur")},
            "ir_ms": sum(i["ms_total"] for i in irs) / len(irs),
        }
        print(json.dumps(line), flush=True)
    ws.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# kernel micro-benchmarks (few launches: used for ncu captures)
# ---------------------------------------------------------------------------
def run_micro(args):
    import torch

    import openmxp_b200 as mxp
    torch.cuda.set_device(0)
    form = mxp.FORMS[args.form]
    m, b = args.n, args.b
    kmul = 3 if form == mxp.FORM_BF16X2 else 1
    es = 1 if form == mxp.FORM_FP8 else 2
    ldk = -(-b * kmul // (16 // es)) * (16 // es)
    g = torch.Generator(device="cuda").manual_seed(1)
    out = {"micro": args.micro, "m": m, "b": b, "form": args.form}
    if args.micro == "schur":
        L = (torch.randn(m * b, device="cuda", generator=g) * 1e-3).float()
        U = (torch.randn(b * m, device="cuda", generator=g) * 0.5).float()
        Cm = torch.randn(m * m, device="cuda", generator=g).float()
        dt = torch.uint8 if es == 1 else torch.int16
        Lp = torch.empty(m * ldk, dtype=dt, device="cuda")
        Rp = torch.empty(m * ldk, dtype=dt, device="cuda")
        nsc = (-(-m // 128)) * (-(-b // 128))
        ls = torch.empty(nsc, dtype=torch.uint8, device="cuda")
        rs = torch.empty(nsc, dtype=torch.uint8, device="cuda")
        ws = mxp.Workspace(m + b, b, form)
        mxp.panel_cast_left(form, m, b, L, m, Lp, ldk, ls if es == 1 else None)
        mxp.panel_cast_right(form, m, b, U, b, Rp, ldk, rs if es == 1 else None)

        def launch():
            mxp.schur_update(form, m, m, b, Lp, ldk, Rp, ldk, Cm, m, ws,
                             ls if es == 1 else None, rs if es == 1 else None)
        flops = 2.0 * m * m * b * kmul
    elif args.micro == "otf_gemv":
        d = torch.full((m,), m / 4.0, dtype=torch.float64, device="cuda")
        x = torch.randn(m, dtype=torch.float64, device="cuda", generator=g)
        y = torch.zeros(m, dtype=torch.float64, device="cuda")
        ws = mxp.Workspace(m, min(b, m), 0)

        def launch():
            mxp.otf_gemv(m, 7, d, -1.0, x, 1.0, y, ws)
        flops = 2.0 * m * m
    else:
        raise SystemExit(f"unknown micro benchmark {args.micro}")
    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        launch()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    out.update(ms_per_launch=ms, tflops=flops / (ms / 1e3) / 1e12)
    print(json.dumps(out), flush=True)
    return 0


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mxp", "reference"], default="mxp")
    ap.add_argument("--n", type=int, default=122880)
    ap.add_argument("--b", type=int, default=2560)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--form", choices=["fp16", "bf16x2", "fp8"], default="fp16")
    ap.add_argument("--diag-rule", type=int, default=0)
    ap.add_argument("--maxit", type=int, default=50)
    ap.add_argument("--ir", choices=["classic", "gmres"], default="classic")
    ap.add_argument("--trsm", choices=["tensor", "simt"], default="tensor")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--micro", choices=["schur", "otf_gemv"], default=None,
                    help="time one kernel alone at m=--n, k=--b (for profiler captures)")
    ap.add_argument("--distinct-seeds", action="store_true",
                    help="rank r solves seed+r instead of the same system")
    return ap.parse_args(argv)


def main(argv=None):
    args = parse(argv)
    if args.warmup < 3:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        return run_reference(args)
    if args.micro:
        return run_micro(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
