#!/usr/bin/env python
"""Credited solve TFLOP/s of the single-GPU HPL-MxP path.

One step = one whole solve of a freshly generated system: blocked no-pivot LU
with the tcgen05 Schur update plus FP64 iterative refinement to scaled
residual < 16.  Credited FLOPs are the reference's (2/3 N^3 + 3/2 N^2,
main.cpp:663); the time is LU + refinement with generation excluded, as in
main.cpp:617-657.  Default workload: N=122880, B=2560, seed 7.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--form fp8|fp16|bf16x2]
                    [--compare fp16|...|none] [--no-forward-error]
    python bench.py --impl reference      # CPU implementation of the path
The headline value is the FP8 form; the plain FP16 form is solved beside it on
the same system ("plain", "ratio_vs_plain"), and both solutions are compared
with an FP64 reference solve ("forward_error").
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

METRIC = "solve TFLOP/s ((2/3N^3+3/2N^2)/t) at residual<16: FP8 form vs FP16 plain"
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


def cpu_kind():
    """"reference" when the reference's CPU kernels were compiled (oracle/_ref),
    else "port" (the oracle's restatement alone)."""
    from oracle import oracle as O
    return "reference" if O.ref_available() else "port"


def cpu_solve_once(form_id: int = 0):
    from oracle import oracle as O
    n, b, seed = CPU_SAMPLE["n"], CPU_SAMPLE["b"], CPU_SAMPLE["seed"]
    rc, x, st = O.solve(n, b, seed, 0, form_id, 50, ref_kernels=cpu_kind() == "reference")
    t = st["t_lu"] + st["t_ir"]
    return hpl_flops(n) / t / 1e12, t, st, O.lib().orc_num_threads()


def cpu_baseline(samples: int = 2):
    """One untimed solve (threads and pages warm), then the mean rate of
    `samples` timed solves."""
    cpu_solve_once()
    tot_t, cores = 0.0, 1
    for _ in range(samples):
        v, t, st, cores = cpu_solve_once()
        tot_t += t
    return {"value": hpl_flops(CPU_SAMPLE["n"]) * samples / tot_t / 1e12, "unit": "TFLOP/s", "cores": cores,
            "kind": cpu_kind(), "sample": cpu_baseline_sample_text(cores)}


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
        "config": cpu_sample_config(),
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": cores, "kind": cpu_kind(),
                         "sample": cpu_baseline_sample_text(cores)},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    barrier(dist)
    return 0


def cpu_baseline_sample_text(cores):
    what = ("the reference's compiled CPU kernels (sgetrf_nopiv_omp<6> for the diagonal blocks, "
            "otf_gemv_kernel for the residual) with the oracle's restated panel TRSM, FP16-emulated "
            "Schur update and triangular solves" if cpu_kind() == "reference" else
            "the oracle's CPU restatement of the reference's path (oracle/mxp_oracle.c)")
    return (f"whole solve (LU + classic IR, generation excluded) at N={CPU_SAMPLE['n']}, B={CPU_SAMPLE['b']}, "
            f"seed {CPU_SAMPLE['seed']} per step on {cores} OpenMP threads: {what}; a bounded sample "
            f"(the N=122880 solve would take hours on the host)")


def cpu_sample_config():
    n, b, seed = CPU_SAMPLE["n"], CPU_SAMPLE["b"], CPU_SAMPLE["seed"]
    return {"workload": (f"HPL-MxP solve N={n} B={b} seed={seed} on the host cores: FP16-emulated Schur, "
                         "FP32 panels, FP64 classic IR to scaled residual<16 (the CPU configuration; a "
                         "bounded sample beside the N=122880 GPU workload)"),
            "n": n, "b": b, "seed": seed, "form": "fp16", "diag_rule": "rowsum", "ir": "classic",
            "trsm": "fp32 substitution", "parallelism": "OpenMP threads of one host"}


def workload_config(args):
    return {"workload": (f"HPL-MxP solve N={args.n} B={args.b} seed={args.seed} "
                         f"{args.form}-Schur + FP64 {args.ir} IR to scaled residual<16"
                         + (f", beside the {args.compare} plain form" if args.compare not in
                            ("none", args.form) else "")),
            "n": args.n, "b": args.b, "seed": args.seed, "form": args.form,
            "compare": args.compare,
            "diag_rule": "rowsum" if args.diag_rule == 0 else "0.55*rowsum+1",
            "ir": args.ir, "trsm": args.trsm, "compare_trsm": args.compare_trsm,
            "merge_depth": args.merge_depth if args.merge_depth is not None else 4,
            "parallelism": "replicas (one independent system per GPU)",
            "l2": f"inputs larger than L2 (A = {args.n * args.n * 4 / 1e9:.1f} GB per GPU)"}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
TRSM_TEXT = {"tensor": "TRSM by inverse, three split-BF16 products (near FP32)",
             "single": "TRSM by inverse, one BF16 product",
             "simt": "FP32 SIMT substitution"}
def _solve_arm(args, form_name, p, dev, dist, local, e2e_on, trsm=None):
    """Warm up, then time args.steps solves of form `form_name` on problem p."""
    import torch

    import openmxp_b200 as mxp

    ws_n = dist_env()[0]
    form = mxp.FORMS[form_name]
    n, b = args.n, args.b
    trsm = args.trsm if trsm is None else trsm
    ws = mxp.Workspace(n, b, form, device=local, trsm_tensor=(trsm != "simt"),
                       trsm_single=(trsm == "single"))
    if args.trsm_pair:
        ws.set_option(mxp.OPT_TRSM_PAIR, 1)
    if args.merge_depth is not None:
        ws.set_option(mxp.OPT_MERGE_DEPTH, args.merge_depth)
    if args.inv_tc is not None:
        ws.set_option(mxp.OPT_INV_TC, args.inv_tc)
    if args.overlap_diag is not None:
        ws.set_option(mxp.OPT_OVERLAP_DIAG, args.overlap_diag)
    if args.overlap_min is not None:
        ws.set_option(mxp.OPT_OVERLAP_MIN, args.overlap_min)
    if args.trsv_inv is not None:
        ws.set_option(mxp.OPT_TRSV_INV, args.trsv_inv)
    if args.fp8_fused_cast is not None:
        ws.set_option(mxp.OPT_FP8_FUSED_CAST, args.fp8_fused_cast)
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
    x_keep = x.clone()

    total_ms = max_over_ranks(sum(step_ms), dist, dev)
    value = hpl_flops(n) * args.steps * ws_n / (total_ms / 1e3) / 1e12

    e2e = None
    if e2e_on:
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
    ws.close()
    last_ir = irs[-1]
    return {
        "form": form_name, "value": value, "ms_per_step": total_ms / args.steps, "e2e": e2e,
        "clocks": clk, "gpu_launches": launches,
        "ir": {"iterations": last_ir["iterations"], "inner": last_ir["inner_iterations"],
               "hpl_harness": last_ir["hpl_harness"], "residual": last_ir["residual"],
               "converged": last_ir["converged"]},
        "phases_ms": {k: sum(l[k] for l in lus) / len(lus)
                      for k in ("ms_total", "ms_diag_lu", "ms_trsm", "ms_trsm_inv", "ms_trsm_gemm",
                                "ms_cast", "ms_schur")},
        "ir_ms": sum(i["ms_total"] for i in irs) / len(irs),
        "overlapped_diag": lus[-1]["overlapped_diag"],
        "x": x_keep,
    }


# DRAM bytes (read + write) per Schur launch over the algorithmic bytes (C read +
# write, L and R panels once), from one ncu capture of each kernel at
# m = n = 16384.  The traffic of a launch of the solve is this ratio
# times its algorithmic bytes: the C read-modify-write dominates both.
SCHUR_TRAFFIC_RATIO = {"schur_tc_f16_kernel": 2.853 / 2.315, "schur_tc_fp8_kernel": 2.857 / 2.315}


def _schur_launch_bytes(n, b, es, kmul, depth=4):
    """Average algorithmic bytes of one trailing Schur launch of the merged
    schedule (groups of `depth` panels, K = depth * b)."""
    tot, cnt = 0.0, 0
    for k in range(0, n // b, depth):
        m = n - (k + depth) * b
        if m <= 0:
            break
        K = depth * b * kmul
        tot += 8.0 * m * m + 2.0 * m * K * es
        cnt += 1
    return tot / max(cnt, 1)


def _roofline(args, arm):
    """Dominant kernel: the tcgen05 Schur update, event-timed on the solve stream."""
    import openmxp_b200 as mxp
    form = mxp.FORMS[arm["form"]]
    kmul = 3 if form == mxp.FORM_BF16X2 else 1
    es = 1 if form == mxp.FORM_FP8 else 2
    schur_ms = arm["phases_ms"]["ms_schur"]
    sflops = schur_flops(args.n, args.b, kmul)
    peaks, peak_kind = load_peaks()
    bf16 = peaks.get("bf16_tflops_sustained", PEAKS_FALLBACK["bf16_tflops_sustained"])
    if form == mxp.FORM_FP8:
        # no FP8 figure is measured for this pool: FP8 dense issues at twice the
        # BF16 rate per SM, so the denominator is 2 x the measured BF16 peak
        peak, src = 2.0 * bf16, f"2 x {peak_kind} bf16 dense sustained (MEASURED_PEAKS.json)"
        kern = "schur_tc_fp8_kernel"
    else:
        peak, src = bf16, f"{peak_kind} bf16 dense sustained (MEASURED_PEAKS.json)"
        kern = "schur_tc_f16_kernel"
    achieved = sflops / (schur_ms / 1e3) / 1e12 if schur_ms > 0 else None
    depth = args.merge_depth if args.merge_depth is not None else 4
    alg = _schur_launch_bytes(args.n, args.b, es, kmul, depth)
    return {"bound": "tensor", "kernel": kern, "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": (achieved / peak) if achieved else None,
            "peak_source": src,
            "traffic": SCHUR_TRAFFIC_RATIO[kern] * alg if kern in SCHUR_TRAFFIC_RATIO else None,
            "traffic_note": ("bytes per average trailing launch: ncu DRAM/algorithmic ratio at "
                             "m=16384 times the launch's algorithmic bytes"),
            "algorithmic_per_launch": ("achieved: sum over steps of 2*m_k^2*B flops (x3 for bf16x2), "
                                       "m_k = N-(k+1)B, over the Schur phase's event time; traffic: "
                                       "C read + write 8*m^2 plus panels m*K per trailing pass, "
                                       f"K = {depth}B")}


def run_gpu(args):
    import torch

    import openmxp_b200 as mxp

    ws_n, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = init_dist("nccl") if ws_n > 1 else None
    n = args.n
    seed = args.seed + (rank if args.distinct_seeds else 0)

    p = mxp.panel_matgen(n, seed, args.diag_rule)
    arm = _solve_arm(args, args.form, p, dev, dist, local, not args.no_e2e)
    plain = None
    if args.compare not in ("none", args.form):
        plain = _solve_arm(args, args.compare, p, dev, dist, local, False, trsm=args.compare_trsm)
    # the headline form again with the plain form's TRSM: a like-for-like ratio
    same = None
    if plain is not None and not args.no_same_trsm and args.trsm != args.compare_trsm:
        same = _solve_arm(args, args.form, p, dev, dist, local, False, trsm=args.compare_trsm)
    rhs = p.rhs.clone()
    del p
    torch.cuda.empty_cache()

    fwd = None
    if not args.no_forward_error:
        from openmxp_b200 import forward_error as fe
        x_ref = fe.reference_solution(n, seed, args.diag_rule, rhs)
        fwd = {arm["form"]: fe.forward_error(arm["x"], x_ref)}
        if plain is not None:
            fwd[plain["form"]] = fe.forward_error(plain["x"], x_ref)
        if same is not None:
            fwd[same["form"] + "_" + args.compare_trsm + "_trsm"] = fe.forward_error(same["x"], x_ref)
        del x_ref
        torch.cuda.empty_cache()

    if rank == 0:
        cpu = None
        if ws_n == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(1)
        line = {
            "metric": METRIC, "value": arm["value"], "unit": "TFLOP/s", "n_gpus": ws_n,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": arm["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp16": "f16", "bf16x2": "bf16", "fp8": "e4m3"}[args.form],
            "data": "synthetic (HPL-MxP LCG generator; generation excluded from t)",
            "config": workload_config(args),
            "roofline": _roofline(args, arm), "cpu_baseline": cpu, "e2e": arm["e2e"],
            "clocks": arm["clocks"], "gpu_launches": arm["gpu_launches"],
            "ir": arm["ir"], "phases_ms": arm["phases_ms"], "ir_ms": arm["ir_ms"],
            "overlapped_diag": arm["overlapped_diag"],
            "forward_error": fwd,
            "forward_error_reference": ("FP64 no-pivot blocked LU of the FP64 system (mxp_matgen_f64) "
                                        "with cuSOLVER/cuBLAS FP64 calls; ||x-x64||inf/||x64||inf"),
        }
        if plain is not None:
            line["plain"] = {k: plain[k] for k in ("form", "value", "ms_per_step", "ir", "phases_ms",
                                                   "ir_ms", "clocks", "gpu_launches", "overlapped_diag")}
            line["plain"]["roofline"] = _roofline(args, plain)
            line["ratio_vs_plain"] = arm["value"] / plain["value"]
            line["trsm_forms"] = {
                args.form: TRSM_TEXT[args.trsm], args.compare: TRSM_TEXT[args.compare_trsm],
                "why": ("the headline form's panels are rounded to E4M3 (2^-4) right after the TRSM, so one "
                        "BF16 product (2^-9) does not limit its factors; the reference's own production "
                        "runs use a single low-precision product too (Alt-TRSM, panel_trf_gdirect.hpp:73-107). "
                        "The plain form keeps FP32-accurate panels, as its method (FP32 panels) specifies")}
        if same is not None:
            line["same_trsm"] = {k: same[k] for k in ("form", "value", "ms_per_step", "ir", "phases_ms", "ir_ms")}
            line["same_trsm"]["trsm"] = TRSM_TEXT[args.compare_trsm]
            line["ratio_vs_plain_same_trsm"] = same["value"] / plain["value"]
        print(json.dumps(line), flush=True)
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
    elif args.micro == "trsm":
        # one panel solve by inverse (mxp_trsm_inv_*: casts + triangular product), m = --n, b = --b,
        # the right side (B <- B inv(U)) and the left side (B <- inv(L) B) in turn
        single = args.trsm == "single"
        ws = mxp.Workspace(m + b, b, mxp.FORM_FP16, trsm_single=single)
        P = (torch.rand(m * b, device="cuda", generator=g) - 0.5).float()
        X = torch.eye(b, device="cuda").t().contiguous()
        X += torch.triu(torch.rand(b, b, device="cuda", generator=g) * 1e-3, 1).t()  # column-major upper
        X = X.reshape(-1)
        XLm = X.view(b, b).t().contiguous().reshape(-1)  # its transpose: unit lower, column-major
        res = {}
        for side in ("right", "left"):
            def launch(side=side):
                if side == "right":
                    mxp.trsm_inv_right_upper(m, b, X, b, P, m, ws, single=single)
                else:
                    mxp.trsm_inv_left_lower(b, m, XLm, b, P, b, ws, single=single)
            for _ in range(args.warmup):
                launch()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(args.steps):
                launch()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / args.steps
            fl = float(m) * b * b * (1 if single else 3)  # triangular: m b^2 (x3 split)
            res[side] = {"ms_per_call": ms, "tflops": fl / ms / 1e9}
        out.update(res, trsm="single BF16" if single else "split BF16 x3")
        ws.close()
        print(json.dumps(out), flush=True)
        return 0
    elif args.micro == "diag":
        # diagonal-block factorisation alone (n = --b): LU, and LU + both triangular
        # inverses, as one cooperative launch and as the per-step launch chain
        n = b
        p = mxp.panel_matgen(n, 3)
        A0 = p.A.clone()
        XU = torch.empty(n * n, device="cuda")
        XL = torch.empty(n * n, device="cuda")
        res = {}
        for coop in (True, False):
            ws = mxp.Workspace(n, n, 0, diag_coop=coop)
            if args.inv_tc is not None:
                ws.set_option(mxp.OPT_INV_TC, args.inv_tc)
            for inv in (False, True):
                tot = 0.0
                for it in range(args.warmup + args.steps):
                    p.A.copy_(A0)
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record()
                    if inv:
                        mxp.getrf_nopiv_inv(p.A, n, n, XU, XL, n, ws)
                    else:
                        mxp.getrf_nopiv(p.A, n, n, ws)
                    e1.record()
                    torch.cuda.synchronize()
                    if it >= args.warmup:
                        tot += e0.elapsed_time(e1)
                res[f"{'coop' if coop else 'chain'}_{'lu_inv' if inv else 'lu'}_ms"] = tot / args.steps
            ws.close()
        out.update(res)
        print(json.dumps(out), flush=True)
        return 0
    elif args.micro == "cublas":
        # vendor yardstick at the Schur shape: C(m x m) = L(m x b) . R(m x b)^T through
        # cuBLAS (torch.mm, FP16 in / FP32 out; torch._scaled_mm for FP8 E4M3 with
        # tensor-wise scales).  Not part of the solve path.
        ws = None
        if es == 1:
            A8 = (torch.randn(m, b, device="cuda", generator=g) * 8).to(torch.float8_e4m3fn)
            B8 = (torch.randn(m, b, device="cuda", generator=g) * 8).to(torch.float8_e4m3fn)
            one = torch.ones((), device="cuda")
            out_dt = torch.float32
            try:
                torch._scaled_mm(A8[:256], B8[:256].t(), scale_a=one, scale_b=one, out_dtype=out_dt)
            except Exception:  # FP32 output not offered: BF16 output (half the C bytes)
                out_dt = torch.bfloat16
            out["out_dtype"] = str(out_dt)

            def launch():
                torch._scaled_mm(A8, B8.t(), scale_a=one, scale_b=one, out_dtype=out_dt)
        else:
            A16 = torch.randn(m, b, device="cuda", generator=g).half()
            B16 = torch.randn(m, b, device="cuda", generator=g).half()
            try:
                torch.mm(A16[:256], B16[:256].t(), out_dtype=torch.float32)
                out["out_dtype"] = "torch.float32"

                def launch():
                    torch.mm(A16, B16.t(), out_dtype=torch.float32)
            except Exception:
                out["out_dtype"] = "torch.float16"

                def launch():
                    torch.mm(A16, B16.t())
        flops = 2.0 * m * m * b
    else:
        raise SystemExit(f"unknown micro benchmark {args.micro}")
    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize()
    if args.micro_seconds > 0:  # sustained: repeat until the power cap has settled
        t_end = time.perf_counter() + args.micro_seconds
        while time.perf_counter() < t_end:
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


# ---------------------------------------------------------------------------
# batched form: 2048 systems of uneven orders in one persistent launch
# ---------------------------------------------------------------------------
def batch_flops(sizes) -> float:
    return sum(hpl_flops(n) for n in sizes)


def run_batched(args):
    """Systems/s and credited TFLOP/s of the batched solve (one graph-replayed
    persistent launch per step), beside a per-system loop of the plain
    single-system path (mxp_solve, FP16 Schur) over the same systems."""
    import torch

    import openmxp_b200 as mxp
    world, rank, local = dist_env()
    dist = init_dist("nccl") if world > 1 else None
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    all_sizes = mxp.batch_sizes(args.batch_count, args.batch_size_seed)
    all_seeds = [1000 + i for i in range(len(all_sizes))]
    # independent systems: each rank solves its part (balanced by n^3), no
    # exchange between GPUs; the job time is the slowest rank's
    part = mxp.batch_partition(all_sizes, world) if world > 1 else [0] * len(all_sizes)
    mine = [i for i in range(len(all_sizes)) if part[i] == rank]
    sizes = [all_sizes[i] for i in mine]
    seeds = [all_seeds[i] for i in mine]
    bt = mxp.Batch(sizes, seeds, device=local)
    bt.matgen()
    tune = bt.autotune() if not args.batch_config else None
    if args.batch_config:
        b, tn, stg = (int(v) for v in args.batch_config.split(","))
        bt.set_config(b, tn, stg)
    flops = batch_flops(all_sizes)
    for _ in range(args.warmup):
        bt.matgen()
        bt.solve()
    ms = []
    clocks = ClockSampler(local)
    clocks.start()
    mxp.reset_kernel_launches()
    for _ in range(args.steps):
        bt.matgen()
        torch.cuda.synchronize()
        barrier(dist)
        ms.append(max_over_ranks(bt.solve()["ms_total"], dist, dev))
    launches = int(sum_over_ranks(mxp.kernel_launches(), dist, dev))
    clk = clocks.stop()
    res = bt.results()
    t = sum(ms) / len(ms) / 1e3
    converged = int(sum_over_ranks(sum(r["converged"] for r in res), dist, dev))
    max_it = int(max_over_ranks(max(r["iterations"] for r in res), dist, dev))
    max_hpl = max_over_ranks(max(r["hpl_harness"] for r in res), dist, dev)
    out = {"metric": "batched solve: systems/s and credited TFLOP/s", "value": len(all_sizes) / t,
           "unit": "systems/s", "tflops": flops / t / 1e12, "ms_per_step": 1e3 * t, "n_gpus": world,
           "scaling": "strong", "steps": args.steps, "warmup": args.warmup, "systems": len(all_sizes),
           "orders": {"min": min(all_sizes), "max": max(all_sizes),
                      "sum_n3": float(sum(n ** 3 for n in all_sizes))},
           "config": tune if tune else {"b": b, "tile_n": tn, "stages": stg},
           "converged": converged, "max_iterations": max_it, "max_hpl_harness": max_hpl,
           "gpu_launches": launches, "clocks": clk}
    if world > 1:
        out["partition"] = "systems split by n^3 (mxp_batch_partition); rank 0 share of n^3: %.3f" % (
            sum(n ** 3 for n in sizes) / sum(n ** 3 for n in all_sizes))
    # per-system loop of the plain single-system path on a sample of the systems
    if args.batch_loop_sample > 0 and world == 1:
        stride = max(1, len(sizes) // args.batch_loop_sample)
        idx = list(range(0, len(sizes), stride))[: args.batch_loop_sample]
        loop_s, loop_flops = 0.0, 0.0
        for i in idx:
            n = sizes[i]
            p = mxp.panel_matgen(n, seeds[i])
            bb = 256 if n % 256 == 0 else 128
            ws = mxp.Workspace(n, bb, mxp.FORM_FP16)
            mxp.solve(p, bb, ws)  # warm
            mxp.regenerate(p)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            mxp.solve(p, bb, ws)
            e1.record()
            torch.cuda.synchronize()
            loop_s += e0.elapsed_time(e1) / 1e3
            loop_flops += hpl_flops(n)
            ws.close()
            del p
        out["per_system_loop"] = {"systems_timed": len(idx), "systems_per_s": len(idx) / loop_s,
                                  "tflops": loop_flops / loop_s / 1e12,
                                  "what": "mxp_solve (FP16 Schur, B=256 or 128, classic IR) one system at a time"}
        out["speedup_vs_loop"] = out["value"] / out["per_system_loop"]["systems_per_s"]
    bt.close()
    if rank == 0:
        print(json.dumps(out), flush=True)
    barrier(dist)
    if dist is not None:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# one system over a P x Q grid of GPUs (2D block-cyclic driver, strong scaling)
# ---------------------------------------------------------------------------
def run_grid(args):
    """Credited TFLOP/s of ONE system of order --n factored and refined by a
    P x Q grid of GPUs (openmxp_b200.grid: block-cyclic layout, the diagonal
    block's triangular inverses (or, with --trsm simt, the factored block) and
    the low-precision panels broadcast over NCCL along process rows and
    columns, panels by inverse on the tensor cores, depth-1 look-ahead unless
    --no-lookahead, tcgen05 Schur update, refinement with the local
    regenerating GEMV summed over all ranks).  One step = one solve of the
    freshly regenerated local blocks; the time is LU + refinement, max over
    ranks."""
    import torch

    import openmxp_b200 as mxp
    from openmxp_b200 import grid as G
    P, Q = (int(v) for v in args.grid.lower().split("x"))
    world, rank, local = dist_env()
    if P * Q != world:
        raise SystemExit(f"--grid {args.grid} needs {P * Q} ranks, got {world}")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = init_dist("nccl") if world > 1 else None
    form = mxp.FORMS[args.form]
    g = G.ProcessGrid(P, Q, dist=dist)
    be = G.CudaBackend(args.b, form)
    gtrsm = {"tensor": "split", "single": "single", "simt": "strsm"}[args.trsm]
    s = G.BlockCyclicSolver(g, args.n, args.b, args.seed, be, form=form, diag_rule=args.diag_rule, trsm=gtrsm,
                            lookahead=not args.no_lookahead)
    h_rhs = s.rhs.cpu().pin_memory()
    h_x = torch.empty(args.n, dtype=torch.float64).pin_memory()

    def step(e2e: bool):
        s.regenerate()
        torch.cuda.synchronize()
        barrier(dist)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        if e2e:
            s.rhs.copy_(h_rhs, non_blocking=True)
        s.factor()
        x, st = s.refine(maxit=args.maxit)
        if e2e:
            h_x.copy_(x, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), dist, dev), st

    for _ in range(args.warmup):
        step(False)
    clocks = ClockSampler(local)
    clocks.start()
    mxp.reset_kernel_launches()
    ms, st = [], None
    for _ in range(args.steps):
        t, st = step(False)
        ms.append(t)
    launches = int(sum_over_ranks(mxp.kernel_launches(), dist, dev))
    clk = clocks.stop()
    e2e_ms = [step(True)[0] for _ in range(max(1, args.e2e_steps))]
    flops = hpl_flops(args.n)
    t = sum(ms) / len(ms) / 1e3
    te = sum(e2e_ms) / len(e2e_ms) / 1e3
    out = {"metric": METRIC, "value": flops / t / 1e12, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "strong",
           "vs_baseline": None, "dtype": {"fp16": "f16", "bf16x2": "bf16", "fp8": "e4m3"}[args.form],
           "data": "synthetic (HPL-MxP LCG generator; generation excluded from t)",
           "config": {"workload": f"HPL-MxP solve N={args.n} B={args.b} seed={args.seed} {args.form}-Schur + "
                                  f"FP64 classic IR over a {P}x{Q} process grid (2D block-cyclic)",
                      "n": args.n, "b": args.b, "seed": args.seed, "form": args.form, "grid": f"{P}x{Q}",
                      "parallelism": f"2D block-cyclic {P}x{Q}, NCCL broadcasts of the diagonal block "
                                     "(its inverses) and the low-precision panels",
                      "trsm": {"split": "by inverse, three split-BF16 tensor-core products",
                               "single": "by inverse, one BF16 tensor-core product",
                               "strsm": "STRSM (SIMT FP32)"}[gtrsm] + " on the local panels",
                      "lookahead": int(s.lookahead),
                      "l2": "inputs larger than L2" if args.n * args.n * 4 // world > 126e6 else "fits L2"},
           "ir": {"iterations": st.iterations, "converged": int(st.converged), "hpl_harness": st.hpl_harness,
                  "residual": st.residual},
           "e2e": {"value": flops / te / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": 8 * args.n,
                   "d2h_bytes_per_step": 8 * args.n,
                   "api": "BlockCyclicSolver.factor + refine, pinned host rhs in / x out on every rank"},
           "gpu_launches": launches, "clocks": clk}
    be.close()
    if rank == 0:
        print(json.dumps(out), flush=True)
    barrier(dist)
    if dist is not None:
        dist.destroy_process_group()
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
    ap.add_argument("--form", choices=["fp16", "bf16x2", "fp8"], default="fp8")
    ap.add_argument("--compare", choices=["fp16", "bf16x2", "fp8", "none"], default="fp16",
                    help="form measured beside --form on the same system (the plain FP16 form)")
    ap.add_argument("--no-forward-error", action="store_true",
                    help="skip the FP64 reference solve (8 N^2 bytes of device memory)")
    ap.add_argument("--diag-rule", type=int, default=0)
    ap.add_argument("--maxit", type=int, default=50)
    ap.add_argument("--ir", choices=["classic", "gmres"], default="classic")
    ap.add_argument("--trsm", choices=["auto", "tensor", "single", "simt"], default="auto",
                    help="panel TRSM: tensor-core by inverse in three split-BF16 products (near FP32), "
                         "one BF16 product, or SIMT FP32; auto = single for the FP8 form "
                         "(its panels are E4M3 next), tensor otherwise")
    ap.add_argument("--compare-trsm", choices=["tensor", "single", "simt"], default="tensor",
                    help="panel TRSM of the --compare arm (the plain method: FP32-accurate)")
    ap.add_argument("--no-lookahead", action="store_true",
                    help="--grid: update the whole trailing matrix before forming the next panel")
    ap.add_argument("--no-same-trsm", action="store_true",
                    help="skip the third arm: --form again with --compare-trsm (the like-for-like ratio)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--micro", choices=["schur", "otf_gemv", "cublas", "diag", "trsm"], default=None,
                    help="time one kernel alone at m=--n, k=--b (for profiler captures)")
    ap.add_argument("--micro-seconds", type=float, default=0.0,
                    help="micro: run the launch this long before timing (sustained clocks)")
    ap.add_argument("--trsm-pair", action="store_true", help="TRSM-by-inverse products on the 2-SM kernel")
    ap.add_argument("--merge-depth", type=int, default=None,
                    help="panels per trailing Schur pass, 1..4 (library default 4)")
    ap.add_argument("--inv-tc", type=int, default=None,
                    help="triangular-inverse doubling levels from this block size on the tensor cores "
                         "(library default 1024; 0: all SIMT FP32)")
    ap.add_argument("--fp8-fused-cast", type=int, default=None,
                    help="1 (library default): the FP8 form's L panels are quantized in the TRSM product's "
                         "epilogue; 0: by a separate cast launch")
    ap.add_argument("--trsv-inv", type=int, default=None,
                    help="1 (library default): refinement solves with the stored inverses of the "
                         "diagonal blocks; 0: the chain of 64-row blocks")
    ap.add_argument("--overlap-diag", type=int, default=None,
                    help="SMs for the diagonal factorisation run beside the trailing pass (0: off)")
    ap.add_argument("--overlap-min", type=int, default=None,
                    help="overlap only while the pair's trailing matrix has this many blocks")
    ap.add_argument("--batched", action="store_true",
                    help="the batched form: --batch-count systems of orders 128*{2..32}")
    ap.add_argument("--batch-count", type=int, default=2048)
    ap.add_argument("--batch-size-seed", type=int, default=3)
    ap.add_argument("--batch-config", default="", help="b,tile_n,stages (default: autotune)")
    ap.add_argument("--batch-loop-sample", type=int, default=128,
                    help="systems timed through the per-system loop for comparison")
    ap.add_argument("--grid", default="",
                    help="PxQ: solve ONE system over a P x Q grid of GPUs (2D block-cyclic; launch "
                         "P*Q ranks with torchrun); strong scaling")
    ap.add_argument("--distinct-seeds", action="store_true",
                    help="rank r solves seed+r instead of the same system")
    return ap.parse_args(argv)


def main(argv=None):
    args = parse(argv)
    if args.trsm == "auto":
        args.trsm = "single" if args.form == "fp8" else "tensor"
    if args.warmup < 3:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        return run_reference(args)
    if args.micro:
        return run_micro(args)
    if args.batched:
        return run_batched(args)
    if args.grid:
        return run_grid(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
