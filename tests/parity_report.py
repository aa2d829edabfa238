#!/usr/bin/env python
"""Factor parity of mxp_panel_lu against the oracle's restatement of the same
algorithm (oracle/blocked.py) at sizes the pytest suite does not reach, such
as the plain configuration N=61440, B=2560, seed 42: the GPU factors the
system, the factors come back to the host, and the oracle factors the same
generated matrix on the host cores.  One JSON line per arm.

    python tests/parity_report.py --n 61440 --b 2560 --seed 42 --arm fp16_split --arm fp8_single_fused

Arms are configured as bench.py runs them: fp16_split (plain FP16 Schur,
split-BF16 TRSM by inverse), fp8_single_fused (FP8 Schur, one BF16 TRSM
product, E4M3 panels from the TRSM epilogues), bf16x2_split.  Bar: relative
Frobenius distance <= 1e-3 (the factor bar of the FP16 forms) overall
and on the strict lower and upper parts.  Host memory: about 2.3 x 4 N^2
bytes (35 GB at N=61440).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

ARMS = {"fp16_split": (0, False, "split"), "fp8_single_fused": (2, True, "single"),
        "bf16x2_split": (1, False, "split")}


def compare(got: np.ndarray, want: np.ndarray, chunk: int = 1024) -> dict:
    """Relative Frobenius distances (all, strict lower, strict upper), the
    largest entry-wise error of each strict part relative to that part's
    largest entry, and the largest relative error on the diagonal; column
    blocks at a time so no N x N temporary is made."""
    n = got.shape[0]
    acc = {k: [0.0, 0.0, 0.0, 0.0] for k in ("all", "low", "up")}  # sum d^2, sum w^2, max|d|, max|w|
    dmax = 0.0
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        g = got[:, c0:c1].astype(np.float64)
        w = want[:, c0:c1].astype(np.float64)
        d = g - w
        rows = np.arange(n)[:, None]
        cols = np.arange(c0, c1)[None, :]
        for key, mask in (("all", None), ("low", rows > cols), ("up", rows < cols)):
            dd = d if mask is None else d[mask]
            ww = w if mask is None else w[mask]
            a = acc[key]
            a[0] += float(np.sum(dd * dd))
            a[1] += float(np.sum(ww * ww))
            a[2] = max(a[2], float(np.max(np.abs(dd))) if dd.size else 0.0)
            a[3] = max(a[3], float(np.max(np.abs(ww))) if ww.size else 0.0)
        idx = np.arange(c0, c1)
        dmax = max(dmax, float(np.max(np.abs(d[idx, idx - c0]) / np.abs(w[idx, idx - c0]))))
    out = {}
    for key, (sd, sw, md, mw) in acc.items():
        out[f"rel_fro_{key}"] = (sd / sw) ** 0.5
        if key != "all":
            out[f"max_err_{key}_over_max"] = md / mw
    out["max_rel_err_diag"] = dmax
    return out


def run(args, arm: str) -> dict:
    import torch

    import openmxp_b200 as mxp
    from oracle import blocked as Bk
    from oracle import oracle as O

    n, b, seed = args.n, args.b, args.seed
    form, single, trsm = ARMS[arm]
    torch.cuda.set_device(0)
    p = mxp.panel_matgen(n, seed)
    ws = mxp.Workspace(n, b, form, trsm_single=single)
    t0 = time.perf_counter()
    st = mxp.panel_lu(p, b, ws)
    torch.cuda.synchronize()
    t_gpu = time.perf_counter() - t0
    got = np.asfortranarray(p.A.view(n, n).cpu().numpy().T)
    ws.close()
    del p
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    A, _, _, _ = O.matgen(n, seed)
    info = Bk.panel_lu(A, b, form, trsm=trsm, inv_tc=1024)
    t_orc = time.perf_counter() - t0
    res = {"arm": arm, "n": n, "b": b, "seed": seed, "oracle_info": info, "gpu_lu_ms": st["ms_total"],
           "gpu_wall_s": t_gpu, "oracle_s": t_orc, "host_threads": O.lib().orc_num_threads()}
    res.update(compare(got, A))
    res["pass_1e-3"] = bool(info == 0 and res["rel_fro_all"] <= 1e-3 and res["rel_fro_low"] <= 1e-3
                            and res["rel_fro_up"] <= 1e-3)
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--n", type=int, default=61440)
    ap.add_argument("--b", type=int, default=2560)
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--arm", action="append", choices=list(ARMS))
    args = ap.parse_args(argv)
    ok = True
    for arm in args.arm or ["fp16_split"]:
        r = run(args, arm)
        ok = ok and r["pass_1e-3"]
        print(json.dumps(r), flush=True)
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
