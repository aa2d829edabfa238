"""Generate the golden fixtures under tests/golden/ from the reference's own
CPU code compiled in place (oracle/_ref/libmxpref.so, built by
`make -C oracle ref` from the reference tree).

Run once, in a container that has the reference tree:
    make -C oracle && python tests/golden/make_golden.py

What is pinned (all produced by reference code, not by this repository):
  gen_n128_s42.npz   full 128 x 128 FP32 block from fill_one_panel_with_rand
                     (hpl_rand.hpp:158-198, CPU calc_diag diagonal), the RHS
                     from panel_fill_one_with_rand (hpl_rand.hpp:80-129) and
                     the CPU-order FP64 diagonal (calc_diag, hpl_rand.hpp:200-214).
  golden.json        SHA-256 of the off-diagonal FP32 matrix / RHS bytes for
                     N in {256, 1024, 2560} x seeds {42, 7, 11}; sampled
                     elements (mat_elem, hpl_rand.hpp:216-222) at the large
                     configurations N = 8192, 32768, 61440, 122880; jump-ahead
                     powers (RandCoeff::pow, hpl_rand.hpp:31-48); FP16
                     conversions through fp16sim's F16C path (fp16sim.hpp:119).
  otf_gemv_ref.npz   otf_gemv_kernel (otf_gemv.cpp:5-133) on an off-diagonal
                     block of the N = 1024, seed 42 matrix.
  sgetrf_ref.npz     sgetrf_nopiv_tuned / _naive (sgetrf_nopiv.cpp:27-61,
                     838-940) on a 96 x 96 diagonally dominant LCG block.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes(order="F")).hexdigest()


def ref_block(n, seed, calc_diag=True):
    R = O.ref()
    A = np.zeros((n, n), np.float32, order="F")
    R.ref_fill_one_panel_f32(n, 0, 0, n, n, A.ctypes.data, n, seed, int(calc_diag))
    b = np.zeros(n, np.float64)
    R.ref_panel_fill_f64(n, 0, n, n, 1, b.ctypes.data, n, seed)
    return A, b


def main() -> None:
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libmxpref.so missing: run `make -C oracle ref` with the reference tree")
    R = O.ref()
    out: dict = {"generator": "hpl_rand.hpp (reference, compiled in place)"}

    # --- full small block ---
    A, b = ref_block(128, 42)
    dcpu = np.array([R.ref_calc_diag(i, 128, 42) for i in range(128)])
    np.savez(os.path.join(HERE, "gen_n128_s42.npz"), A=A, rhs=b, d_cpu=dcpu)

    # --- hashes ---
    hashes = []
    for n in (256, 1024, 2560):
        for seed in (42, 7, 11):
            A, b = ref_block(n, seed, calc_diag=False)
            A0 = A.copy(order="F")
            np.fill_diagonal(A0, 0.0)
            hashes.append({"n": n, "seed": seed, "offdiag_f32_sha256": sha(A0),
                           "rhs_f64_sha256": sha(b)})
    out["hashes"] = hashes

    # --- sampled elements at the large configurations ---
    rng = np.random.default_rng(2024)
    samples = []
    for n, seed in ((8192, 42), (32768, 11), (61440, 42), (122880, 7)):
        idx = rng.integers(0, n, size=(48, 2))
        idx = np.vstack([idx, [[0, 1], [1, 0], [n - 1, n - 2], [n - 2, n - 1], [n // 2, n // 3]]])
        vals = [R.ref_mat_elem(n, int(i), int(j), seed) for i, j in idx]
        rhs_rows = [0, 1, n // 2, n - 1]
        rhs_vals = []
        for r in rhs_rows:
            v = np.zeros(1, np.float64)
            R.ref_panel_fill_f64(n, r, n, 1, 1, v.ctypes.data, 1, seed)
            rhs_vals.append(float(v[0]))
        samples.append({"n": n, "seed": seed, "ij": idx.tolist(),
                        "f64_hex": [float(v).hex() for v in vals],
                        "rhs_rows": rhs_rows, "rhs_f64_hex": [float(v).hex() for v in rhs_vals]})
    out["samples"] = samples

    # --- jump-ahead powers ---
    pw = []
    for e in (0, 1, 2, 3, 512, 8192, 8192 * 512, 122880 * 122880, 2**40 + 12345):
        oa = np.zeros(1, np.uint64)
        oc = np.zeros(1, np.uint64)
        R.ref_rand_pow(6364136223846793005, 1, e, oa.ctypes.data, oc.ctypes.data)
        pw.append({"e": e, "a": int(oa[0]), "c": int(oc[0])})
    out["powers"] = pw

    # --- FP16 conversions via fp16sim (F16C, round-to-nearest-even) ---
    xs = np.concatenate([
        rng.standard_normal(2000).astype(np.float32) * np.float32(3e-5),
        rng.standard_normal(2000).astype(np.float32),
        np.float32([65504.0, 65519.996, 65520.0, 1e5, 6.1035156e-05, 6.0e-05, 5.96e-08,
                    2.98e-08, 2.9802322e-08, 1e-45, 0.0, -0.0, -1.5e-7, 0.33333334]),
    ]).astype(np.float32)
    hb = np.array([R.ref_fp16_bits(float(v)) for v in xs], np.uint16)
    np.savez(os.path.join(HERE, "fp16_ref.npz"), x=xs, h=hb)

    # --- otf_gemv_kernel on an off-diagonal block ---
    n, seed = 1024, 42
    i0, j0, mb, nb = 256, 640, 64, 96
    x = rng.standard_normal(nb)
    y0 = rng.standard_normal(mb)
    y = y0.copy()
    st = O.lib().orc_state(n, seed, i0, j0)
    R.otf_gemv_kernel(n, mb, nb, -1.0, x.ctypes.data, y.ctypes.data, st)
    np.savez(os.path.join(HERE, "otf_gemv_ref.npz"), n=n, seed=seed, i0=i0, j0=j0, x=x, y0=y0, y=y)

    # --- sgetrf_nopiv on a diagonally dominant block ---
    m = 96
    A, _ = ref_block(m, 3)  # diagonal = off-diagonal row sum (calc_diag)
    At = A.copy(order="F")
    An = A.copy(order="F")
    R.ref_sgetrf_nopiv_tuned(m, At.ctypes.data, m)
    R.ref_sgetrf_nopiv_naive(m, m, An.ctypes.data, m)
    np.savez(os.path.join(HERE, "sgetrf_ref.npz"), A=A, lu_tuned=At, lu_naive=An)

    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
