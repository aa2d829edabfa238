"""Build libmxp.so (the CUDA kernels + C ABI) in-tree for sm_100a with nvcc.

    python -m openmxp_b200.build            # or openmxp_b200.build.build()

Objects go to _build/ at the repository root; the shared library lands next
to this file (openmxp_b200/libmxp.so) so it travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libmxp.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(src: str, extra: list[str]) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    deps = [src] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    deps.append(os.path.join(ROOT, "include", "mxp.h"))
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        tmp = LIB + ".tmp"
        cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart_static", "-ldl", "-lpthread", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    build_cli()
    if verbose:
        print("built", LIB)
    return LIB


CLI_SRC = os.path.join(PKG, "cli", "mxp_main.cpp")
CLI = os.path.join(PKG, "mxp")


def build_cli() -> str:
    """The `mxp` command-line driver (C++ over the C ABI), linked to libmxp.so."""
    deps = [CLI_SRC, LIB, os.path.join(ROOT, "include", "mxp.h")]
    if os.path.exists(CLI) and all(os.path.getmtime(CLI) >= os.path.getmtime(d) for d in deps):
        return CLI
    cmd = [nvcc(), "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), CLI_SRC, "-o", CLI + ".tmp",
           "-L", PKG, "-lmxp", "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN", "-lcudart_static", "-ldl",
           "-lpthread", "-lrt"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"CLI build failed:\n{r.stdout}\n{r.stderr}")
    os.replace(CLI + ".tmp", CLI)
    return CLI


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
