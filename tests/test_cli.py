"""The `mxp` command-line driver: the reference's report layout (banner, IR
lines, summary line, "Submission Output" block) over the C ABI."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "openmxp_b200", "mxp")


def run(*args, timeout=600):
    return subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, timeout=timeout)


def test_cli_built_and_help(mxp):
    assert os.path.exists(CLI)
    r = run("--help")
    assert r.returncode == 0 and r.stdout.startswith("usage: mxp N B")


def test_cli_rejects_grids_like_the_reference(mxp):
    r = run(1024, 128, 2, 2)
    assert r.returncode == 1
    assert "OpenMxP - High Performance Mixed Precision Benchmark" in r.stdout
    assert "Can't run this grid configuration" in r.stdout
    r = run(1000, 128)
    assert r.returncode == 1 and "multiple of B" in r.stdout


def _fields(out):
    return {m.group(1).strip(): m.group(2).strip() for m in re.finditer(r"^(\w[\w()]*)\s*: (.*)$", out, re.M)}


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp16", "fp8"])
def test_cli_solves_and_reports(mxp, torch_cuda, form):
    r = run(2048, 256, 1, 1, "-form", form, "-sys", "test-box", "--job-id", "7", "-unknownflag")
    assert r.returncode == 0, r.stdout + r.stderr
    out = r.stdout
    assert "Ignoring unknown option: -unknownflag" in out
    steps = re.findall(r"# iterative refinement: step=(\d+), residual=(\S+), hpl-harness=(\S+)", out)
    assert steps and float(steps[-1][2]) < 16.0
    assert re.search(r"^\d+\.\d+ sec\. \d+\.\d+ GFlop/s resid = .* hpl-harness = .* TFlop/s per GPU = ", out, re.M)
    f = _fields(out)
    assert f["N"] == "2048" and f["NB"] == "256" and f["P"] == "1" and f["Q"] == "1"
    assert f["System"] == "test-box" and f["JobID"] == "7"
    assert float(f["HARNESS"]) < 16.0 and float(f["RESID"]) > 0.0 and float(f["GFLOPS"]) > 0.0
    assert "GEMM_UPDATE" in r.stderr and "GEMM_TOTAL" in r.stderr
