"""The pruned first stage of the register DFTs (rdft_z, cfd_b200/csrc/fft_reg.cuh) against
the unpruned one (rdft) for every production two-step length and both of its splits (the
cfd_tuning xsplit/zsplit radix orders), on the CPU.

tests/fft_prune_check.cu includes the header, is compiled by nvcc as host code (no GPU is
needed) and compares the two element by element for the masks gap_blocks<N1, N2, N/3>
the x-line kernel uses: the values must be equal; a zero may differ in its sign only.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _nvcc():
    for p in (os.environ.get("CUDA_HOME", ""), "/usr/local/cuda"):
        c = os.path.join(p, "bin", "nvcc") if p else ""
        if c and os.path.exists(c):
            return c
    return shutil.which("nvcc")


def test_rdft_z_matches_rdft(tmp_path):
    nvcc = _nvcc()
    if not nvcc:
        pytest.skip("nvcc not available")
    exe = str(tmp_path / "fft_prune_check")
    subprocess.run([nvcc, "-O2", "-std=c++17", "-o", exe, os.path.join(HERE, "fft_prune_check.cu")],
                   check=True, capture_output=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines[-1] == "OK"
    # every production length in both splits, both signs, both precisions
    assert len(lines) == 1 + 12 * 2 * 2
    # the masks are not empty for the lengths the pruning is for (N1 a multiple of 4)
    cases = [ln for ln in lines if "(" in ln]
    assert all("mask=0 " not in ln for ln in cases if ln.split("(")[1].split("x")[0] in ("16", "24", "32"))
