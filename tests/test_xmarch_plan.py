"""Launch geometry, thread roles and y-step sequence of the x-line pass marching in y
(cfd_b200/csrc/xmarch_plan.cuh, the functions the kernel k_xmarch computes them with), on
the CPU.

tests/xmarch_check.cu includes the header, is compiled by nvcc as host code (no GPU is
needed) and checks, for every split the kernel is built for and 2 and 4 rows per CTA, that
every shared-memory index lies in its buffer, that each work item of a phase is taken once,
that each phase reads exactly the cells the previous one wrote, the shuffle sources and the
unpack partners; and, for channel heights 4-70 and the named workloads' plane counts with
y-chunks of 2-100 steps, that every u-plane and v-plane is produced once from the planes its
y-interpolation needs.
"""
import os
import subprocess

import pytest

from test_fft_prune import _nvcc

HERE = os.path.dirname(os.path.abspath(__file__))


def test_xmarch_plan(tmp_path):
    nvcc = _nvcc()
    if not nvcc:
        pytest.skip("nvcc not available")
    exe = str(tmp_path / "xmarch_check")
    subprocess.run([nvcc, "-O2", "-std=c++17", "-Wno-deprecated-gpu-targets", "-o", exe,
                    os.path.join(HERE, "xmarch_check.cu")], check=True, capture_output=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines[-1] == "OK"
    assert sum(ln.startswith("roles ") for ln in lines) == 5 * 2
    assert int(lines[-2].split()[1]) > 700
