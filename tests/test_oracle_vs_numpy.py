"""The C++ oracle against the independent numpy restatement (tests/golden/numpy_ref.py)
and against the committed golden fixtures it generated."""
import numpy as np
import pytest

from fixtures import NAMES, load
from numpy_ref import NumpyChannel
from oracle.oracle import OracleChannel

STAGES = ("rhs0", "nonlinear", "solve_uvw", "meanflow", "solve_p", "vcorr")
FIELDS = ("u1", "u2", "u3", "p", "du1", "du2", "du3", "nu1", "nu2", "nu3", "psi")


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("name", NAMES)
def test_golden_fixture(name):
    s, z = load(name)
    o = OracleChannel(s)
    o.upload_state()
    o.rk_substep(1)
    st = o.download_state()
    for k in st:
        assert rel(st[k], z["sub1_" + k]) < 1e-12, k
    o = OracleChannel(s)
    o.upload_state()
    o.step(2)
    st = o.download_state()
    for k in st:
        assert rel(st[k], z["step2_" + k]) < 1e-12, k
    assert abs(o.scalars()["mpgx"] - float(z["step2_mpgx"])) <= 1e-14 * abs(float(z["step2_mpgx"]))


@pytest.mark.parametrize("name", NAMES)
def test_stage_by_stage(name):
    s, _ = load(name)
    n = NumpyChannel(s)
    n.upload_state(s.state())
    o = OracleChannel(s)
    o.upload_state()
    for krk in (1, 2, 3):
        for stage in STAGES:
            getattr(o, stage)(krk)
            getattr(n, stage)(krk)
            for k in FIELDS:
                assert rel(o.download(k), getattr(n, k)) < 1e-12, (krk, stage, k)
