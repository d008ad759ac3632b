"""Restart through the reference's record_out files: a channel written after two steps and
read into a fresh context continues exactly as the original (FP64, identical fields)."""
import numpy as np
import pytest

from cfd_b200 import Channel, build_channel
from cfd_b200.config import tiny

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_restart_from_record_out(torch_cuda, tmp_path):
    s = build_channel(tiny(96, 64, 21, cyl_diameter=0.3, cyl_spacing=1.0, seed=9))
    a = Channel(s, device=0, precision="fp64")
    a.upload_state()
    a.step(2)
    a.save_record_out(str(tmp_path), "r", t=2 * s.dt, it=2)
    b = Channel(s, device=0, precision="fp64")
    h = b.load_record_out(str(tmp_path), "r")
    assert h["iter"] == 2
    for ch in (a, b):
        ch.step(2)
    sa, sb = a.download_state(), b.download_state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k
    a.close()
    b.close()
