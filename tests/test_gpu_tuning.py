"""Launch shapes through cfd_create_tuned / cfd_get_tuning and the autotuner: every shape
gives the same fields (FP64 to 1e-10 of the default shapes), and the tuner returns one of
the shapes it timed."""
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


SHAPES = [dict(xline_path=2), dict(xline_path=1, xline_rows=2, zlines=4), dict(xline_path=3),
          dict(xline_path=3, xline_rows=2, rhs_chunk=16),
          dict(xline_rows=4, zlines=8, solve_cols=64), dict(xsplit=2, zsplit=2, solve_cols=32)]


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_tuned_shapes_agree(torch_cuda):
    s = build_channel(tiny(96, 192, 13, cyl_diameter=0.3, cyl_spacing=1.5, seed=5))
    ref = Channel(s, device=0, precision="fp64")
    ref.upload_state()
    ref.step(2)
    base = ref.download_state()
    ref.close()
    for shape in SHAPES:
        ch = Channel(s, device=0, precision="fp64", tuning=shape)
        got = ch.tuning()
        for k, v in shape.items():
            assert got[k] == v, (shape, got)
        ch.upload_state()
        ch.step(2)
        st = ch.download_state()
        for k in st:
            assert rel(st[k], base[k]) < 1e-10, (shape, k)
        ch.close()


def test_autotune_small(torch_cuda, tmp_path, monkeypatch):
    from cfd_b200 import autotune
    monkeypatch.setenv("CFD_TUNE_CACHE", str(tmp_path / "tune.json"))
    s = build_channel(tiny(64, 96, 17, cyl_diameter=0.3, cyl_spacing=1.5, seed=3))
    best, t = autotune.autotune(s, "mixed", 0, steps=2)
    assert t > 0 and best["xline_path"] in (1, 2, 3, 4, 5, 6) and best["solve_kind"] == 1
    assert autotune.tuned(s, "mixed", 0) in (best, autotune.tuned(s, "mixed", 0))
    ch = Channel(s, device=0, precision="mixed", tuning="auto")
    assert ch.tuning() == autotune.tuned(s, "mixed", 0)
    ch.close()


def test_pair_xline_shapes(torch_cuda):
    """Line-pair x-line kernel (xline_path 4) at every row count it takes: the same state as
    the scalar FP32 path to 1e-6 after two RK3 steps (1e-5 on the pressure)."""
    s = build_channel(tiny(96, 192, 13, cyl_diameter=0.3, cyl_spacing=1.5, seed=5))
    ref = Channel(s, device=0, precision="mixed", tuning=dict(xline_path=1))
    ref.upload_state()
    ref.step(2)
    base = ref.download_state()
    ref.close()
    for rows in (2, 4, 8):
        ch = Channel(s, device=0, precision="mixed", tuning=dict(xline_path=4, xline_rows=rows))
        got = ch.tuning()
        assert got["xline_path"] == 4 and got["xline_rows"] == rows, got
        ch.upload_state()
        ch.step(2)
        st = ch.download_state()
        for k in ("u1", "u2", "u3", "p"):
            tol = 1e-5 if k == "p" else 1e-6  # the pressure is the most sensitive field
            assert rel(st[k], base[k]) < tol, (rows, k, rel(st[k], base[k]))
        ch.close()
