"""Three-band resolution on the GPU (start.f90:76-111): the wall bands at Ngal1 x Ngal2, a
coarser middle band, the short columns solved per wall band with the band-interface rows,
every plane transformed at its band's size.  Against the oracle doing the same: stage by
stage in FP64 (1e-11 relative L2 on every field), 10 RK3 steps in FP64 (1e-10) and in
FP32-mixed (1e-5 on u, v, w and p); the one-band-only entry points refuse."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STAGES = ("rhs0", "nonlinear", "solve_uvw", "meanflow", "solve_p", "vcorr")
FIELDS = ("u1", "u2", "u3", "p", "du1", "du2", "du3", "nu1", "nu2", "nu3", "psi")
CASES = [dict(ngal1=48, ngal2=96, ny=33, band_vface=6, ngal1_mid=24, ngal2_mid=64),
         dict(ngal1=96, ngal2=96, ny=29, band_vface=5, ngal1_mid=64, ngal2_mid=64, flag_ctpress=0, qxt=2.0)]


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def setup_of(kw):
    from cfd_b200.channel import build_channel
    from cfd_b200.config import tiny
    base = dict(cyl_diameter=0.3, cyl_spacing=1.5, seed=9)
    base.update(kw)
    return build_channel(tiny(**base))


@pytest.mark.parametrize("kw", CASES)
def test_stages_fp64(torch_cuda, kw):
    from cfd_b200.channel import Channel
    from oracle.oracle import OracleChannel
    s = setup_of(kw)
    g = Channel(s, device=0, precision="fp64")
    g.upload_state()
    o = OracleChannel(s)
    o.upload_state()
    for krk in (1, 2, 3):
        for stage in STAGES:
            getattr(g, stage)(krk)
            getattr(o, stage)(krk)
            for k in FIELDS:
                e = rel(g.download(k), o.download(k))
                assert e < 1e-11, (krk, stage, k, e)
    g.close()


@pytest.mark.parametrize("kw", CASES)
def test_ten_steps(torch_cuda, kw):
    from cfd_b200.bands import long_columns, wall_planes
    from cfd_b200.channel import Channel
    from oracle.oracle import OracleChannel
    s = setup_of(kw)
    o = OracleChannel(s)
    o.upload_state()
    o.step(10)
    ref = o.download_state()
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-5)):
        g = Channel(s, device=0, precision=prec)
        g.upload_state()
        g.step(10)
        st = g.download_state()
        for k in ("u1", "u2", "u3", "p"):
            assert rel(st[k], ref[k]) < tol, (prec, k, rel(st[k], ref[k]))
        if prec == "fp64":
            assert g.divergence_max() < 1e-11
            short = ~long_columns(s.cfg)
            assert np.abs(st["u1"][np.ix_(short, ~wall_planes(s.cfg, s.grid, "u"))]).max() == 0.0
        g.close()


def test_one_band_entry_points_refuse(torch_cuda):
    from cfd_b200.channel import Channel
    s = setup_of(CASES[0])
    g = Channel(s, device=0, precision="fp64")
    g.upload_state()
    with pytest.raises(RuntimeError, match="three-band"):
        g.stats_configure(s.grid.jv0 - 1, 0, 0)
    with pytest.raises(RuntimeError, match="three-band"):
        g.cfl()
    with pytest.raises(RuntimeError, match="one band"):
        g.set_lastplane(True)
    g.close()
