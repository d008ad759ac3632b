"""GPU statistics (cfd_stats_*) and CFL (cfd_cfl) against the FP64 oracle on the same state.

The statistics pass is FP64 in both precisions, so both contexts must match the oracle to
round-off (1e-10 of each sum's scale; zero-mean first moments on sqrt(points * second
moment)), after one and after several accumulations.
"""
import numpy as np
import pytest

from cfd_b200 import build_channel, capi
from cfd_b200.config import tiny
from cfd_b200.geometry import lattice_params

pytestmark = pytest.mark.gpu

PLANE = capi.STATS_U + capi.STATS_V + capi.STATS_P
COND = tuple(n + "C" for n in PLANE)
SECOND = {"Um": "U2m", "Vm": "V2m", "Wm": "W2m", "Pm": "P2m", "wxm": "wx2m"}


def close(got, ref, k, tol, npts):
    a, b = got[k], ref[k]
    base = k[:-1] if k.endswith("C") and k[:-1] in PLANE else k
    floor = 0.0
    if base in SECOND:
        floor = tol * np.sqrt(npts * np.abs(ref[SECOND[base] + ("C" if base != k else "")]).max())
    return np.abs(a - b).max() <= tol * np.abs(b).max() + floor + 1e-300


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def stepped(cfg, nsteps=2):
    from oracle.oracle import OracleChannel
    s = build_channel(cfg)
    o = OracleChannel(s)
    o.upload_state()
    o.step(nsteps)
    return s, o


CASES = [tiny(24, 18, 17), tiny(96, 64, 21, cyl_diameter=0.3, cyl_spacing=1.0)]


@pytest.mark.parametrize("cfg", CASES, ids=lambda c: c.name)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_stats_vs_oracle(torch_cuda, cfg, precision):
    from cfd_b200.channel import Channel
    s, o = stepped(cfg)
    _, _, dnx, dnz, *_ = lattice_params(s.cfg)
    jband = s.grid.jv0 + s.grid.nyv // 3
    g = Channel(s, device=0, precision=precision)
    g.upload_state(o.download_state())
    npts = s.cfg.ngal1 * s.cfg.ngal2
    for ch in (g, o):
        ch.stats_configure(jband, dnx, dnz)
    for n in (1, 3):
        while o.stats_read()["istat"] < n:
            g.stats_accumulate()
            o.stats_accumulate()
        got, ref = g.stats_read(), o.stats_read()
        assert got["istat"] == ref["istat"] == n
        for k in PLANE + COND:
            assert got[k].shape == ref[k].shape, k
            assert close(got, ref, k, 1e-10, npts), (n, k)
    g.stats_reset()
    z = g.stats_read()
    assert z["istat"] == 0 and not any(np.any(z[k]) for k in PLANE + COND)
    g.close()


@pytest.mark.parametrize("cfg", CASES, ids=lambda c: c.name)
def test_cfl_vs_oracle(torch_cuda, cfg):
    from cfd_b200.channel import Channel
    s, o = stepped(cfg)
    g = Channel(s, device=0, precision="fp64")
    g.upload_state(o.download_state())
    dtc, t = g.cfl()
    dto, to = o.cfl()
    assert np.allclose(t, to, rtol=1e-11), (t, to)
    assert dtc == min(t[0], t[1]) and abs(dtc - dto) <= 1e-11 * dto
    g.close()


def test_stats_bad_tile(torch_cuda):
    from cfd_b200.channel import Channel
    s = build_channel(tiny(24, 18, 17))
    g = Channel(s, device=0)
    g.upload_state()
    with pytest.raises(RuntimeError, match="tile"):
        g.stats_configure(s.grid.jv0 + 3, 5, 3)
    with pytest.raises(RuntimeError, match="not configured"):
        g.stats_accumulate()
    g.close()


def test_set_dt_recaptures_graph(torch_cuda):
    """A CFL-driven dt change between graph replays: 1 step at dt, 2 steps at 0.8 dt,
    against the oracle doing the same (FP64 path, 1e-10 relative L2)."""
    from cfd_b200.channel import Channel
    from oracle.oracle import OracleChannel
    s = build_channel(tiny(24, 18, 17))
    g = Channel(s, device=0, precision="fp64")
    o = OracleChannel(s)
    for ch in (g, o):
        ch.upload_state()
        ch.step(1)
    dtc, _ = g.cfl()
    new = min(0.8 * s.dt, 0.5 * dtc)
    for ch in (g, o):
        ch.set_dt(new)
        ch.step(2)
    a, b = g.download_state(), o.download_state()
    for k in a:
        assert np.linalg.norm(a[k] - b[k]) <= 1e-10 * np.linalg.norm(b[k]), k
    with pytest.raises(RuntimeError, match="dt"):
        g.set_dt(-1.0)
    g.close()


@pytest.mark.parametrize("cfg", CASES, ids=lambda c: c.name)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_spectra_vs_oracle(torch_cuda, cfg, precision):
    """spectra (spectra.f90:1-56) accumulated with the statistics: the |.|^2 spectra are
    bit-exact against the oracle (same FP64 state, same order of additions), spUV within
    1e-13 of its scale (interp_v weights rounded differently); reset zeroes them; the
    write_spect files of both are the same to that tolerance."""
    from cfd_b200.channel import Channel
    from cfd_b200.checkpoint import fold_spectrum
    s, o = stepped(cfg)
    g = Channel(s, device=0, precision=precision)
    g.upload_state(o.download_state())
    for ch in (g, o):
        ch.stats_configure(s.grid.jv0 - 1, 0, 0)
        ch.stats_accumulate()
        ch.stats_accumulate()
    got, ref = g.spectra_read(), o.spectra_read()
    for k in capi.SPECTRA:
        assert got[k].shape == ref[k].shape, k
        if k == "spUV":
            assert np.abs(got[k] - ref[k]).max() <= 1e-13 * np.abs(ref[k]).max(), k
        else:
            assert np.array_equal(got[k], ref[k]), k
        fg, fo = fold_spectrum(got[k], s), fold_spectrum(ref[k], s)
        assert np.abs(fg - fo).max() <= 1e-13 * np.abs(fo).max(), k
    g.stats_reset()
    z = g.spectra_read()
    assert not any(np.any(z[k]) for k in capi.SPECTRA)
    g.stats_configure(s.grid.jv0 - 1, 0, 0, spectra=False)
    with pytest.raises(RuntimeError, match="spectra not configured"):
        g.spectra_read()
    g.close()


def test_nonfinite_watchdog(torch_cuda):
    """A NaN planted in one interior spectral coefficient of u (host data, no GPU fault):
    the CFL query reports CFD_ERR_NONFINITE at once, and after one RK3 step the mean-mode
    scalars and the divergence do; a clean context is unaffected."""
    from cfd_b200.channel import Channel
    s = build_channel(tiny(24, 18, 17))
    st = s.state()
    bad = {k: v.copy() for k, v in st.items()}
    bad["u1"][5, s.grid.nyu // 2] = complex(np.nan, 0.0)
    for prec in ("fp64", "mixed"):
        g = Channel(s, device=0, precision=prec)
        g.upload_state(st)
        g.step(1)
        g.cfl()
        g.scalars()
        g.upload_state(bad)
        with pytest.raises(RuntimeError, match="CFD_ERR_NONFINITE|non-finite"):
            g.cfl()
        g.step(1)
        with pytest.raises(RuntimeError, match="CFD_ERR_NONFINITE|non-finite"):
            g.scalars()
        with pytest.raises(RuntimeError, match="CFD_ERR_NONFINITE|non-finite"):
            g.divergence_max()
        g.close()
