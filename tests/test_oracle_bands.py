"""Three-band resolution in the oracle (start.f90:76-111, 1382-1651): the wall bands at
Ngal1 x Ngal2, the middle band coarser, the modes the middle band lacks ("short" columns)
solved per wall band with the band-interface rows of LU_buildU/V/P (CPU).

* With the middle band at the wall bands' size every column is long and every plane is
  transformed at one size, so the three-band code paths must give the one-band fields bit
  for bit.
* With a coarser middle band: the short columns stay zero outside their segments, the
  velocity is divergence-free on every column segment after each substep (solveP + v_corr
  per band), the v rows at the band interfaces are zero, and the middle band's truncation
  changes the flow (the run differs from the one-band run).
"""
import numpy as np
import pytest

from oracle.oracle import OracleChannel


def _setup(**kw):
    from cfd_b200.channel import build_channel
    from cfd_b200.config import tiny
    base = dict(ngal1=48, ngal2=36, ny=33, cyl_diameter=0.3, cyl_spacing=1.5, seed=4)
    base.update(kw)
    return build_channel(tiny(**base))


def test_equal_bands_reproduce_one_band():
    one = _setup()
    three = _setup(band_vface=6, ngal1_mid=48, ngal2_mid=36)
    a, b = OracleChannel(one), OracleChannel(three)
    for o in (a, b):
        o.upload_state(one.state())
        o.step(2)
    sa, sb = a.download_state(), b.download_state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k


@pytest.fixture(scope="module")
def banded():
    s = _setup(band_vface=6, ngal1_mid=24, ngal2_mid=18)
    o = OracleChannel(s)
    o.upload_state()
    return s, o


def test_short_columns_live_in_their_segments(banded):
    from cfd_b200.bands import long_columns, wall_planes
    s, o = banded
    short = ~long_columns(s.cfg)
    assert short.sum() > 0 and (~short).sum() > 0
    o.step(2)
    st = o.download_state()
    g = s.grid
    for k, which in (("u1", "u"), ("u3", "u"), ("u2", "v"), ("p", "p")):
        outside = ~wall_planes(s.cfg, g, which)
        assert np.abs(st[k][np.ix_(short, outside)]).max() == 0.0, k
        assert np.abs(st[k][np.ix_(short, ~outside)]).max() > 0.0, k
    # v is zero on the interface faces of the short segments (the identity rows of LU_buildV)
    jb, m = s.cfg.band_vface, s.cfg.ny - 2 - s.cfg.band_vface
    for j in (jb + 1, m):
        assert np.abs(st["u2"][short, j - g.jv0]).max() == 0.0


def test_divergence_free_per_segment(banded):
    s, o = banded
    for krk in (1, 2, 3):
        o.rk_substep(krk)
        div = o.download("div")
        u = o.download("u1")
        assert np.abs(div).max() <= 1e-11 * np.abs(u).max(), krk


def test_middle_band_truncation_acts():
    one = _setup()
    three = _setup(band_vface=6, ngal1_mid=24, ngal2_mid=18)
    a, b = OracleChannel(one), OracleChannel(three)
    a.upload_state(three.state())   # the same (band-restricted) start
    b.upload_state(three.state())
    a.step(1)
    b.step(1)
    from cfd_b200.bands import long_columns
    lc = long_columns(three.cfg)
    ua, ub = a.download("u1"), b.download("u1")
    rel = np.linalg.norm(ua[lc] - ub[lc]) / np.linalg.norm(ua[lc])
    assert 1e-8 < rel < 1e-1


def test_band_arguments_are_checked():
    from oracle import oracle as O
    s = _setup(band_vface=15, ngal1_mid=24, ngal2_mid=18)   # m = 16: no middle band
    with pytest.raises(RuntimeError, match="middle band"):
        OracleChannel(s)
    s = _setup(band_vface=6, ngal1_mid=24, ngal2_mid=18)
    o = OracleChannel(s)
    assert O.lib().orc_set_quirk(o.h, 1) == 1  # CFD_ERR_ARG
    assert O.lib().orc_stats_configure(o.h, s.grid.jv0 - 1, 0, 0, 0) == 1  # CFD_ERR_ARG


@pytest.mark.parametrize("kw", [dict(band_vface=6, ngal1_mid=24, ngal2_mid=18),
                                dict(band_vface=5, ngal1_mid=36, ngal2_mid=24, ngal1=48, ngal2=48, seed=8)])
def test_oracle_vs_numpy_blocks(kw):
    """The oracle's three-band restatement (wall-band column layout with per-column
    segments) against the numpy one built on the reference's per-band column blocks
    (tests/golden/numpy_bands.py), stage by stage over one RK3 step: 1e-12 relative L2 on
    every field."""
    from numpy_bands import NumpyBands
    s = _setup(**kw)
    n = NumpyBands(s)
    n.upload_state(s.state())
    o = OracleChannel(s)
    o.upload_state()
    fields = ("u1", "u2", "u3", "p", "du1", "du2", "du3", "nu1", "nu2", "nu3", "psi")
    for krk in (1, 2, 3):
        for stage in ("rhs0", "nonlinear", "solve_uvw", "solve_p", "vcorr"):
            getattr(o, stage)(krk)
            getattr(n, stage)(krk)
            for k in fields:
                a, b = o.download(k), n.download(k)
                e = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)
                assert e < 1e-12, (krk, stage, k, e)
