"""Statistics (stats.f90:1-253) and CFL (dtc_calc, FOU3D.f90:516-544) of the C++ oracle
against the independent numpy restatement, on a stepped tiny channel with a cylinder
lattice (CPU only)."""
import numpy as np
import pytest

from cfd_b200 import build_channel, capi
from cfd_b200.config import tiny
from cfd_b200.geometry import lattice_params
from numpy_ref import NumpyChannel
from oracle.oracle import OracleChannel

PLANE = capi.STATS_U + capi.STATS_V + capi.STATS_P
COND = tuple(n + "C" for n in PLANE)


# first moments of a field with zero plane mean (v, the fluctuating w, wx ...) are
# round-off: they are compared on the scale sqrt(points * second moment) instead
SECOND = {"Um": "U2m", "Vm": "V2m", "Wm": "W2m", "Pm": "P2m", "wxm": "wx2m"}


def close(got, ref, k, tol, npts=1):
    a, b = got[k], ref[k]
    base = k[:-1] if k.endswith("C") and k[:-1] in PLANE else k
    floor = 0.0
    if base in SECOND:
        sq = ref[SECOND[base] + ("C" if base != k else "")]
        floor = tol * np.sqrt(npts * max(np.abs(sq).max(), 0.0))
    return np.abs(a - b).max() <= tol * np.abs(b).max() + floor + 1e-300


@pytest.fixture(scope="module")
def stepped():
    s = build_channel(tiny(24, 18, 17))
    o = OracleChannel(s)
    o.upload_state()
    o.step(2)  # non-trivial p and a developed perturbation
    n = NumpyChannel(s)
    n.upload_state(o.download_state())
    _, _, dnx, dnz, *_ = lattice_params(s.cfg)
    jband = s.grid.jv0 + s.grid.nyv // 3
    return s, o, n, jband, dnx, dnz


def test_stats_oracle_vs_numpy(stepped):
    s, o, n, jband, dnx, dnz = stepped
    o.stats_configure(jband, dnx, dnz)
    o.stats_accumulate()
    got = o.stats_read()
    ref = n.stats(jband, dnx, dnz)
    assert got["istat"] == 1
    for k in PLANE + COND:
        assert got[k].shape == ref[k].shape, k
        assert close(got, ref, k, 1e-11, s.cfg.ngal1 * s.cfg.ngal2), k
    # the top band is mirrored: the wall v plane carries v = 0, the ghost u plane its
    # extrapolation; conditional sums are non-trivial on both sides
    assert np.abs(got["UmC"]).max() > 0 and np.abs(got["wx2mC"]).max() > 0


def test_stats_accumulate_and_reset(stepped):
    s, o, n, jband, dnx, dnz = stepped
    o.stats_configure(jband, dnx, dnz)
    o.stats_accumulate()
    one = o.stats_read()
    o.stats_accumulate()
    two = o.stats_read()
    assert two["istat"] == 2
    dbl = {k: 2 * one[k] for k in PLANE + COND}
    for k in PLANE + COND:
        assert close(two, dbl, k, 1e-13, s.cfg.ngal1 * s.cfg.ngal2), k
    o.stats_configure(jband, dnx, dnz)
    z = o.stats_read()
    assert z["istat"] == 0 and all(not np.any(z[k]) for k in PLANE + COND)


def test_stats_without_band(stepped):
    s, o, n, jband, dnx, dnz = stepped
    o.stats_configure(s.grid.jv0 - 1, 0, 0)
    o.stats_accumulate()
    got = o.stats_read()
    ref = n.stats(jband, dnx, dnz)
    for k in PLANE:
        assert close(got, ref, k, 1e-11, s.cfg.ngal1 * s.cfg.ngal2), k
    assert got["UmC"].size == 0


def test_cfl_oracle_vs_numpy(stepped):
    s, o, n, *_ = stepped
    dtc, t = o.cfl()
    dtn, tn = n.cfl()
    assert np.allclose(t, tn, rtol=1e-12)
    assert dtc == min(t[0], t[1]) and abs(dtc - dtn) <= 1e-12 * dtn
    # the step the setup chose is CFL-stable for this state
    assert s.dt < dtc


def test_spectra_oracle_vs_numpy(stepped):
    """spectra (spectra.f90:1-56) of the oracle: one call equals the numpy restatement,
    two calls double it, a configuration without spectra holds none."""
    s, o, n, jband, dnx, dnz = stepped
    o.stats_configure(jband, dnx, dnz)
    o.stats_accumulate()
    one = o.spectra_read()
    ref = n.spectra()
    for k in capi.SPECTRA:
        assert one[k].shape == ref[k].shape, k
        scale = np.abs(ref[k]).max()
        assert scale > 0 and np.abs(one[k] - ref[k]).max() <= 1e-13 * scale, k
    # |.|^2 spectra are exact in the accumulation order of buildsp
    assert np.array_equal(one["spU"], (o.download_state()["u1"].real ** 2) + o.download_state()["u1"].imag ** 2)
    o.stats_accumulate()
    two = o.spectra_read()
    for k in capi.SPECTRA:
        assert np.abs(two[k] - 2 * one[k]).max() <= 1e-15 * np.abs(one[k]).max(), k
    o.stats_configure(jband, dnx, dnz, spectra=False)
    o.stats_accumulate()
    with pytest.raises(AssertionError):
        o.spectra_read()
