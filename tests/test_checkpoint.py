"""Field files in the reference's record_out format (cfd_b200.checkpoint): byte layout of
the Fortran records, round trip, and rejection of mismatched grids (CPU)."""
import struct

import numpy as np
import pytest

from cfd_b200 import build_channel
from cfd_b200.checkpoint import band_array, read_record_out, write_record_out
from cfd_b200.config import tiny


@pytest.fixture(scope="module")
def setup():
    return build_channel(tiny(24, 18, 17))


def test_round_trip(tmp_path, setup):
    st = setup.state()
    write_record_out(str(tmp_path), "t1", st, setup, t=1.5, it=42)
    back = read_record_out(str(tmp_path), "t1", setup)
    for k in ("u1", "u2", "u3", "p"):
        assert back[k].shape == st[k].shape
        assert np.array_equal(back[k], st[k]), k
    h = back["header"]
    assert h["t"] == 1.5 and h["iter"] == 42 and h["nband"] == 3
    assert h["N"][0, 1] == setup.cfg.n1 and h["N"][1, 1] == setup.cfg.n2
    assert h["j0_p"] == setup.grid.jp0


def test_record_layout(tmp_path, setup):
    """The bytes follow record_out: header (400 bytes), N, y record, then per plane
    j, field, nx, nz, y(j), buff(nx, nz) with buff row q = kz mode q, entries 2m, 2m+1 = kx m."""
    cfg, g = setup.cfg, setup.grid
    st = setup.state()
    write_record_out(str(tmp_path), "x", st, setup)
    raw = (tmp_path / "u2_x.dat").read_bytes()
    off = 0

    def rec():
        nonlocal off
        (n,) = struct.unpack_from("<i", raw, off)
        data = raw[off + 4: off + 4 + n]
        (m,) = struct.unpack_from("<i", raw, off + 4 + n)
        assert m == n
        off += n + 8
        return data
    assert len(rec()) == 5 * 8 + 2 * 4 + 88 * 4
    assert np.array_equal(np.frombuffer(rec(), "<i4").reshape(-1, 4).T, band_array(setup))
    assert len(rec()) == 8 * (2 * g.nyv + 1)
    r = rec()
    j, fno, nx, nz, yj = struct.unpack_from("<4id", r)
    assert (j, fno, nx, nz) == (g.jv0, 2, cfg.n1 + 2, cfg.n2) and yj == g.yv[0]
    buff = np.frombuffer(r, "<f8", offset=24).reshape(nz, nx)
    q, m = 3, 2
    col = q * cfg.nkx + m
    assert buff[q, 2 * m] == st["u2"][col, 0].real and buff[q, 2 * m + 1] == st["u2"][col, 0].imag


def test_mismatch_rejected(tmp_path, setup):
    write_record_out(str(tmp_path), "a", setup.state(), setup)
    other = build_channel(tiny(24, 18, 21))
    with pytest.raises(ValueError):
        read_record_out(str(tmp_path), "a", other)


def test_stats_file_round_trip(tmp_path):
    """write_stats layout from the oracle's statistics (the GPU gives the same dictionary)."""
    from cfd_b200.geometry import lattice_params
    from cfd_b200.checkpoint import read_stats, write_stats
    from oracle.oracle import OracleChannel
    s = build_channel(tiny(24, 18, 17))
    o = OracleChannel(s)
    o.upload_state()
    o.step(1)
    _, _, dnx, dnz, *_ = lattice_params(s.cfg)
    o.stats_configure(s.grid.jv0 + 5, dnx, dnz)
    o.stats_accumulate()
    st = o.stats_read()
    path = str(tmp_path / "stats.dat")
    write_stats(path, st, s, t=0.5, it=7)
    back = read_stats(path, s, dnx, dnz)
    assert back["istat"] == 1 and back["iter"] == 7
    for k in ("Um", "U2m", "Vm", "Pm", "wx2m", "VWm"):
        assert np.array_equal(back[k], st[k]), k
    for k in ("UmC", "V2mC", "PmC", "wx2mC"):
        assert np.array_equal(back[k], st[k]), k


def _fold_loops(sp, nkx, n2, nranks):
    """recvwrspec (spectra.f90:115-167) as the reference's loops: rank 0 stores, every
    other rank adds, in column order; then the i >= 1 entries are doubled."""
    from cfd_b200.checkpoint import column_owner
    ncol, ny = sp.shape
    own = column_owner(ncol, nranks)
    buff = np.zeros((ny, n2 // 2 + 1, nkx))
    for r in range(nranks):
        for col in np.nonzero(own == r)[0]:
            i, k = col % nkx, col // nkx + 1
            kk = n2 + 2 - k if k > n2 // 2 else k
            if r == 0:
                buff[:, kk - 1, i] = sp[col]
            else:
                buff[:, kk - 1, i] += sp[col]
    buff[:, :, 1:] *= 2.0
    return buff


@pytest.mark.parametrize("nranks", [1, 2, 3, 7])
def test_spectrum_fold(setup, nranks):
    from cfd_b200.checkpoint import column_owner, fold_spectrum
    cfg = setup.cfg
    rng = np.random.default_rng(5)
    sp = rng.random((cfg.ncol, 6))
    got = fold_spectrum(sp, setup, nranks)
    assert np.array_equal(got, _fold_loops(sp, cfg.nkx, cfg.n2, nranks))
    own = column_owner(cfg.ncol, nranks)
    assert own.size == cfg.ncol and np.all(np.diff(own) >= 0) and own[-1] == nranks - 1
    nkx, n2 = cfg.nkx, cfg.n2
    kz = lambda k: sp[(k - 1) * nkx:(k - 1) * nkx + nkx].T  # [plane][i] of the column row k
    # kz = 0 and the last row have no mirror
    assert np.array_equal(got[:, 0, 0], kz(1)[:, 0]) and np.allclose(got[:, 0, 1:], 2 * kz(1)[:, 1:])
    assert np.allclose(got[:, n2 // 2, 1:], 2 * kz(n2 // 2 + 1)[:, 1:])
    if nranks == 1:  # one rank: the -kz column replaces the +kz one
        assert np.allclose(got[:, 1, 1:], 2 * kz(n2)[:, 1:])
    else:            # more: the two are summed
        assert np.allclose(got[:, 1, 1:], 2 * (kz(2) + kz(n2))[:, 1:])


def test_spect_file_round_trip(tmp_path):
    """write_spect layout from the oracle's spectra (the GPU gives the same dictionary)."""
    from cfd_b200.checkpoint import SPECTRA_FILES, fold_spectrum, read_spect, spectra_filename, write_spect
    from oracle.oracle import OracleChannel
    s = build_channel(tiny(24, 18, 17))
    o = OracleChannel(s)
    o.upload_state()
    o.step(1)
    o.stats_configure(s.grid.jv0 - 1, 0, 0)
    o.stats_accumulate()
    o.stats_accumulate()
    sp = o.spectra_read()
    paths = write_spect(str(tmp_path), sp, s, istat=2, t=1.25, it=9)
    assert [p.split("/")[-1] for p in paths] == [spectra_filename(n, s, 1.25) for n, _ in SPECTRA_FILES]
    assert paths[0].endswith(f"spU_{s.cfg.n1:04d}x{s.cfg.n2:04d}x{s.cfg.ny:04d}_00012.dat")
    g = s.grid
    for (name, grid), path in zip(SPECTRA_FILES, paths):
        back = read_spect(path)
        assert back["istat"] == 2 and back["iter"] == 9 and back["t"] == 1.25
        ny = {"U": g.nyu, "V": g.nyv, "P": g.nyp}[grid]
        assert back["buff"].shape == (ny, s.cfg.n2 // 2 + 1, s.cfg.nkx)
        assert np.array_equal(back["buff"], fold_spectrum(sp[name], s, 2)), name
    # the record holds buffSP(0:N1/2, 1:N2/2+1, j) with i fastest
    with open(paths[0], "rb") as f:
        for _ in range(5):
            (n,) = struct.unpack("<i", f.read(4))
            f.seek(n + 4, 1)
        (n,) = struct.unpack("<i", f.read(4))
        assert n == 8 * g.nyu * (s.cfg.n2 // 2 + 1) * s.cfg.nkx
        first = struct.unpack("<2d", f.read(16))
    b = read_spect(paths[0])["buff"]
    assert first == (b[0, 0, 0], b[0, 0, 1])
