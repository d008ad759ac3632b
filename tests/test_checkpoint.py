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
