"""Field files in the reference's restart format (record_out, FOU3D.f90:2172-2340, read by
read_in, start.f90:2251-2420).

One file per field (u1, u2, u3, p), Fortran unformatted sequential records, each framed by
its byte length as a 4-byte little-endian integer before and after:

  1. t, Re, alp, bet, mpgx (float64), nband, iter (int32), 88 int32 zeros
  2. N(4, 0:nband+1) (int32, Fortran order)
  3. y, dthetavi, dthdy of the field's grid (float64; u1, u3 and p carry yu/dthdyu, u2 yv/dthdyv)
  4. one record per plane j of the grid, bottom to top:
       j, field number (1 u1, 2 u2, 3 u3, 4 p), nx = N1+2, nz = N2 (int32), y(j) (float64),
       buff(nx, nz) (float64): the spectral plane with the dealiasing gap removed (u_to_buff,
       FOU3D.f90:2598-2624), i.e. row q holds kz mode q and entries 2m, 2m+1 the kx mode m —
       exactly one plane of a field in column order, interleaved re/im.
     The p file writes yu(j) beside every p plane, as record_out does.

Only single-band files (every plane N1+2 by N2) are accepted, the configuration of the GPU
path.  dthetavi is written as 0: the reference never assigns it (declaration.f90:72).
"""
from __future__ import annotations

import os
import struct

import numpy as np

FIELDS = (("u1", 1), ("u2", 2), ("u3", 3), ("p", 4))


def _rec(f, payload: bytes):
    n = struct.pack("<i", len(payload))
    f.write(n)
    f.write(payload)
    f.write(n)


def _read_rec(f) -> bytes:
    head = f.read(4)
    if len(head) < 4:
        raise EOFError
    (n,) = struct.unpack("<i", head)
    data = f.read(n)
    (m,) = struct.unpack("<i", f.read(4))
    if len(data) != n or m != n:
        raise ValueError("corrupt Fortran record")
    return data


def band_array(setup, nband: int = 3, jband: int | None = None) -> np.ndarray:
    """N(4, 0:nband+1) of a single-band run, as a (4, nband+2) int32 array [row][band]:
    rows 1-2 hold the dealiased N1, N2 of bands 1..nband, rows 3-4 the band plane limits of
    y_grid_canopy.f90:248-274.  nband = 3: the bottom band ends at v plane jband (default a
    third of the way up) and the top band mirrors it; nband = 1: one band for every plane."""
    if nband not in (1, 3):
        raise ValueError("nband must be 1 or 3")
    cfg, g = setup.cfg, setup.grid
    dny = -g.jv0
    nn = cfg.ny - 2
    N = np.zeros((4, nband + 2), dtype=np.int32)
    N[0, 1:nband + 1], N[1, 1:nband + 1] = cfg.n1, cfg.n2
    N[2, 0] = N[3, 0] = -dny
    if nband == 1:
        N[2, 1] = nn + dny
        N[3, 1] = nn + dny + 1
    else:
        if jband is None:
            jband = (nn + 2 * dny) // 3 - dny
        N[2, 1], N[2, 2], N[2, 3] = jband, nn - jband, nn + dny
        N[3, 1], N[3, 2], N[3, 3] = jband + 1, nn - jband, nn + dny + 1
    return N


def write_record_out(directory: str, tag: str, state: dict, setup, t: float = 0.0, it: int = 0,
                     mpgx: float | None = None, N: np.ndarray | None = None, nband: int = 3) -> list:
    """Write u1_<tag>.dat, u2_<tag>.dat, u3_<tag>.dat, p_<tag>.dat; state holds the spectral
    fields as (columns, planes) complex arrays (the reference's f(j,column) layout)."""
    cfg, g = setup.cfg, setup.grid
    from .bands import multiband
    if multiband(cfg):
        raise ValueError("record_out files of a three-band channel (planes of two sizes) are not written")
    if N is None:
        N = band_array(setup, nband)
    nband = N.shape[1] - 2
    nx, nz, nkx = cfg.n1 + 2, cfg.n2, cfg.nkx
    mp = cfg.mpgx if mpgx is None else mpgx
    head = struct.pack("<5d2i", t, cfg.re_b, cfg.alp, cfg.bet, mp, nband, it) + bytes(4 * 88)
    nbytes = np.asarray(N, dtype="<i4").T.tobytes()  # Fortran order: row index fastest
    paths = []
    os.makedirs(directory, exist_ok=True)
    for name, fid in FIELDS:
        y, dth, j0 = ((g.yv, g.dthdyv, g.jv0) if name == "u2" else (g.yu, g.dthdyu, g.ju0))
        f_j0 = g.jp0 if name == "p" else j0
        arr = np.asarray(state[name])
        path = os.path.join(directory, f"{name}_{tag}.dat")
        with open(path, "wb") as f:
            _rec(f, head)
            _rec(f, nbytes)
            _rec(f, np.asarray(y, "<f8").tobytes() + struct.pack("<d", 0.0) + np.asarray(dth, "<f8").tobytes())
            for jj in range(arr.shape[1]):
                j = f_j0 + jj
                plane = np.ascontiguousarray(arr[:, jj]).reshape(nz, nkx)  # [q][m]
                buff = plane.view(np.float64).reshape(nz, nx)              # (re, im) interleaved
                yj = float(g.yu[j - g.ju0])
                if name == "u2":
                    yj = float(g.yv[j - g.jv0])
                _rec(f, struct.pack("<4id", j, fid, nx, nz, yj) + buff.astype("<f8").tobytes())
        paths.append(path)
    return paths


def read_record_out(directory: str, tag: str, setup=None) -> dict:
    """Read the four files of write_record_out / the reference's record_out.  Returns the
    fields as (columns, planes) complex arrays plus "header" (t, re, alp, bet, mpgx, nband,
    iter, N, j0 per field).  With a setup, the sizes are checked against it."""
    out = {"header": {}}
    for name, fid in FIELDS:
        path = os.path.join(directory, f"{name}_{tag}.dat")
        with open(path, "rb") as f:
            h = _read_rec(f)
            t, re, alp, bet, mpgx, nband, it = struct.unpack("<5d2i", h[:48])
            nrec = _read_rec(f)
            N = np.frombuffer(nrec, "<i4").reshape(nband + 2, 4).T.copy()
            _read_rec(f)  # y, dthetavi, dthdy
            planes, js = [], []
            while True:
                try:
                    r = _read_rec(f)
                except EOFError:
                    break
                j, fno, nx, nz, _ = struct.unpack("<4id", r[:24])
                if fno != fid:
                    raise ValueError(f"{path}: plane record of field {fno}, expected {fid}")
                if nx != N[0, 1] + 2 or nz != N[1, 1]:
                    raise ValueError(f"{path}: plane {j} is {nx} x {nz}; only single-band files are read")
                buff = np.frombuffer(r[24:], "<f8").reshape(nz, nx)
                planes.append(buff.copy().view(np.complex128).reshape(-1))
                js.append(j)
        if js != list(range(js[0], js[0] + len(js))):
            raise ValueError(f"{path}: planes are not consecutive")
        out[name] = np.stack(planes, axis=1)
        out["header"].update(t=t, re=re, alp=alp, bet=bet, mpgx=mpgx, nband=nband, iter=it, N=N)
        out["header"][f"j0_{name}"] = js[0]
    if setup is not None:
        cfg, g = setup.cfg, setup.grid
        for name, n, j0 in (("u1", g.nyu, g.ju0), ("u2", g.nyv, g.jv0), ("u3", g.nyu, g.ju0), ("p", g.nyp, g.jp0)):
            if out[name].shape != (cfg.ncol, n) or out["header"][f"j0_{name}"] != j0:
                raise ValueError(f"{name}: file holds {out[name].shape} from j={out['header'][f'j0_{name}']}, "
                                 f"the channel needs {(cfg.ncol, n)} from j={j0}")
    return out


# ----------------------------------------------------------------------------------------
# Statistics file of write_stats (stats.f90:255-440): header, Ngal, both y-grids, istat,
# the 13 plane-sum profiles and, when conditional sums were taken, the 13 tile-folded
# arrays of the bottom plus mirrored top band (recvX / recvXC, :443-512).
# ----------------------------------------------------------------------------------------
STATS_ORDER = ("Um", "U2m", "Vm", "V2m", "Wm", "W2m", "Pm", "P2m", "UVm", "UWm", "VWm", "wxm", "wx2m")


def _grid_bytes(y, dthdy) -> bytes:
    """The y, dthetai, dthdy record; dthetai is never assigned by the reference
    (declaration.f90:71) and is written as 0."""
    return np.asarray(y, "<f8").tobytes() + struct.pack("<d", 0.0) + np.asarray(dthdy, "<f8").tobytes()


def write_stats(path: str, stats: dict, setup, t: float = 0.0, it: int = 0, mpgx: float | None = None,
                nband: int = 3, jband: int | None = None):
    """Write the dictionary of Channel.stats_read() as write_stats does."""
    cfg, g = setup.cfg, setup.grid
    ngal = band_array(setup, nband, jband)
    ngal[0, 1:nband + 1], ngal[1, 1:nband + 1] = cfg.ngal1, cfg.ngal2
    mp = cfg.mpgx if mpgx is None else mpgx
    with open(path, "wb") as f:
        _rec(f, struct.pack("<5d2i", t, cfg.re_b, cfg.alp, cfg.bet, mp, nband, it) + bytes(4 * 88))
        _rec(f, np.asarray(ngal, "<i4").T.tobytes())
        _rec(f, _grid_bytes(g.yu, g.dthdyu))
        _rec(f, _grid_bytes(g.yv, g.dthdyv))
        _rec(f, struct.pack("<i", int(stats["istat"])))
        for k in STATS_ORDER:
            _rec(f, np.asarray(stats[k], "<f8").tobytes())
        if stats["UmC"].size:
            for k in STATS_ORDER:
                _rec(f, np.ascontiguousarray(stats[k + "C"], "<f8").tobytes())


def read_stats(path: str, setup, dnx: int = 0, dnz: int = 0) -> dict:
    """Read a write_stats file; the conditional arrays come back as [j1][dnz][dnx]."""
    g = setup.grid
    sizes = {"U": g.nyu, "V": g.nyv, "W": g.nyu, "P": g.nyp}
    out = {}
    with open(path, "rb") as f:
        h = _read_rec(f)
        out["t"], _, _, _, out["mpgx"], nband, out["iter"] = struct.unpack("<5d2i", h[:48])
        for _ in range(3):
            _read_rec(f)
        (out["istat"],) = struct.unpack("<i", _read_rec(f))
        for k in STATS_ORDER:
            out[k] = np.frombuffer(_read_rec(f), "<f8").copy()
        for k in STATS_ORDER:
            try:
                a = np.frombuffer(_read_rec(f), "<f8").copy()
            except EOFError:
                break
            out[k + "C"] = a.reshape(-1, dnz, dnx) if dnx and dnz else a
    for k in STATS_ORDER:
        grid = "V" if k in ("Vm", "V2m", "VWm", "wxm", "wx2m") else ("P" if k.startswith("P") else "U")
        if out[k].size != sizes[grid]:
            raise ValueError(f"{path}: {k} has {out[k].size} planes, expected {sizes[grid]}")
    return out


# ----------------------------------------------------------------------------------------
# Spectra files of write_spect / recvwrspec (spectra.f90:58-182): one file per spectrum,
# header, N, both y-grids, istat and buffSP(0:N1/2, 1:N2/2+1, j) (float64, Fortran order).
# ----------------------------------------------------------------------------------------
SPECTRA_FILES = (("spU", "U"), ("spV", "V"), ("spW", "U"), ("spUV", "U"), ("spP", "P"))


def column_owner(ncol: int, nranks: int) -> np.ndarray:
    """Rank of every column of the long-column list: contiguous chunks, the remainder to the
    first ranks (start.f90:1421-1444, 1500-1510)."""
    cnt = np.full(nranks, ncol // nranks)
    cnt[: ncol - cnt.sum()] += 1
    return np.repeat(np.arange(nranks), cnt)


def fold_spectrum(sp: np.ndarray, setup, nranks: int = 2) -> np.ndarray:
    """buffSP of recvwrspec (spectra.f90:115-167) from sp(j,column) [column][plane]: the
    column (i, k) goes to (i, kk) with kk = k for k <= N2/2, N2+2-k above (the -kz modes
    onto +kz), then the i >= 1 entries are doubled.  The master's own columns are stored
    (later columns replace earlier ones) and every other rank's are added, so the fold
    depends on the rank count the run used: with one rank the -kz value replaces the +kz
    one, with two or more every owner of a +kz column is rank 0 or below its mirror's and
    the two are summed.  Returns [plane][N2/2+1][N1/2+1] (C order of buffSP(i,kk,j))."""
    cfg = setup.cfg
    nkx, n2 = cfg.nkx, cfg.n2
    ncol, ny = sp.shape
    col = np.arange(ncol)
    i, k = col % nkx, col // nkx + 1
    kk = np.where(k > n2 // 2, n2 + 2 - k, k)
    out = np.zeros((ny, n2 // 2 + 1, nkx))
    own = column_owner(ncol, nranks)
    tgt = (kk - 1) * nkx + i
    # the master's columns: the last column of each target is the one that stays
    c0 = col[own == 0][::-1]
    _, first = np.unique(tgt[c0], return_index=True)
    keep = c0[first]
    out.reshape(ny, -1)[:, tgt[keep]] = sp[keep].T
    for r in range(1, nranks):
        m = own == r
        np.add.at(out, (slice(None), kk[m] - 1, i[m]), sp[m].T)
    out[:, :, 1:] *= 2.0
    return out


def spectra_filename(name: str, setup, t: float) -> str:
    """<name>_<N1>x<N2>x<ny>_<int(10t)>.dat, the names of write_spect (spectra.f90:86-95,
    ext1..ext4 of start.f90:235-237 and FOU3D.f90:2238)."""
    cfg = setup.cfg
    return f"{name}_{cfg.n1:04d}x{cfg.n2:04d}x{cfg.ny:04d}_{int(10.0 * t):05d}.dat"


def write_spect(directory: str, spectra: dict, setup, istat: int, t: float = 0.0, it: int = 0,
                mpgx: float | None = None, nranks: int = 2, nband: int = 3) -> list:
    """Write the five files of write_spect from the dictionary of Channel.spectra_read()."""
    cfg, g = setup.cfg, setup.grid
    mp = cfg.mpgx if mpgx is None else mpgx
    N = band_array(setup, nband)
    head = struct.pack("<5d2i", t, cfg.re_b, cfg.alp, cfg.bet, mp, N.shape[1] - 2, it) + bytes(4 * 88)
    os.makedirs(directory, exist_ok=True)
    paths = []
    for name, _ in SPECTRA_FILES:
        buff = fold_spectrum(np.asarray(spectra[name]), setup, nranks)
        path = os.path.join(directory, spectra_filename(name, setup, t))
        with open(path, "wb") as f:
            _rec(f, head)
            _rec(f, np.asarray(N, "<i4").T.tobytes())
            _rec(f, _grid_bytes(g.yu, g.dthdyu))
            _rec(f, _grid_bytes(g.yv, g.dthdyv))
            _rec(f, struct.pack("<i", int(istat)))
            _rec(f, buff.astype("<f8").tobytes())
        paths.append(path)
    return paths


def read_spect(path: str) -> dict:
    """Read one write_spect file: header values, N, istat and buffSP as
    [plane][N2/2+1][N1/2+1]."""
    with open(path, "rb") as f:
        h = _read_rec(f)
        t, re, alp, bet, mpgx, nband, it = struct.unpack("<5d2i", h[:48])
        N = np.frombuffer(_read_rec(f), "<i4").reshape(nband + 2, 4).T.copy()
        _read_rec(f)
        _read_rec(f)
        (istat,) = struct.unpack("<i", _read_rec(f))
        raw = np.frombuffer(_read_rec(f), "<f8")
    nkx, nkz = N[0, 1] // 2 + 1, N[1, 1] // 2 + 1
    if raw.size % (nkx * nkz):
        raise ValueError(f"{path}: spectrum of {raw.size} values is not a whole number of {nkx} x {nkz} planes")
    return {"t": t, "re": re, "alp": alp, "bet": bet, "mpgx": mpgx, "nband": nband, "iter": it, "N": N,
            "istat": istat, "buff": raw.reshape(-1, nkz, nkx).copy()}
