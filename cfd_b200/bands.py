"""Three-band resolution (start.f90:76-111, 1382-1651) on the host: which (kx,kz) columns
exist in the middle band ("long") and the y segments of each column (jlim,
start.f90:1538-1557).  The device layout and the C ABI keep the wall bands' column list for
every plane; a short column (a mode of the wall bands only) holds data in its bottom and
top segments and zero elsewhere."""
from __future__ import annotations

import numpy as np


def multiband(cfg) -> bool:
    return cfg.band_vface > 0 and ((cfg.ngal1_mid or cfg.ngal1) != cfg.ngal1 or
                                   (cfg.ngal2_mid or cfg.ngal2) != cfg.ngal2)


def long_columns(cfg) -> np.ndarray:
    """Boolean mask over the column list (column = q*nkx + i): True where the mode exists in
    the middle band (the reference's columns_long_list, start.f90:1476-1496)."""
    n1m = 2 * ((cfg.ngal1_mid or cfg.ngal1) // 3)
    n2m = 2 * ((cfg.ngal2_mid or cfg.ngal2) // 3)
    i = np.arange(cfg.ncol) % cfg.nkx
    q = np.arange(cfg.ncol) // cfg.nkx
    return (i <= n1m // 2) & ((q < n2m // 2) | (q >= cfg.n2 - n2m // 2))


def wall_planes(cfg, grid, which: str) -> np.ndarray:
    """Boolean mask over the planes of a grid ("u", "v" or "p", array index j - j0) that lie
    in a wall band's segment of the short columns (planelim/jlim, start.f90:1538-1557)."""
    jb, m = cfg.band_vface, cfg.ny - 2 - cfg.band_vface
    if which == "u":
        j = grid.ju0 + np.arange(grid.nyu)
        return (j <= jb + 2) | (j >= m)
    if which == "v":
        j = grid.jv0 + np.arange(grid.nyv)
        return (j <= jb + 1) | (j >= m)
    j = grid.jp0 + np.arange(grid.nyp)
    return (j <= jb + 1) | (j >= m + 1)


def restrict(cfg, grid, f: np.ndarray, which: str) -> np.ndarray:
    """Zero the short columns of a [column][plane] field outside their segments."""
    if not multiband(cfg):
        return f
    out = f.copy()
    short = ~long_columns(cfg)
    out[np.ix_(short, ~wall_planes(cfg, grid, which))] = 0.0
    return out
