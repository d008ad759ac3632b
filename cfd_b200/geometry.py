"""Immersed-boundary point lists of a lattice of vertical cylinders (host set-up).

The hot path consumes the lists in the reference's format (f_list_ib_u(9,n) /
w_list_ib_u(3,n), start.f90:1133-1145): for every point ``(i,k,j)`` the two fluid
neighbours ``(i2,k2,j2)``, ``(i3,k3,j3)`` and the weights ``Lap, w2, w3`` of the mixed
forcing ``rhs(p) = Lap*(w2*u(p2) + w3*u(p3) - u(p) + rhs(p))``
(tridLU_3D_IB.f90:193-211).

This generator follows the classification of geom_circ_rough_mixed_forcing_24pt.f90:

* one tile of ``dnx x dnz`` points holds a circle of radius ``r`` (grid units) about
  ``(c_i, c_k)`` (:94-150); points strictly inside with an outside 4-neighbour are
  forcing points with the ``lin_interp`` weights (:634-738); when a weight is below -1
  the point is solid and its outside neighbour is forced instead (:175-192); other
  inside points and points on the circle are solid (Lap = 0) (:202-214);
* the pattern is extruded over the canopy planes, the plane next to the crest forcing
  every point with Lap = 1 (:288-494), tiled with the z-stagger of odd tile rows
  (:496-576) and sorted by (j,k,i) (:578-606).

Deliberate differences (the reference's generator cannot build the lattices of the named
workloads): the four hard-coded extra points (:219-259) are not added; a circle that
does not contain a grid point (sub-cell cylinder) collapses to one solid point at the
grid point nearest its centre; a point at the exact circle centre is solid (lin_interp
divides by zero there); tile counts are the divisors of Ngal nearest to L/spacing; the
radius in grid units uses the geometric mean of dx and dz (the reference's circle lives
in index space).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class IBList:
    idx: np.ndarray   # int32 [n, 9]
    w: np.ndarray     # float64 [n, 3]
    jlo: tuple        # (bottom, top)
    jhi: tuple

    @property
    def n(self) -> int:
        return int(self.idx.shape[0])


def _circ(x, z, r, ci, ck):
    return (x - ci) ** 2 + (z - ck) ** 2 - r ** 2


def _sign(v):
    return 1 if v > 0 else -1


def lin_interp(i, k, r, ci, ck):
    """Restates lin_interp (geom_circ_rough_mixed_forcing_24pt.f90:634-738).
    Returns (z2, x2, z3, x3), (w2, w3)."""
    i = float(i)
    k = float(k)
    aa = 1.0 if i >= ci else -1.0
    d = math.sqrt((k - ck) ** 2 + (i - ci) ** 2)
    zb = ck + (k - ck) * r / d
    xb = aa * math.sqrt(max(r * r - (zb - ck) ** 2, 0.0)) + ci
    nn = math.sqrt((zb - ck) ** 2 + (xb - ci) ** 2)
    n_z = (zb - ck) / nn
    n_x = (xb - ci) / nn
    if i == ci:
        xb = ci
        nzs = _sign(n_z)
        z2, x2, z3, x3 = int(k) + nzs, int(i), int(k) + nzs, int(i)
        return (z2, x2, z3, x3), ((k - zb) / (z2 - zb), 0.0)
    if k == ck:
        nxs = _sign(n_x)
        z2, x2, z3, x3 = int(k), int(i) + nxs, int(k), int(i) + nxs
        return (z2, x2, z3, x3), ((i - xb) / (x2 - xb), 0.0)
    nzs = _sign(n_z)
    nxs = _sign(n_x)
    if abs(i - ci) == abs(k - ck):
        z2, x2, z3, x3 = int(k) + nzs, int(i), int(k), int(i) + nxs
    elif abs(n_x) < abs(n_z):
        z2, x2, z3, x3 = int(k) + nzs, int(i), int(k) + nzs, int(i) + nxs
    else:
        z2, x2, z3, x3 = int(k), int(i) + nxs, int(k) + nzs, int(i) + nxs
    den = xb * z2 - x2 * zb - xb * z3 + x3 * zb + x2 * z3 - x3 * z2
    w2 = -(xb * z3 - x3 * zb - xb * k + i * zb + x3 * k - i * z3) / den
    w3 = (xb * z2 - x2 * zb - xb * k + i * zb + x2 * k - i * z2) / den
    return (z2, x2, z3, x3), (w2, w3)


def tile_pattern(dnx: int, dnz: int, r: float, ci: float, ck: float):
    """Points of one tile: list of (i, k, i2, k2, i3, k3, w2, w3, lap), 1-based, wrapped
    into the tile (add_forcing_point / add_solid_point, :741-788)."""

    def wrap(a, n):
        return 1 + int(math.fmod(a - 1.0 + n, float(n)))

    def solid(i, k):
        return (wrap(i, dnx), wrap(k, dnz), wrap(i, dnx), wrap(k, dnz),
                wrap(i, dnx), wrap(k, dnz), 0.0, 0.0, 0.0)

    def forcing(i, k, interpp, wei):
        z2, x2, z3, x3 = interpp
        return (wrap(i, dnx), wrap(k, dnz), wrap(x2, dnx), wrap(z2, dnz),
                wrap(x3, dnx), wrap(z3, dnz), float(wei[0]), float(wei[1]), 1.0)

    x1, x2b = math.floor(ci - r - 1), math.ceil(ci + r + 1)
    z1, z2b = math.floor(ck - r - 1), math.ceil(ck + r + 1)
    inside_any = any(_circ(i, k, r, ci, ck) < 0 for k in range(z1 + 1, z2b)
                     for i in range(x1 + 1, x2b))
    if not inside_any:
        # sub-cell cylinder: one solid point at the nearest grid point
        return [solid(int(round(ci)), int(round(ck)))]
    if x1 < 1 or z1 < 1 or x2b > dnx or z2b > dnz:
        raise ValueError(f"cylinder r={r:.3f} does not fit a {dnx}x{dnz} tile")

    pts = []
    for k in range(z1 + 1, z2b):
        for i in range(x1 + 1, x2b):
            t = _circ(i, k, r, ci, ck)
            if t < 0:
                out = (_circ(i - 1, k, r, ci, ck) > 0 or _circ(i + 1, k, r, ci, ck) > 0 or
                       _circ(i, k + 1, r, ci, ck) > 0 or _circ(i, k - 1, r, ci, ck) > 0)
                if out and not (i == ci and k == ck):
                    interpp, wei = lin_interp(i, k, r, ci, ck)
                    if wei[0] < -1.0 or wei[1] < -1.0:
                        pts.append(solid(i, k))
                        io, ko = interpp[1], interpp[0]
                        interpp2, wei2 = lin_interp(io, ko, r, ci, ck)
                        pts.append(forcing(io, ko, interpp2, wei2))
                    else:
                        pts.append(forcing(i, k, interpp, wei))
                else:
                    pts.append(solid(i, k))
            if t == 0:
                pts.append(solid(i, k))
    return pts


def _nearest_divisor(n: int, target: float, even: bool) -> int:
    divs = [d for d in range(1, n + 1) if n % d == 0 and (not even or d % 2 == 0)]
    return min(divs, key=lambda d: (abs(d - target), d))


def _fits(n: int, r: float, c: float) -> bool:
    """The circle and its interpolation stencil (one point beyond it) stay in the tile."""
    return math.floor(c - r - 1) >= 1 and math.ceil(c + r + 1) <= n


def lattice_params(cfg):
    """Tile counts and circle of the cylinder lattice of a ChannelConfig.  The counts are the
    valid divisors nearest to Lx/spacing, Lz/spacing; where a tile that small cannot hold a
    resolved circle with its stencil, the count drops to the next divisor that can (the
    reference stops there instead, geom_circ_rough_mixed_forcing_24pt.f90:81-92, 132-140)."""
    dx, dz = cfg.lx / cfg.ngal1, cfg.lz / cfg.ngal2
    r = 0.5 * cfg.cyl_diameter / math.sqrt(dx * dz)
    ntilex = _nearest_divisor(cfg.ngal1, cfg.lx / cfg.cyl_spacing, even=True)
    ntilez = _nearest_divisor(cfg.ngal2, cfg.lz / cfg.cyl_spacing, even=False)

    def resolved(dnx, dnz):
        ci, ck = (dnx + 1) / 2.0, (dnz + 1) / 2.0
        return any(_circ(i, k, r, ci, ck) < 0 for k in range(math.floor(ck - r), math.ceil(ck + r) + 1)
                   for i in range(math.floor(ci - r), math.ceil(ci + r) + 1))

    def smaller(n, cur, even):
        divs = [d for d in range(1, cur) if n % d == 0 and (not even or d % 2 == 0)]
        return max(divs) if divs else cur

    while True:
        dnx, dnz = cfg.ngal1 // ntilex, cfg.ngal2 // ntilez
        ci, ck = (dnx + 1) / 2.0, (dnz + 1) / 2.0
        if not resolved(dnx, dnz) or (_fits(dnx, r, ci) and _fits(dnz, r, ck)):
            break
        nx = ntilex if _fits(dnx, r, ci) else smaller(cfg.ngal1, ntilex, True)
        nz = ntilez if _fits(dnz, r, ck) else smaller(cfg.ngal2, ntilez, False)
        if (nx, nz) == (ntilex, ntilez):
            break
        ntilex, ntilez = nx, nz
    return ntilex, ntilez, dnx, dnz, r, (dnx + 1) / 2.0, (dnz + 1) / 2.0


def ib_lists(cfg, grid):
    """(u-list, v-list) of the lattice for every canopy plane of both walls."""
    dny = grid.dny
    empty_u = IBList(np.zeros((0, 9), np.int32), np.zeros((0, 3)), (0, 0), (-1, -1))
    if dny == 0 or cfg.cyl_diameter <= 0 or cfg.posth <= 0:
        return empty_u, IBList(empty_u.idx, empty_u.w, (0, 0), (-1, -1))
    ntilex, ntilez, dnx, dnz, r, ci, ck = lattice_params(cfg)
    pat = tile_pattern(dnx, dnz, r, ci, ck)

    ny = cfg.ny
    # plane ranges (geom_circ_rough_mixed_forcing_24pt.f90:58-67 with Ngal(4,3) = ny+dny-1,
    # Ngal(3,3) = ny+dny-2)
    nyu11, nyu21 = -dny + 1, 0
    nyv11, nyv21 = -dny + 1, -1
    nyu12, nyu22 = ny, ny + dny - 1
    nyv12, nyv22 = ny, ny + dny - 2

    def extrude(planes_xz, tip_plane, first_tip):
        rows = []
        for j in planes_xz:
            for (i, k, i2, k2, i3, k3, w2, w3, lap) in pat:
                rows.append((i, k, j, i2, k2, j, i3, k3, j, lap, w2, w3))
        if tip_plane is not None:
            for (i, k, i2, k2, i3, k3, w2, w3, lap) in pat:
                rows.append((i, k, tip_plane, i2, k2, tip_plane, i3, k3, tip_plane, 1.0, w2, w3))
        return rows

    def tile(rows):
        out = []
        for ix in range(1, ntilex + 1):
            for iz in range(1, ntilez + 1):
                sh = dnz * (iz - 1) + ((ix + 1) % 2) * dnz * cfg.stagger - 1.0
                for (i, k, j, i2, k2, j2, i3, k3, j3, lap, w2, w3) in rows:
                    def kk(kv):
                        return 1 + int(math.fmod(kv + sh, float(cfg.ngal2)))
                    out.append((i + dnx * (ix - 1), kk(k), j, i2 + dnx * (ix - 1), kk(k2), j2,
                                i3 + dnx * (ix - 1), kk(k3), j3, lap, w2, w3))
        return out

    def finish(rows, jlo, jhi):
        # a point is only forced when its plane lies in a round-trip range
        # (getbounds distributes list points by plane, start.f90:1112-1126)
        rows = [r_ for r_ in rows if any(jlo[s] <= r_[2] <= jhi[s] for s in (0, 1))]
        if not rows:
            return IBList(np.zeros((0, 9), np.int32), np.zeros((0, 3)), jlo, jhi)
        a = np.array(rows, dtype=np.float64)
        idx = a[:, :9].astype(np.int32)
        w = a[:, 9:12].copy()
        order = np.lexsort((idx[:, 0], idx[:, 1], idx[:, 2]))  # by j, then k, then i
        return IBList(np.ascontiguousarray(idx[order]), np.ascontiguousarray(w[order]), jlo, jhi)

    rows_u = tile(extrude(range(nyu11, nyu21), nyu21, True)) + \
        tile(extrude([], nyu12, True) + extrude(range(nyu12 + 1, nyu22 + 1), None, False))
    rows_v = tile(extrude(range(nyv11, nyv21), nyv21, True)) + \
        tile(extrude([], nyv12, True) + extrude(range(nyv12 + 1, nyv22 + 1), None, False))
    lu = finish(rows_u, (nyu11, nyu12), (nyu21, nyu22))
    lv = finish(rows_v, (nyv11, nyv12), (nyv21, nyv22))
    return lu, lv
