"""Wall-normal grid, wavenumbers and grid weights of the channel (host set-up).

The grid is host input to both the CUDA path and the oracle, so its construction cannot
break parity; it is restated here so that the synthetic workloads have the reference's
grid structure:

* ``y_grid_rough`` (y_grid_rough.f90:1-189): a polynomial map between the crests
  ``y(j) = a (j-q)^p/5 + b (j-q)^(p-2)/3 + c (j-q)`` with ``dy(centre)/dy(crest) = dyq``,
  and an almost uniform grid of ``dny = ceil(posth/dy1)`` planes inside each canopy
  (``y = -1 - posth .. -1`` and ``1 .. 1 + posth``).
* 3-point second-derivative coefficients ``dyu2i``/``dyv2i`` (y_grid_rough.f90:110-139).
* wavenumbers (start.f90:937-1018) and the ghost-point weights ``gridweighting`` /
  ``gridweighting_interp`` (start.f90:493-508) for one uniform y-band.

Index convention: arrays start at ``j = -dny``; u/w (ugrid) planes are
``-dny .. ny+dny``, v (vgrid) ``-dny .. ny+dny-1``, p (pgrid) ``-dny+1 .. ny+dny-1``.
The reference's ``y_grid_rough`` leaves ``yv(nn)``/``yu(nn+1)`` unset when ``dny == 0``
(y_grid_rough.f90:66-70); the polynomial value is used there, as ``y_grid_canopy.f90:71-76``
does.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class YGrid:
    ny: int
    dny: int
    yu: np.ndarray       # [ny + 2 dny + 1]
    yv: np.ndarray       # [ny + 2 dny]
    dthdyu: np.ndarray
    dthdyv: np.ndarray
    dyu2i: np.ndarray    # [nyu, 3]
    dyv2i: np.ndarray    # [nyv, 3]

    @property
    def ju0(self) -> int:
        return -self.dny

    @property
    def ju1(self) -> int:
        return self.ny + self.dny

    @property
    def jv0(self) -> int:
        return -self.dny

    @property
    def jv1(self) -> int:
        return self.ny + self.dny - 1

    @property
    def jp0(self) -> int:
        return -self.dny + 1

    @property
    def jp1(self) -> int:
        return self.ny + self.dny - 1

    @property
    def nyu(self) -> int:
        return self.ny + 2 * self.dny + 1

    @property
    def nyv(self) -> int:
        return self.ny + 2 * self.dny

    @property
    def nyp(self) -> int:
        return self.ny + 2 * self.dny - 1

    def u(self, j: int) -> float:
        return float(self.yu[j + self.dny])

    def v(self, j: int) -> float:
        return float(self.yv[j + self.dny])


def y_grid_rough(ny: int, dyq: float, ppp: int, posth: float) -> YGrid:
    """Restates y_grid_rough.f90:22-139 (nn = ny-1 points between crests)."""
    nn = ny - 1
    q = nn / 2.0
    aaa = 15.0 * (dyq - 1.0) / ((8.0 * dyq + 7.0) * q ** ppp)
    bbb = -30.0 * (dyq - 1.0) / ((8.0 * dyq + 7.0) * q ** (ppp - 2))
    ccc = 15.0 * dyq / ((8.0 * dyq + 7.0) * q)
    dy1 = aaa * q ** 4 + bbb * q ** 2 + ccc
    dny = int(math.ceil(posth / dy1 - 1e-12)) if posth > 0 else 0
    aab = -(posth - dy1 * dny) / (dny * (dny + 1.0)) if dny > 0 else 0.0

    nyu = nn + 2 * dny + 2
    nyv = nn + 2 * dny + 1
    yu = np.full(nyu, np.nan)
    yv = np.full(nyv, np.nan)
    dthdyu = np.full(nyu, np.nan)
    dthdyv = np.full(nyv, np.nan)
    ou = dny  # offset: array index = j + dny
    ov = dny

    def poly(s):
        return aaa * s ** ppp / 5.0 + bbb * s ** (ppp - 2) / 3.0 + ccc * s

    def dpoly(s):
        return aaa * s ** (ppp - 1) + bbb * s ** (ppp - 3) + ccc

    for j in range(0, nn):
        s, t = j - q, j + 0.5 - q
        yv[j + ov] = poly(s)
        yu[j + 1 + ou] = poly(t)
        dthdyv[j + ov] = 1.0 / dpoly(s)
        dthdyu[j + 1 + ou] = 1.0 / dpoly(t)

    if dny == 0:
        s = -0.5 - q
        yu[0 + ou] = poly(s)
        dthdyu[0 + ou] = 1.0 / dpoly(s)
        j = nn
        yv[j + ov] = poly(j - q)
        yu[j + 1 + ou] = poly(j + 0.5 - q)
        dthdyv[j + ov] = 1.0 / dpoly(j - q)
        dthdyu[j + 1 + ou] = 1.0 / dpoly(j + 0.5 - q)
    else:
        yu[-dny + ou] = -1.0 + dy1 * (-dny - 0.5) + aab * (dny ** 2 + 2.0 * dny + 0.75)
        dthdyu[-dny + ou] = 1.0 / (dy1 + 2.0 * aab * (-dny - 1.0))
        for j in range(-dny, 0):
            yv[j + ov] = -1.0 + dy1 * j + aab * (j ** 2 - j)
            yu[j + 1 + ou] = -1.0 + dy1 * (j + 0.5) + aab * (j ** 2 - 0.25)
            dthdyv[j + ov] = 1.0 / (dy1 + 2.0 * aab * (j - 0.5))
            dthdyu[j + 1 + ou] = 1.0 / (dy1 + 2.0 * aab * j)
        for j in range(0, dny + 1):
            yv[j + nn + ov] = 1.0 + dy1 * j - aab * (j ** 2 + j)
            yu[j + nn + 1 + ou] = 1.0 + dy1 * (j + 0.5) - aab * (j ** 2 + 2.0 * j + 0.75)
            dthdyv[j + nn + ov] = 1.0 / (dy1 - 2.0 * aab * (j + 0.5))
            dthdyu[j + nn + 1 + ou] = 1.0 / (dy1 - 2.0 * aab * (j + 1.0))

    assert np.all(np.isfinite(yu)) and np.all(np.isfinite(yv))

    dyu2i = np.zeros((nyu, 3))
    dyv2i = np.zeros((nyv, 3))

    def U(j):
        return yu[j + ou]

    def V(j):
        return yv[j + ov]

    j = -dny
    dyu2i[j + ou] = (0.0, -2.0 / (U(j + 1) - U(j)) ** 2, 1.0 / (U(j + 1) - U(j)) ** 2)
    dyv2i[j + ov] = (0.0, -2.0 / (V(j + 1) - V(j)) ** 2, 1.0 / (V(j + 1) - V(j)) ** 2)
    for j in range(-dny + 1, nn + dny):
        dyu2i[j + ou] = (2.0 / ((U(j) - U(j - 1)) * (U(j + 1) - U(j - 1))),
                         -2.0 / ((U(j + 1) - U(j)) * (U(j) - U(j - 1))),
                         2.0 / ((U(j + 1) - U(j)) * (U(j + 1) - U(j - 1))))
        dyv2i[j + ov] = (2.0 / ((V(j) - V(j - 1)) * (V(j + 1) - V(j - 1))),
                         -2.0 / ((V(j + 1) - V(j)) * (V(j) - V(j - 1))),
                         2.0 / ((V(j + 1) - V(j)) * (V(j + 1) - V(j - 1))))
    j = nn + dny
    dyu2i[j + ou] = (2.0 / ((U(j) - U(j - 1)) * (U(j + 1) - U(j - 1))),
                     -2.0 / ((U(j + 1) - U(j)) * (U(j) - U(j - 1))),
                     2.0 / ((U(j + 1) - U(j)) * (U(j + 1) - U(j - 1))))
    dyv2i[j + ov] = (1.0 / (V(j) - V(j - 1)) ** 2, -2.0 / (V(j) - V(j - 1)) ** 2, 0.0)
    j = nn + dny + 1
    dyu2i[j + ou] = (1.0 / (U(j) - U(j - 1)) ** 2, -2.0 / (U(j) - U(j - 1)) ** 2, 0.0)

    return YGrid(ny=ny, dny=dny, yu=yu, yv=yv, dthdyu=dthdyu, dthdyv=dthdyv,
                 dyu2i=dyu2i, dyv2i=dyv2i)


def wavenumbers(n1: int, n2: int, alp: float, bet: float):
    """kx(i) = alp*i, i = 0..N1/2; kz(q) = bet*q (q < N2/2), -bet*(N2-q) (start.f90:971-986)."""
    kx = alp * np.arange(n1 // 2 + 1, dtype=np.float64)
    q = np.arange(n2)
    kz = np.where(q < n2 // 2, bet * q, -bet * (n2 - q)).astype(np.float64)
    return kx, kz


def grid_weights(g: YGrid):
    """Ghost-point weights of one uniform band (start.f90:495-508, midband rows)."""
    yu, yv = g.u, g.v
    ju0, ju1, jv0, jv1 = g.ju0, g.ju1, g.jv0, g.jv1
    gw_bot = -(yv(jv0) - yu(ju0)) / (yv(jv0) - yu(ju0 + 1))
    gw_top = (yu(ju1) - yv(jv1)) / (yv(jv1) - yu(ju1 - 1))
    gwi_bot = (yu(ju0) - yu(ju0 + 1)) / (yv(jv0) - yu(ju0 + 1))
    gwi_top = (yu(ju1) - yu(ju1 - 1)) / (yv(jv1) - yu(ju1 - 1))
    return gw_bot, gw_top, gwi_bot, gwi_top
