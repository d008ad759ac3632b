"""Seeded initial fields and the CFL time step (host set-up).

The reference starts from a restart file or from ``mblock_ini_parabolic_profile``
(start.f90:2109-2249), which adds only constant-mode "noise".  The named workloads
start instead from laminar Poiseuille flow with unit bulk velocity between the crests
(u = 1.5 (1 - y^2), zero inside the canopies) plus a divergence-free random
perturbation: complex Gaussian amplitudes on the modes |i|, |k| <= kmax with a smooth
(1 - y^2)^2 envelope, projected onto the discretely solenoidal space with the
reference's own D.G operator (LU_buildP, tridLU_3D_IB.f90:417-491, and the v_corr
update, littleharsh.f90:796-907), then scaled to the requested rms.

``cfl_dt`` restates dtc_calc (FOU3D.f90:516-544) and the dt rule of nonlinear
(FOU3D.f90:181): dt = min(2.5 dtv, CFL dtc), dtv from start.f90:432.
"""
from __future__ import annotations

import numpy as np

from .grid import YGrid, grid_weights, wavenumbers


def _dg_solve(grid: YGrid, k2: float, rhs: np.ndarray) -> np.ndarray:
    """Solve the pressure Poisson system D.G psi + k2 psi = rhs of one column."""
    from scipy.linalg import solve_banded
    n = grid.nyp
    ab = np.zeros((3, n))
    j0 = grid.jp0
    for jj in range(n):
        j = j0 + jj
        du = grid.dthdyu[j + grid.dny]
        dvm = grid.dthdyv[j - 1 + grid.dny]
        dvp = grid.dthdyv[j + grid.dny]
        diag = k2
        if jj > 0:
            diag += -du * dvm
            ab[2, jj - 1] = du * dvm          # sub-diagonal (row jj, col jj-1)
        if jj < n - 1:
            diag += -du * dvp
            ab[0, jj + 1] = du * dvp          # super-diagonal (row jj, col jj+1)
        ab[1, jj] = diag
    return solve_banded((1, 1), ab, rhs)


def project(cfg, grid: YGrid, u, v, w, cols):
    """Make (u, v, w) discretely divergence-free on the given columns (in place)."""
    nkx = cfg.nkx
    kx, kz = wavenumbers(cfg.n1, cfg.n2, cfg.alp, cfg.bet)
    d = grid.dny
    gwb, gwt, _, _ = grid_weights(grid)
    for col in cols:
        i, q = col % nkx, col // nkx
        ikx, ikz = 1j * kx[i], 1j * kz[q]
        k2 = -(kx[i] ** 2) - (kz[q] ** 2)
        if k2 == 0.0:
            continue
        js = np.arange(grid.jp0, grid.jp1 + 1)
        div = (ikx * u[col, js + d] + ikz * w[col, js + d] +
               grid.dthdyu[js + d] * (v[col, js + d] - v[col, js - 1 + d]))
        psi = _dg_solve(grid, k2, div)
        u[col, js + d] -= ikx * psi
        w[col, js + d] -= ikz * psi
        jv = np.arange(grid.jv0 + 1, grid.jv1)
        v[col, jv + d] -= grid.dthdyv[jv + d] * (psi[jv + 1 - grid.jp0] - psi[jv - grid.jp0])
        v[col, 0] = 0.0
        v[col, -1] = 0.0
        u[col, 0] = -gwb * u[col, 1]
        u[col, -1] = -gwt * u[col, -2]
        w[col, 0] = -gwb * w[col, 1]
        w[col, -1] = -gwt * w[col, -2]


def initial_state(cfg, grid: YGrid):
    """(u1, u2, u3, p) as complex128 arrays [column, j - j0] (reference f(j,column))."""
    nkx, n2, ncol = cfg.nkx, cfg.n2, cfg.ncol
    rng = np.random.default_rng(cfg.seed)
    u = np.zeros((ncol, grid.nyu), np.complex128)
    v = np.zeros((ncol, grid.nyv), np.complex128)
    w = np.zeros((ncol, grid.nyu), np.complex128)
    p = np.zeros((ncol, grid.nyp), np.complex128)
    yu, yv = grid.yu, grid.yv
    inside_u = np.abs(yu) < 1.0
    inside_v = np.abs(yv) < 1.0
    env_u = np.where(inside_u, (1.0 - yu ** 2) ** 2, 0.0)
    env_v = np.where(inside_v, (1.0 - yv ** 2) ** 2, 0.0)

    kmax = min(cfg.kmax, cfg.n1 // 2, n2 // 2 - 1)
    cols = []
    for i in range(0, kmax + 1):
        for qs in range(-kmax, kmax + 1):
            if i == 0 and qs <= 0:
                continue
            q = qs % n2
            col = q * nkx + i
            cols.append(col)

            def amp():
                a = rng.standard_normal(2) + 1j * rng.standard_normal(2)
                return a[0] + a[1] * yu, a[0] + a[1] * yv
            au, _ = amp()
            _, av = amp()
            aw, _ = amp()
            u[col] = au * env_u
            v[col] = av * env_v
            w[col] = aw * env_u
    # kx = 0 columns of a real field are Hermitian in kz
    for qs in range(1, kmax + 1):
        cp, cm = (qs % n2) * nkx, ((-qs) % n2) * nkx
        u[cm], v[cm], w[cm] = np.conj(u[cp]), np.conj(v[cp]), np.conj(w[cp])
        cols.append(cm)
    project(cfg, grid, u, v, w, cols)

    # scale to the requested rms over the fluid region (Parseval, u(x) = sum uhat e^{ikx})
    fac = np.where((np.arange(ncol) % nkx) > 0, 2.0, 1.0)[:, None]
    e = (fac * (np.abs(u[:, inside_u]) ** 2)).sum(0) + (fac * (np.abs(w[:, inside_u]) ** 2)).sum(0)
    ev = (fac * (np.abs(v[:, inside_v]) ** 2)).sum(0)
    rms = np.sqrt((e.mean() + ev.mean()) / 3.0) if e.size else 0.0
    if rms > 0:
        s = cfg.perturbation / rms
        u *= s
        v *= s
        w *= s
    u[0] = np.where(inside_u, 1.5 * (1.0 - yu ** 2), 0.0)
    gwb, gwt, _, _ = grid_weights(grid)
    u[0, 0] = -gwb * u[0, 1]
    u[0, -1] = -gwt * u[0, -2]
    return u, v, w, p


def to_physical_plane(f_col: np.ndarray, cfg) -> np.ndarray:
    """Physical samples (Ngal2, Ngal1) of one plane of spectral column values (ncol,)."""
    nkx, n2 = cfg.nkx, cfg.n2
    full = np.zeros((cfg.ngal2, cfg.ngal1 // 2 + 1), np.complex128)
    sp = f_col.reshape(n2, nkx)
    full[: n2 // 2, :nkx] = sp[: n2 // 2]
    full[cfg.ngal2 - n2 // 2:, :nkx] = sp[n2 // 2:]
    full[:, 0] = full[:, 0]
    # inverse, unnormalised: u = sum uhat e^{i(kx x + kz z)}; kx=0 column uses Re only
    zc = np.fft.ifft(full, axis=0) * cfg.ngal2
    zc[:, 0] = zc[:, 0].real
    return np.fft.irfft(zc, n=cfg.ngal1, axis=1) * cfg.ngal1


def cfl_dt(cfg, grid: YGrid, u, v, w) -> float:
    umax = max(np.abs(to_physical_plane(u[:, j], cfg)).max() for j in range(grid.nyu))
    wmax = max(np.abs(to_physical_plane(w[:, j], cfg)).max() for j in range(grid.nyu))
    vmax = 1e-6
    for jj in range(1, grid.nyv - 1):
        vmax = max(vmax, np.abs(to_physical_plane(v[:, jj], cfg)).max() * grid.dthdyv[jj])
    dtc = min(1.0 / (cfg.alp * (cfg.n1 // 2) * umax), 1.0 / (cfg.bet * (cfg.n2 // 2) * wmax),
              1.0 / vmax)
    return float(min(2.5 * viscous_dt(cfg, grid), cfg.cfl * dtc))


def viscous_dt(cfg, grid: YGrid) -> float:
    """dtv of start.f90:432: Re / (kx_max^2 + kz_max^2 + 4 / (yv(1) - yv(0))^2), with the
    reference's kx = alp N1/2 and kz = bet (N2/2 - 1) extremes."""
    kx, _ = wavenumbers(cfg.n1, cfg.n2, cfg.alp, cfg.bet)
    k2x = -(kx[cfg.n1 // 2] ** 2)
    k2z = -(cfg.bet * (cfg.n2 // 2 - 1)) ** 2
    return float(cfg.re_b / (-k2x - k2z + 4.0 / (grid.yv[1] - grid.yv[0]) ** 2))
