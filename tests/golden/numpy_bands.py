"""Independent numpy restatement of one RK3 substep of a THREE-band channel (test
infrastructure).

Structured as the reference stores it, not as the C++ oracle does: the state is three
column blocks, the reference's u(iband)%f(j,column) (declaration.f90:140-142) -- band 1 the
short columns over the bottom band's rows, band 2 the long columns over the whole channel,
band 3 the short columns over the top band's rows (jlim, start.f90:1538-1557) -- and every
stage loops over the blocks with that block's row range and end coefficients.  Planes are
assembled from the blocks that have rows there (modes_to_planes_UVP, FOU3D.f90:808-906) and
transformed at their band's size with numpy.fft under the FFTPACK scaling of the reference's
rft/cft.  It pins the oracle's three-band restatement stage by stage.

Citations (Mel222/CFD): start.f90:76-111 (band sizes), :1382-1557 (column lists, jlim),
:494-508 (gridweighting per band), FOU3D.f90:261-308 (interp_u/v per band), :1529-1617
(ops_in_planes at bandPL's size), :310-414 (der_x/der_z), :453-493 (der_yu_h/der_yv_h),
tridLU_3D_IB.f90:50-160, 349-413 (LUsolU/V, LU_buildU/V per band), :284-318, 417-491
(LUsolP, LU_buildP per band), littleharsh.f90:209-244 (divergence), 556-611 (solveP),
613-730 (RHS0), 732-794 (solveU/V), 796-907 (v_corr).
"""
from __future__ import annotations

import numpy as np

from numpy_ref import A, B, CC, D, G, NumpyChannel


class NumpyBands:
    def __init__(self, setup):
        cfg, g = setup.cfg, setup.grid
        self.cfg, self.g, self.dt = cfg, g, setup.dt
        self.re = cfg.re_b
        self.mpgx = cfg.mpgx
        self.ibu, self.ibv = setup.ibu, setup.ibv
        self.ng = {1: (cfg.ngal1, cfg.ngal2), 2: (cfg.ngal1_mid, cfg.ngal2_mid), 3: (cfg.ngal1, cfg.ngal2)}
        self.n = {b: (2 * (a // 3), 2 * (c // 3)) for b, (a, c) in self.ng.items()}
        n1, n2 = self.n[1]
        n1m, n2m = self.n[2]
        nkx = n1 // 2 + 1
        col = np.arange(nkx * n2)
        i, q = col % nkx, col // nkx
        islong = (i <= n1m // 2) & ((q < n2m // 2) | (q >= n2 - n2m // 2))
        self.cols = {1: col[~islong], 2: col[islong], 3: col[~islong]}  # global column of each block entry
        self.ci = {b: c % nkx for b, c in self.cols.items()}
        self.cq = {b: c // nkx for b, c in self.cols.items()}
        self.kx = {b: cfg.alp * self.ci[b] for b in self.cols}
        self.kz = {b: cfg.bet * np.where(self.cq[b] < n2 // 2, self.cq[b], self.cq[b] - n2) for b in self.cols}
        self.ncol_all = nkx * n2
        self.n2 = n2
        jb = cfg.band_vface
        m = cfg.ny - 2 - jb
        self.jb, self.m = jb, m
        # (u0, u1, v0, v1, p0, p1) of each block (jlim)
        self.rng = {1: (g.ju0, jb + 2, g.jv0, jb + 1, g.ju0 + 1, jb + 1),
                    2: (g.ju0, g.ju1, g.jv0, g.jv1, g.jp0, g.jp1),
                    3: (m, g.ju1, m, g.jv1, m + 1, g.jp1)}
        yu = lambda j: g.yu[j - g.ju0]
        yv = lambda j: g.yv[j - g.jv0]
        gw_bot = -(yv(g.jv0) - yu(g.ju0)) / (yv(g.jv0) - yu(g.ju0 + 1))
        gw_top = (yu(g.ju1) - yv(g.jv1)) / (yv(g.jv1) - yu(g.ju1 - 1))
        gwi_bot = (yu(g.ju0) - yu(g.ju0 + 1)) / (yv(g.jv0) - yu(g.ju0 + 1))
        gwi_top = (yu(g.ju1) - yu(g.ju1 - 1)) / (yv(g.jv1) - yu(g.ju1 - 1))
        # gridweighting(band, 1:2) and gridweighting_interp(band, 1:2) (start.f90:494-508)
        self.gw = {1: (gw_bot, (yu(jb + 2) - yv(jb + 1)) / (yv(jb + 1) - yu(jb + 1))),
                   2: (gw_bot, gw_top),
                   3: (-(yv(m) - yu(m)) / (yv(m) - yu(m + 1)), gw_top)}
        self.gwi = {1: (gwi_bot, (yu(jb + 2) - yu(jb + 1)) / (yv(jb + 1) - yu(jb + 1))),
                    2: (gwi_bot, gwi_top),
                    3: ((yu(m) - yu(m + 1)) / (yv(m) - yu(m + 1)), gwi_top)}
        self.yu, self.yv = yu, yv
        z = lambda b, a, c: np.zeros((len(self.cols[b]), c - a + 1), np.complex128)
        self.f = {}
        for b in (1, 2, 3):
            u0, u1, v0, v1, p0, p1 = self.rng[b]
            blk = {k: z(b, u0, u1) for k in ("u1", "u3", "nu1", "nu3", "du1", "du3", "vvc", "u2i")}
            blk.update({k: z(b, v0, v1) for k in ("u2", "nu2", "du2", "uvf", "vwf", "u1i", "u3i")})
            blk.update({k: z(b, p0, p1) for k in ("p", "psi", "div")})
            self.f[b] = blk

    # --- blocks <-> the wall-band column layout (columns x all rows) ------------------------
    def _rows(self, b, which):
        u0, u1, v0, v1, p0, p1 = self.rng[b]
        g = self.g
        return {"u": (u0 - g.ju0, u1 - g.ju0), "v": (v0 - g.jv0, v1 - g.jv0), "p": (p0 - g.jp0, p1 - g.jp0)}[which]

    GRID = {"u1": "u", "u3": "u", "nu1": "u", "nu3": "u", "du1": "u", "du3": "u",
            "u2": "v", "nu2": "v", "du2": "v", "p": "p", "psi": "p", "div": "p"}

    def upload(self, name, arr):
        which = self.GRID[name]
        for b in (1, 2, 3):
            r0, r1 = self._rows(b, which)
            self.f[b][name][:] = arr[self.cols[b], r0:r1 + 1]

    def download(self, name):
        g = self.g
        which = self.GRID[name]
        nrow = {"u": g.nyu, "v": g.nyv, "p": g.nyp}[which]
        out = np.zeros((self.ncol_all, nrow), np.complex128)
        for b in (1, 2, 3):
            r0, r1 = self._rows(b, which)
            out[self.cols[b], r0:r1 + 1] = self.f[b][name]
        return out

    def upload_state(self, st):
        for k in ("u1", "u2", "u3", "p"):
            self.upload(k, st[k])

    def download_state(self):
        return {k: self.download(k) for k in ("u1", "u2", "u3", "p")}

    # --- planes --------------------------------------------------------------------------
    def _band_u(self, j):
        return 1 if j <= self.jb + 1 else (3 if j > self.m else 2)

    def _band_v(self, j):
        return 1 if j <= self.jb else (3 if j > self.m else 2)

    def _blocks_on(self, band):
        # a plane of a wall band carries the long block and that band's short block
        return (2,) if band == 2 else (band, 2)

    def _to_phys(self, band, spec):
        """spec: {block: values (ncol_b,)} -> physical plane (ng2, ng1) of the band's size."""
        ng1, ng2 = self.ng[band]
        n1, n2 = self.n[band]
        full = np.zeros((ng2, ng1 // 2 + 1), np.complex128)
        for b, v in spec.items():
            q = self.cq[b]
            rows = np.where(q < self.n2 // 2, q, q - self.n2 + ng2)
            full[rows, self.ci[b]] = v
        zc = np.fft.ifft(full, axis=0) * ng2
        zc[:, 0] = zc[:, 0].real
        zc[:, -1] = zc[:, -1].real
        return np.fft.irfft(zc, n=ng1, axis=1) * ng1

    def _to_spec(self, band, x, blocks):
        ng1, ng2 = self.ng[band]
        xr = np.fft.rfft(x, axis=1) / ng1
        xr[:, 0] = xr[:, 0].real
        zc = np.fft.fft(xr, axis=0) / ng2
        out = {}
        for b in blocks:
            q = self.cq[b]
            rows = np.where(q < self.n2 // 2, q, q - self.n2 + ng2)
            out[b] = zc[rows, self.ci[b]]
        return out

    def _plane(self, band, name, j, grid):
        spec = {}
        for b in self._blocks_on(band):
            u0, u1, v0, v1 = self.rng[b][:4]
            a = u0 if grid == "u" else v0
            spec[b] = self.f[b][name][:, j - a]
        return self._to_phys(band, spec)

    # --- stages ----------------------------------------------------------------------------
    def rhs0(self, krk):
        r, g = krk - 1, self.g
        C1, C2 = A[r] / self.re, -CC[r]
        for b in (1, 2, 3):
            f = self.f[b]
            u0, u1, v0, v1, p0, p1 = self.rng[b]
            k2 = -(self.kx[b] ** 2) - (self.kz[b] ** 2)
            for u, du, nu, C3 in ((f["u1"], f["du1"], f["nu1"], -D[r] * 1j * self.kx[b]),
                                  (f["u3"], f["du3"], f["nu3"], -D[r] * 1j * self.kz[b])):
                for j in range(u0 + 1, u1):
                    c = g.dyu2i[j - g.ju0]
                    jj = j - u0
                    L = c[0] * u[:, jj - 1] + (k2 + c[1]) * u[:, jj] + c[2] * u[:, jj + 1]
                    du[:, jj] = C1 * L + C2 * nu[:, jj] + C3 * f["p"][:, j - p0]
            if b == 2:
                f["du1"][0, 1:-1] += -D[r] * self.mpgx
            for j in range(v0 + 1, v1):
                c = g.dyv2i[j - g.jv0]
                jj = j - v0
                L = c[0] * f["u2"][:, jj - 1] + (k2 + c[1]) * f["u2"][:, jj] + c[2] * f["u2"][:, jj + 1]
                C3 = -D[r] * g.dthdyv[j - g.jv0]
                f["du2"][:, jj] = C1 * L + C2 * f["nu2"][:, jj] + C3 * (f["p"][:, j + 1 - p0] - f["p"][:, j - p0])

    def _interp(self):
        yu, yv = self.yu, self.yv
        for b in (1, 2, 3):
            f = self.f[b]
            u0, u1, v0, v1 = self.rng[b][:4]
            for j in range(v0, v1 + 1):
                w = ((yv(j) - yu(j)), (yu(j + 1) - yv(j)), (yu(j + 1) - yu(j)))
                for s, d in (("u1", "u1i"), ("u3", "u3i")):
                    f[d][:, j - v0] = (w[0] * f[s][:, j + 1 - u0] + w[1] * f[s][:, j - u0]) / w[2]
            for j in range(u0 + 1, u1):
                f["u2i"][:, j - u0] = ((yu(j) - yv(j - 1)) * f["u2"][:, j - v0] +
                                       (yv(j) - yu(j)) * f["u2"][:, j - 1 - v0]) / (yv(j) - yv(j - 1))
            gb, gt = self.gwi[b]
            f["u2i"][:, 0] = gb * (f["u2"][:, 0] - f["u2i"][:, 1]) + f["u2i"][:, 1]
            f["u2i"][:, -1] = gt * (f["u2"][:, -1] - f["u2i"][:, -2]) + f["u2i"][:, -2]

    def _dxz(self, band, b, a, c):
        n2b = self.n[band][1]
        v = 1j * self.kx[b] * a + 1j * self.kz[b] * c
        v[self.cq[b] == self.n2 - n2b // 2] = 0.0   # the band's kz = -N2/2 mode
        return v

    def nonlinear(self, krk):
        g = self.g
        self._interp()
        xz1 = {b: np.zeros_like(self.f[b]["u1"]) for b in (1, 2, 3)}
        xz3 = {b: np.zeros_like(self.f[b]["u1"]) for b in (1, 2, 3)}
        xz2 = {b: np.zeros_like(self.f[b]["u2"]) for b in (1, 2, 3)}
        for j in range(g.ju0, g.ju1 + 1):
            band = self._band_u(j)
            U, V, W = (self._plane(band, k, j, "u") for k in ("u1", "u2i", "u3"))
            blocks = self._blocks_on(band)
            uu, uw, vv, ww = (self._to_spec(band, x, blocks) for x in (U * U, U * W, V * V, W * W))
            for b in blocks:
                jj = j - self.rng[b][0]
                self.f[b]["vvc"][:, jj] = vv[b]
                if g.ju0 < j < g.ju1:
                    xz1[b][:, jj] = self._dxz(band, b, uu[b], uw[b])
                    xz3[b][:, jj] = self._dxz(band, b, uw[b], ww[b])
        for j in range(g.jv0, g.jv1 + 1):
            band = self._band_v(j)
            U, V, W = (self._plane(band, k, j, "v") for k in ("u1i", "u2", "u3i"))
            blocks = self._blocks_on(band)
            uv, vw = (self._to_spec(band, x, blocks) for x in (U * V, W * V))
            for b in blocks:
                jj = j - self.rng[b][2]
                self.f[b]["uvf"][:, jj] = uv[b]
                self.f[b]["vwf"][:, jj] = vw[b]
                if g.jv0 < j < g.jv1:
                    xz2[b][:, jj] = self._dxz(band, b, uv[b], vw[b])
        C1 = -G[krk - 1]
        for b in (1, 2, 3):
            f = self.f[b]
            u0, u1, v0, v1 = self.rng[b][:4]
            for j in range(u0 + 1, u1):
                jj, jv = j - u0, j - v0
                f["nu1"][:, jj] = xz1[b][:, jj] + (f["uvf"][:, jv] - f["uvf"][:, jv - 1]) * g.dthdyu[j - g.ju0]
                f["nu3"][:, jj] = xz3[b][:, jj] + (f["vwf"][:, jv] - f["vwf"][:, jv - 1]) * g.dthdyu[j - g.ju0]
                f["du1"][:, jj] += C1 * f["nu1"][:, jj]
                f["du3"][:, jj] += C1 * f["nu3"][:, jj]
            for j in range(v0 + 1, v1):
                jj, ju = j - v0, j - u0
                f["nu2"][:, jj] = xz2[b][:, jj] + (f["vvc"][:, ju + 1] - f["vvc"][:, ju]) * g.dthdyv[j - g.jv0]
                f["du2"][:, jj] += C1 * f["nu2"][:, jj]

    def _ib(self, name_u, name_r, lst, grid):
        g = self.g
        if lst is None or lst.n == 0:
            return
        j0, j1 = (g.ju0, g.ju1) if grid == "u" else (g.jv0, g.jv1)
        planes = sorted({j for s in range(2) for j in range(max(lst.jlo[s], j0 + 1), min(lst.jhi[s], j1 - 1) + 1)})
        R = {j: self._plane(self._band_u(j) if grid == "u" else self._band_v(j), name_r, j, grid) for j in planes}
        Uv = {j: self._plane(self._band_u(j) if grid == "u" else self._band_v(j), name_u, j, grid) for j in planes}
        for p in range(lst.n):
            i, k, j, i2, k2, j2, i3, k3, j3 = (int(x) for x in lst.idx[p])
            lap, w2, w3 = lst.w[p]
            vf = w2 * Uv[j2][k2 - 1, i2 - 1] + w3 * Uv[j3][k3 - 1, i3 - 1]
            R[j][k - 1, i - 1] = lap * (vf - Uv[j][k - 1, i - 1] + R[j][k - 1, i - 1])
        for j in planes:
            band = self._band_u(j) if grid == "u" else self._band_v(j)
            blocks = self._blocks_on(band)
            spec = self._to_spec(band, R[j], blocks)
            for b in blocks:
                a = self.rng[b][0] if grid == "u" else self.rng[b][2]
                self.f[b][name_r][:, j - a] = spec[b]

    def solve_uvw(self, krk):
        g, dt = self.g, self.dt
        beta = B[krk - 1] * dt / self.re
        for b in (1, 2, 3):
            f = self.f[b]
            for u, du in (("u1", "du1"), ("u3", "du3"), ("u2", "du2")):
                f[du][:, 0] = 0
                f[du][:, 1:-1] = f[u][:, 1:-1] + dt * f[du][:, 1:-1]
                f[du][:, -1] = 0
        self._ib("u1", "du1", self.ibu, "u")
        self._ib("u2", "du2", self.ibv, "v")
        self._ib("u3", "du3", self.ibu, "u")
        for b in (1, 2, 3):
            f = self.f[b]
            u0, u1, v0, v1 = self.rng[b][:4]
            k2x, k2z = -(self.kx[b] ** 2)[:, None], -(self.kz[b] ** 2)[:, None]
            nc = len(self.cols[b])
            n = u1 - u0 + 1
            c = g.dyu2i[u0 - g.ju0:u1 - g.ju0 + 1]
            a1, a2, a3 = np.zeros((nc, n)), np.zeros((nc, n)), np.zeros((nc, n))
            a2[:, 0], a3[:, 0] = 1.0, self.gw[b][0]
            a1[:, 1:-1] = -beta * c[None, 1:-1, 0]
            a2[:, 1:-1] = 1.0 - beta * ((c[None, 1:-1, 1] + k2x) + k2z)
            a3[:, 1:-1] = -beta * c[None, 1:-1, 2]
            a1[:, -1], a2[:, -1] = self.gw[b][1], 1.0
            f["u1"][:] = NumpyChannel._thomas(a1, a2, a3, f["du1"])
            f["u3"][:] = NumpyChannel._thomas(a1, a2, a3, f["du3"])
            n = v1 - v0 + 1
            c = g.dyv2i[v0 - g.jv0:v1 - g.jv0 + 1]
            a1, a2, a3 = np.zeros((nc, n)), np.ones((nc, n)), np.zeros((nc, n))
            a1[:, 1:-1] = -beta * c[None, 1:-1, 0]
            a2[:, 1:-1] = 1.0 - beta * ((c[None, 1:-1, 1] + k2x) + k2z)
            a3[:, 1:-1] = -beta * c[None, 1:-1, 2]
            f["u2"][:] = NumpyChannel._thomas(a1, a2, a3, f["du2"])

    def meanflow(self, krk):
        if self.cfg.flag_ctpress == 1:
            return
        raise NotImplementedError("the constant-flow-rate mean mode is covered by the one-band restatement")

    def _divergence(self, b):
        g, f = self.g, self.f[b]
        u0, u1, v0, v1, p0, p1 = self.rng[b]
        j = np.arange(p0, p1 + 1)
        return (1j * self.kx[b][:, None] * f["u1"][:, j - u0] + 1j * self.kz[b][:, None] * f["u3"][:, j - u0] +
                g.dthdyu[None, j - g.ju0] * (f["u2"][:, j - v0] - f["u2"][:, j - 1 - v0]))

    def solve_p(self, krk):
        g = self.g
        dtirk = (1.0 / self.dt) / (A[krk - 1] + B[krk - 1])
        for b in (1, 2, 3):
            f = self.f[b]
            p0, p1 = self.rng[b][4:]
            f["div"][:] = self._divergence(b)
            r = dtirk * f["div"]
            if b == 2:
                r[0, 0] = 0.0
            jp = np.arange(p0, p1 + 1)
            du = g.dthdyu[jp - g.ju0]
            dvm = g.dthdyv[jp - 1 - g.jv0]
            dvp = g.dthdyv[jp - g.jv0]
            n, nc = len(jp), len(self.cols[b])
            k2x, k2z = -(self.kx[b] ** 2)[:, None], -(self.kz[b] ** 2)[:, None]
            a1, a2, a3 = np.zeros((nc, n)), np.zeros((nc, n)), np.zeros((nc, n))
            a2[:, 0:1] = (du[0] * -dvp[0]) + k2x + k2z
            a3[:, 0] = du[0] * dvp[0]
            a2[:, -1:] = ((-du[-1]) * dvm[-1]) + k2x + k2z
            a1[:, -1] = (-du[-1]) * (-dvm[-1])
            mid = slice(1, n - 1)
            a2[:, mid] = (((-du[mid]) * dvm[mid]) + (du[mid] * -dvp[mid]))[None, :] + k2x + k2z
            a1[:, mid] = ((-du[mid]) * (-dvm[mid]))[None, :]
            a3[:, mid] = (du[mid] * dvp[mid])[None, :]
            if b == 2:
                a1[0, 0], a2[0, 0], a3[0, 0] = 0.0, 1.0 / (g.u(2) - g.u(1)) ** 2, 0.0
            f["psi"][:] = NumpyChannel._thomas(a1, a2, a3, r)
            f["p"][:] = f["p"] + f["psi"]

    def vcorr(self, krk):
        g = self.g
        dtrk = self.dt * (A[krk - 1] + B[krk - 1])
        for b in (1, 2, 3):
            f = self.f[b]
            u0, u1, v0, v1, p0, p1 = self.rng[b]
            f["u1"][:, 1:-1] -= (dtrk * 1j * self.kx[b])[:, None] * f["psi"]
            f["u3"][:, 1:-1] -= (dtrk * 1j * self.kz[b])[:, None] * f["psi"]
            # ghost rows from the channel's gridweighting: bottom of bands 1-2, top of 2-3
            for u in (f["u1"], f["u3"]):
                if b in (1, 2):
                    u[:, 0] = -self.gw[1][0] * u[:, 1]
                if b in (2, 3):
                    u[:, -1] = -self.gw[3][1] * u[:, -2]
            jv = np.arange(v0 + 1, v1)
            f["u2"][:, 1:-1] -= dtrk * g.dthdyv[None, jv - g.jv0] * (f["psi"][:, 1:] - f["psi"][:, :-1])
            f["u2"][:, 0] = 0
            f["u2"][:, -1] = 0
            f["div"][:] = self._divergence(b)
