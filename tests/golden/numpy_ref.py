"""Second, independent FP64 restatement of one RK3 substep in numpy (test infrastructure).

Written from the reference Fortran directly and structured differently from the C++
oracle: transforms use numpy.fft (pocketfft) with the FFTPACK scaling/storage of the
reference wrappers, columns are vectorised, and the Thomas sweeps run over all columns
at once.  It pins the C++ oracle on small grids and generates the committed golden
fixtures (make_golden.py).

Reference citations (Mel222/CFD): littleharsh.f90:163-189 (substep), :613-730 (RHS0),
FOU3D.f90:41-259, 1529-1617 (nonlinear), tridLU_3D_IB.f90:50-318 (solves, IB),
littleharsh.f90:556-611, 796-907 (solveP, v_corr), start.f90:395-409 (RK3).
"""
from __future__ import annotations

import numpy as np

A = np.array([4 / 15, 1 / 15, 1 / 6])
B = np.array([4 / 15, 1 / 15, 1 / 6])
G = np.array([8 / 15, 5 / 12, 3 / 4])
CC = np.array([0.0, -17 / 60, -5 / 12])
D = np.array([8 / 15, 2 / 15, 1 / 3])


class NumpyChannel:
    def __init__(self, setup):
        cfg, g = setup.cfg, setup.grid
        self.cfg, self.g, self.dt = cfg, g, setup.dt
        self.re = cfg.re_b
        self.ng1, self.ng2 = cfg.ngal1, cfg.ngal2
        self.n1, self.n2 = cfg.n1, cfg.n2
        self.nkx, self.ncol = cfg.nkx, cfg.ncol
        i = np.arange(self.ncol) % self.nkx
        q = np.arange(self.ncol) // self.nkx
        self.kx = cfg.alp * i
        qs = np.where(q < self.n2 // 2, q, q - self.n2)
        self.kz = cfg.bet * qs
        self.q = q
        self.i = i
        self.rows = np.where(q < self.n2 // 2, q, q + self.ng2 - self.n2)
        self.k2 = -(self.kx ** 2) - (self.kz ** 2)
        self.ibu, self.ibv = setup.ibu, setup.ibv
        self.mpgx = cfg.mpgx
        self.qxt = cfg.qxt
        self.ctp = cfg.flag_ctpress
        self.Qx = 0.0
        yu, yv = g.yu, g.yv
        self.gwb = -(yv[0] - yu[0]) / (yv[0] - yu[1])
        self.gwt = (yu[-1] - yv[-1]) / (yv[-1] - yu[-2])
        self.gwib = (yu[0] - yu[1]) / (yv[0] - yu[1])
        self.gwit = (yu[-1] - yu[-2]) / (yv[-1] - yu[-2])
        z = lambda n: np.zeros((self.ncol, n), np.complex128)
        self.u1, self.u3, self.u2, self.p = z(g.nyu), z(g.nyu), z(g.nyv), z(g.nyp)
        self.nu1, self.nu3, self.nu2 = z(g.nyu), z(g.nyu), z(g.nyv)
        self.du1, self.du3, self.du2 = z(g.nyu), z(g.nyu), z(g.nyv)
        self.psi, self.div = z(g.nyp), z(g.nyp)

    # --- transforms of one plane: spectral columns (ncol,) <-> physical (ng2, ng1) --------
    def to_phys(self, f):
        full = np.zeros((self.ng2, self.ng1 // 2 + 1), np.complex128)
        full[self.rows, self.i] = f
        zc = np.fft.ifft(full, axis=0) * self.ng2          # cft inverse (unscaled)
        zc[:, 0] = zc[:, 0].real                          # rft ignores Im of kx = 0
        zc[:, -1] = zc[:, -1].real
        return np.fft.irfft(zc, n=self.ng1, axis=1) * self.ng1

    def to_spec(self, x):
        xr = np.fft.rfft(x, axis=1) / self.ng1            # rft forward, x 1/n
        xr[:, 0] = xr[:, 0].real
        zc = np.fft.fft(xr, axis=0) / self.ng2            # cft forward, x 1/n
        return zc[self.rows, self.i]

    # --- stages -------------------------------------------------------------------------
    def rhs0(self, krk):
        r, g = krk - 1, self.g
        C1, C2 = A[r] / self.re, -CC[r]
        for u, du, nu, C3 in ((self.u1, self.du1, self.nu1, -D[r] * 1j * self.kx),
                              (self.u3, self.du3, self.nu3, -D[r] * 1j * self.kz)):
            for jj in range(1, g.nyu - 1):
                c = g.dyu2i[jj]
                L = c[0] * u[:, jj - 1] + (self.k2 + c[1]) * u[:, jj] + c[2] * u[:, jj + 1]
                du[:, jj] = C1 * L + C2 * nu[:, jj] + C3 * self.p[:, jj - 1]
        self.du1[0, 1:g.nyu - 1] += -D[r] * self.mpgx
        for jj in range(1, g.nyv - 1):
            c = g.dyv2i[jj]
            L = c[0] * self.u2[:, jj - 1] + (self.k2 + c[1]) * self.u2[:, jj] + c[2] * self.u2[:, jj + 1]
            C3 = -D[r] * g.dthdyv[jj]
            # p index: p(j) at array index j - jp0 = jj - 1
            self.du2[:, jj] = C1 * L + C2 * self.nu2[:, jj] + C3 * (self.p[:, jj] - self.p[:, jj - 1])

    def nonlinear(self, krk):
        g = self.g
        yu, yv = g.yu, g.yv
        nyu, nyv = g.nyu, g.nyv
        # interp_u: face j from centres j, j+1 (array index jj = j - jv0 = j - ju0)
        u1i = np.zeros((self.ncol, nyv), np.complex128)
        u3i = np.zeros_like(u1i)
        for jj in range(nyv):
            w = ((yv[jj] - yu[jj]), (yu[jj + 1] - yv[jj]), (yu[jj + 1] - yu[jj]))
            u1i[:, jj] = (w[0] * self.u1[:, jj + 1] + w[1] * self.u1[:, jj]) / w[2]
            u3i[:, jj] = (w[0] * self.u3[:, jj + 1] + w[1] * self.u3[:, jj]) / w[2]
        # interp_v: centre j from faces j-1, j
        u2i = np.zeros((self.ncol, nyu), np.complex128)
        for jj in range(1, nyu - 1):
            u2i[:, jj] = ((yu[jj] - yv[jj - 1]) * self.u2[:, jj] + (yv[jj] - yu[jj]) * self.u2[:, jj - 1]) / \
                (yv[jj] - yv[jj - 1])
        u2i[:, 0] = self.gwib * (self.u2[:, 0] - u2i[:, 1]) + u2i[:, 1]
        u2i[:, -1] = self.gwit * (self.u2[:, -1] - u2i[:, -2]) + u2i[:, -2]
        zrow = self.q == self.n2 // 2
        ikx, ikz = 1j * self.kx, 1j * self.kz

        def dxz(a, b):
            v = ikx * a + ikz * b
            v[zrow] = 0.0
            return v
        vvc = np.zeros((self.ncol, nyu), np.complex128)
        nu1, nu3 = np.zeros_like(vvc), np.zeros_like(vvc)
        for jj in range(nyu):
            U, V, W = self.to_phys(self.u1[:, jj]), self.to_phys(u2i[:, jj]), self.to_phys(self.u3[:, jj])
            uu, uw, vv, ww = (self.to_spec(U * U), self.to_spec(U * W), self.to_spec(V * V), self.to_spec(W * W))
            vvc[:, jj] = vv
            nu1[:, jj] = dxz(uu, uw)
            nu3[:, jj] = dxz(uw, ww)
        uvf = np.zeros((self.ncol, nyv), np.complex128)
        vwf, nu2 = np.zeros_like(uvf), np.zeros_like(uvf)
        for jj in range(nyv):
            U, V, W = self.to_phys(u1i[:, jj]), self.to_phys(self.u2[:, jj]), self.to_phys(u3i[:, jj])
            uv, vw = self.to_spec(U * V), self.to_spec(W * V)
            uvf[:, jj], vwf[:, jj] = uv, vw
            nu2[:, jj] = dxz(uv, vw)
        C1 = -G[krk - 1]
        for jj in range(1, nyu - 1):
            self.nu1[:, jj] = nu1[:, jj] + (uvf[:, jj] - uvf[:, jj - 1]) * g.dthdyu[jj]
            self.nu3[:, jj] = nu3[:, jj] + (vwf[:, jj] - vwf[:, jj - 1]) * g.dthdyu[jj]
            self.du1[:, jj] += C1 * self.nu1[:, jj]
            self.du3[:, jj] += C1 * self.nu3[:, jj]
        for jj in range(1, nyv - 1):
            self.nu2[:, jj] = nu2[:, jj] + (vvc[:, jj + 1] - vvc[:, jj]) * g.dthdyv[jj]
            self.du2[:, jj] += C1 * self.nu2[:, jj]

    # --- statistics (stats.f90:1-253 with FOU3D.f90:187-207) and dtc_calc (:516-544) ------
    def _interp(self):
        g = self.g
        yu, yv = g.yu, g.yv
        u3i = np.zeros((self.ncol, g.nyv), np.complex128)
        for jj in range(g.nyv):
            u3i[:, jj] = ((yv[jj] - yu[jj]) * self.u3[:, jj + 1] + (yu[jj + 1] - yv[jj]) * self.u3[:, jj]) / \
                (yu[jj + 1] - yu[jj])
        u2i = np.zeros((self.ncol, g.nyu), np.complex128)
        for jj in range(1, g.nyu - 1):
            u2i[:, jj] = ((yu[jj] - yv[jj - 1]) * self.u2[:, jj] + (yv[jj] - yu[jj]) * self.u2[:, jj - 1]) / \
                (yv[jj] - yv[jj - 1])
        u2i[:, 0] = self.gwib * (self.u2[:, 0] - u2i[:, 1]) + u2i[:, 1]
        u2i[:, -1] = self.gwit * (self.u2[:, -1] - u2i[:, -2]) + u2i[:, -2]
        return u2i, u3i

    def stats(self, jband, dnx, dnz):
        """One stats() call on zeroed accumulators: plane sums and the conditional sums of
        the bottom band plus the mirrored top band (the layout write_stats stores)."""
        g = self.g
        u2i, u3i = self._interp()
        ntx, ntz = self.ng1 // dnx, self.ng2 // dnz

        def fold(x):
            return x.reshape(ntz, dnz, ntx, dnx).sum(axis=(0, 2))
        nbu, nbv, nbp = (jband + 1 - g.ju0 + 1, jband - g.jv0 + 1, jband - g.jp0 + 1) if jband >= g.jv0 else (0, 0, 0)
        out = {}
        cond = {k: np.zeros((nb, dnz, dnx)) for k, nb in
                (("UmC", nbu), ("U2mC", nbu), ("WmC", nbu), ("W2mC", nbu), ("UVmC", nbu), ("UWmC", nbu),
                 ("VmC", nbv), ("V2mC", nbv), ("wxmC", nbv), ("wx2mC", nbv), ("VWmC", nbv),
                 ("PmC", nbp), ("P2mC", nbp))}
        su = np.zeros((6, g.nyu))
        for jj in range(g.nyu):
            U, W, Vi = self.to_phys(self.u1[:, jj]), self.to_phys(self.u3[:, jj]), self.to_phys(u2i[:, jj])
            su[:, jj] = [U.sum(), (U * U).sum(), W.sum(), (W * W).sum(), (U * Vi).sum(), (U * W).sum()]
            for j1, sg in ((jj, 1.0), (g.nyu - 1 - jj, -1.0)):
                if j1 < nbu:
                    for k, x in (("UmC", U), ("U2mC", U * U), ("WmC", W), ("W2mC", W * W),
                                 ("UVmC", U * Vi * sg), ("UWmC", U * W)):
                        cond[k][j1] += fold(x)
        sv = np.zeros((5, g.nyv))
        zrow = self.q == self.n2 // 2
        for jj in range(g.nyv):
            V, Wi = self.to_phys(self.u2[:, jj]), self.to_phys(u3i[:, jj])
            dz = 1j * self.kz * self.u2[:, jj]
            dz[zrow] = 0.0
            wx = self.to_phys(-dz + (self.u3[:, jj + 1] - self.u3[:, jj]) * g.dthdyv[jj])
            wxs = wx[:self.n2, :self.n1]
            sv[:, jj] = [V.sum(), (V * V).sum(), wxs.sum(), (wxs * wxs).sum(), (V * Wi).sum()]
            for j1, sg in ((jj, 1.0), (g.nyv - 1 - jj, -1.0)):
                if j1 < nbv:
                    for k, x in (("VmC", V * sg), ("V2mC", V * V), ("wxmC", wx), ("wx2mC", wx * wx),
                                 ("VWmC", V * sg * Wi)):
                        cond[k][j1] += fold(x)
        sp = np.zeros((2, g.nyp))
        for jj in range(g.nyp):
            P = self.to_phys(self.p[:, jj])
            sp[:, jj] = [P.sum(), (P * P).sum()]
            for j1 in (jj, g.nyp - 1 - jj):
                if j1 < nbp:
                    cond["PmC"][j1] += fold(P)
                    cond["P2mC"][j1] += fold(P * P)
        for names, a in ((("Um", "U2m", "Wm", "W2m", "UVm", "UWm"), su), (("Vm", "V2m", "wxm", "wx2m", "VWm"), sv),
                         (("Pm", "P2m"), sp)):
            for q, n in enumerate(names):
                out[n] = a[q]
        out.update(cond)
        return out

    def spectra(self):
        """One spectra() call on zeroed accumulators (spectra.f90:1-56), sp(j,column)."""
        u2i, _ = self._interp()
        a = self.u1
        return {"spU": np.abs(a) ** 2, "spV": np.abs(self.u2) ** 2, "spW": np.abs(self.u3) ** 2,
                "spUV": a.real * u2i.real + a.imag * u2i.imag, "spP": np.abs(self.p) ** 2}

    def cfl(self):
        g = self.g
        um = max(np.abs(self.to_phys(self.u1[:, jj])).max() for jj in range(g.nyu))
        wm = max(np.abs(self.to_phys(self.u3[:, jj])).max() for jj in range(g.nyu))
        vm = max([1e-6] + [np.abs(self.to_phys(self.u2[:, jj])).max() * g.dthdyv[jj] for jj in range(1, g.nyv - 1)])
        t = np.array([1.0 / (self.cfg.alp * (self.n1 // 2) * um), 1.0 / (self.cfg.bet * (self.n2 // 2) * wm), 1.0 / vm])
        return min(t[0], t[1]), t

    def _ib(self, u, rhs, lst, j0, n):
        if lst is None:
            return
        planes = []
        for s in range(2):
            for j in range(max(lst.jlo[s], j0 + 1), min(lst.jhi[s], j0 + n - 2) + 1):
                if j not in planes:
                    planes.append(j)
        if not planes:
            return
        R = {j: self.to_phys(rhs[:, j - j0]) for j in planes}
        Uv = {j: self.to_phys(u[:, j - j0]) for j in planes}
        for p in range(lst.n):
            i, k, j, i2, k2, j2, i3, k3, j3 = (int(x) for x in lst.idx[p])
            lap, w2, w3 = lst.w[p]
            vf = w2 * Uv[j2][k2 - 1, i2 - 1] + w3 * Uv[j3][k3 - 1, i3 - 1]
            R[j][k - 1, i - 1] = lap * (vf - Uv[j][k - 1, i - 1] + R[j][k - 1, i - 1])
        for j in planes:
            rhs[:, j - j0] = self.to_spec(R[j])

    @staticmethod
    def _thomas(a1, a2, a3, r):
        # LU_dec + substitution over all columns (a*: [ncol, n])
        a2 = a2.copy()
        a3 = a3.copy()
        n = r.shape[1]
        a2[:, 0] = 1.0 / a2[:, 0]
        for j in range(1, n):
            a3[:, j - 1] = a3[:, j - 1] * a2[:, j - 1]
            a2[:, j] = 1.0 / (a2[:, j] - a1[:, j] * a3[:, j - 1])
        x = np.empty_like(r)
        x[:, 0] = r[:, 0] * a2[:, 0]
        for j in range(1, n):
            x[:, j] = (r[:, j] - a1[:, j] * x[:, j - 1]) * a2[:, j]
        for j in range(n - 2, -1, -1):
            x[:, j] = x[:, j] - a3[:, j] * x[:, j + 1]
        return x

    def solve_uvw(self, krk):
        g, dt = self.g, self.dt
        beta = B[krk - 1] * dt / self.re
        for u, du in ((self.u1, self.du1), (self.u3, self.du3)):
            du[:, 0] = 0
            du[:, 1:-1] = u[:, 1:-1] + dt * du[:, 1:-1]
            du[:, -1] = 0
        self.du2[:, 0] = 0
        self.du2[:, 1:-1] = self.u2[:, 1:-1] + dt * self.du2[:, 1:-1]
        self.du2[:, -1] = 0
        self._ib(self.u1, self.du1, self.ibu, g.ju0, g.nyu)
        self._ib(self.u2, self.du2, self.ibv, g.jv0, g.nyv)
        self._ib(self.u3, self.du3, self.ibu, g.ju0, g.nyu)
        n = g.nyu
        a1 = np.zeros((self.ncol, n)); a2 = np.zeros((self.ncol, n)); a3 = np.zeros((self.ncol, n))
        a2[:, 0], a3[:, 0] = 1.0, self.gwb
        a1[:, 1:-1] = -beta * g.dyu2i[None, 1:-1, 0]
        a2[:, 1:-1] = 1.0 - beta * ((g.dyu2i[None, 1:-1, 1] + (-(self.kx ** 2))[:, None]) + (-(self.kz ** 2))[:, None])
        a3[:, 1:-1] = -beta * g.dyu2i[None, 1:-1, 2]
        a1[:, -1], a2[:, -1] = self.gwt, 1.0
        self.u1[:] = self._thomas(a1, a2, a3, self.du1)
        self.u3[:] = self._thomas(a1, a2, a3, self.du3)
        n = g.nyv
        a1 = np.zeros((self.ncol, n)); a2 = np.ones((self.ncol, n)); a3 = np.zeros((self.ncol, n))
        a1[:, 1:-1] = -beta * g.dyv2i[None, 1:-1, 0]
        a2[:, 1:-1] = 1.0 - beta * ((g.dyv2i[None, 1:-1, 1] + (-(self.kx ** 2))[:, None]) + (-(self.kz ** 2))[:, None])
        a3[:, 1:-1] = -beta * g.dyv2i[None, 1:-1, 2]
        self.u2[:] = self._thomas(a1, a2, a3, self.du2)

    def _flowrate(self, col0):
        g = self.g
        d = g.dny
        nn = g.ny - 2
        return sum((g.yv[j + d] - g.yv[j - 1 + d]) * col0[j + d].real for j in range(1, nn + 2))

    def meanflow(self, krk):
        g = self.g
        if self.ctp == 1:
            self.Qx = self._flowrate(self.u1[0])
            return
        d = g.dny
        nn = g.ny - 2
        n = nn + 3
        beta = B[krk - 1] * self.dt / self.re
        a1, a2, a3 = np.zeros((1, n)), np.zeros((1, n)), np.zeros((1, n))
        a2[0, 0], a3[0, 0] = 1.0, self.gwb
        for j in range(1, nn + 2):
            c = g.dyu2i[j + d]
            a1[0, j], a2[0, j], a3[0, j] = -beta * c[0], 1.0 - beta * c[1], -beta * c[2]
        a1[0, -1], a2[0, -1] = self.gwt, 1.0
        r = np.zeros((1, n))
        r[0, 1:nn + 2] = -D[krk - 1] * self.dt
        x = self._thomas(a1, a2, a3, r)[0]
        qx1 = sum((g.yv[j + d] - g.yv[j - 1 + d]) * x[j] for j in range(1, nn + 2))
        gg = (self.qxt - self._flowrate(self.u1[0])) / qx1
        self.mpgx += gg
        for j in range(0, nn + 3):
            self.u1[0, j + d] += gg * x[j]

    def divergence(self):
        g = self.g
        return (1j * self.kx[:, None] * self.u1[:, 1:-1] + 1j * self.kz[:, None] * self.u3[:, 1:-1] +
                g.dthdyu[None, 1:-1] * (self.u2[:, 1:] - self.u2[:, :-1]))

    def solve_p(self, krk):
        g = self.g
        dtirk = (1.0 / self.dt) / (A[krk - 1] + B[krk - 1])
        self.div = self.divergence()
        r = dtirk * self.div
        r[0, 0] = 0.0
        n = g.nyp
        du = g.dthdyu[1:-1]          # dthdyu(j), j = jp0..jp1
        dvm = g.dthdyv[:-1]          # dthdyv(j-1)
        dvp = g.dthdyv[1:]           # dthdyv(j)
        a1 = np.zeros((self.ncol, n)); a2 = np.zeros((self.ncol, n)); a3 = np.zeros((self.ncol, n))
        k2x, k2z = -(self.kx ** 2)[:, None], -(self.kz ** 2)[:, None]
        a2[:, 0:1] = (du[0] * -dvp[0]) + k2x + k2z
        a3[:, 0] = du[0] * dvp[0]
        a2[:, -1:] = ((-du[-1]) * dvm[-1]) + k2x + k2z
        a1[:, -1] = (-du[-1]) * (-dvm[-1])
        mid = slice(1, n - 1)
        a2[:, mid] = (((-du[mid]) * dvm[mid]) + (du[mid] * -dvp[mid]))[None, :] + k2x + k2z
        a1[:, mid] = ((-du[mid]) * (-dvm[mid]))[None, :]
        a3[:, mid] = (du[mid] * dvp[mid])[None, :]
        a1[0, 0], a2[0, 0], a3[0, 0] = 0.0, 1.0 / (g.u(2) - g.u(1)) ** 2, 0.0
        self.psi = self._thomas(a1, a2, a3, r)
        self.p = self.p + self.psi

    def vcorr(self, krk):
        g = self.g
        dtrk = self.dt * (A[krk - 1] + B[krk - 1])
        self.u1[:, 1:-1] -= (dtrk * 1j * self.kx)[:, None] * self.psi
        self.u3[:, 1:-1] -= (dtrk * 1j * self.kz)[:, None] * self.psi
        for u in (self.u1, self.u3):
            u[:, 0] = -self.gwb * u[:, 1]
            u[:, -1] = -self.gwt * u[:, -2]
        self.u2[:, 1:-1] -= dtrk * g.dthdyv[None, 1:-1] * (self.psi[:, 1:] - self.psi[:, :-1])
        self.u2[:, 0] = 0
        self.u2[:, -1] = 0
        self.div = self.divergence()

    def rk_substep(self, krk):
        self.rhs0(krk)
        self.nonlinear(krk)
        self.solve_uvw(krk)
        if self.ctp == 0:
            self.meanflow(krk)
        self.solve_p(krk)
        self.vcorr(krk)

    def step(self, n=1):
        for _ in range(n):
            for k in (1, 2, 3):
                self.rk_substep(k)
            if self.ctp == 1:
                self.meanflow(1)

    def upload_state(self, st):
        for k in ("u1", "u2", "u3", "p"):
            setattr(self, k, np.array(st[k], dtype=np.complex128))

    def download_state(self):
        return {k: getattr(self, k).copy() for k in ("u1", "u2", "u3", "p")}
