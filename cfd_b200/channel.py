"""Host-side driver of the B200 hot path, mirroring the reference's main loop.

``Channel`` exposes the subroutine entry points of littleharsh.f90 (RHS0_u1..3,
nonlinear, solveU/solveV, meanflow_ctU/ctP, solveP, v_corr; littleharsh.f90:163-196)
over the C ABI of ``libcfdb200.so``.  State lives on the GPU; host arrays use the
reference's cfield layout f(j,column) as complex128 arrays of shape [column, plane].

``build_channel`` produces everything the step consumes from a ChannelConfig: the
y-grid, the IB lists, the seeded initial fields and the fixed time step.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import capi
from .config import ChannelConfig
from .geometry import IBList, ib_lists
from .grid import YGrid, y_grid_rough
from .initial import cfl_dt, initial_state, viscous_dt


@dataclass
class ChannelSetup:
    cfg: ChannelConfig
    grid: YGrid
    ibu: IBList
    ibv: IBList
    dt: float
    u1: np.ndarray
    u2: np.ndarray
    u3: np.ndarray
    p: np.ndarray

    def state(self):
        return {"u1": self.u1, "u2": self.u2, "u3": self.u3, "p": self.p}

    @property
    def grid_points(self) -> int:
        """Ngal1 * Ngal2 * ny_tot (faces, walls included) - the unit of grid-pt updates."""
        return self.cfg.ngal1 * self.cfg.ngal2 * self.grid.nyv


def build_channel(cfg: ChannelConfig, with_fields: bool = True) -> ChannelSetup:
    grid = y_grid_rough(cfg.ny, cfg.dyq, cfg.ppp, cfg.posth)
    ibu, ibv = ib_lists(cfg, grid)
    if with_fields:
        u1, u2, u3, p = initial_state(cfg, grid)
        # three bands: the short columns start from zero outside their segments
        from .bands import restrict
        u1, u3 = restrict(cfg, grid, u1, "u"), restrict(cfg, grid, u3, "u")
        u2, p = restrict(cfg, grid, u2, "v"), restrict(cfg, grid, p, "p")
        dt = cfg.dt if cfg.dt is not None else cfl_dt(cfg, grid, u1, u2, u3)
    else:
        u1 = u2 = u3 = p = None
        dt = cfg.dt if cfg.dt is not None else 1e-4
    return ChannelSetup(cfg=cfg, grid=grid, ibu=ibu, ibv=ibv, dt=float(dt),
                        u1=u1, u2=u2, u3=u3, p=p)


def field_planes(setup: ChannelSetup, name: str) -> int:
    g = setup.grid
    return {"u1": g.nyu, "u3": g.nyu, "nu1": g.nyu, "nu3": g.nyu, "du1": g.nyu, "du3": g.nyu,
            "u2": g.nyv, "nu2": g.nyv, "du2": g.nyv,
            "p": g.nyp, "div": g.nyp, "psi": g.nyp}[name]


class Channel:
    """One channel on one GPU, driven through the C ABI."""

    def __init__(self, setup: ChannelSetup, device: int = 0, precision: Optional[str] = None,
                 tuning=None):
        """tuning: None (library defaults), a dict of cfd_tuning fields, or "auto" (the
        cached or freshly measured choice of cfd_b200.autotune for this grid and GPU)."""
        self.setup = setup
        self.lib = capi.load()
        self._keep = []
        cfg = setup.cfg if precision is None else setup.cfg.with_(precision=precision)
        self.cfg = cfg
        if tuning == "auto":
            from .autotune import tuned
            tuning = tuned(setup, cfg.precision, device)
        c = capi.make_config(cfg, setup.grid, setup.dt, self._keep)
        ibu = capi.make_iblist(setup.ibu, self._keep)
        ibv = capi.make_iblist(setup.ibv, self._keep)
        ctx = C.c_void_p()
        tun = capi.CfdTuning(**tuning) if tuning else None
        st = self.lib.cfd_create_tuned(C.byref(c), C.byref(ibu) if ibu else None,
                                       C.byref(ibv) if ibv else None, device,
                                       C.byref(tun) if tun else None, C.byref(ctx))
        if st != capi.CFD_OK:
            msg = self.lib.cfd_last_error(ctx).decode() if ctx else ""
            if ctx:
                self.lib.cfd_destroy(ctx)
            raise capi.CfdError(f"cfd_create failed: {capi.ERRORS.get(st, st)}: {msg}")
        self.ctx = ctx

    # -- lifetime -----------------------------------------------------------------------
    def close(self):
        if getattr(self, "ctx", None):
            self.lib.cfd_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st, what):
        capi.check(self.lib, self.ctx, st, what)

    # -- state ----------------------------------------------------------------------------
    def upload(self, name: str, arr: np.ndarray, layout: int = capi.LAYOUT_REF):
        a = np.ascontiguousarray(arr, dtype=np.complex128)
        self._chk(self.lib.cfd_upload_field(self.ctx, capi.FIELDS[name],
                                            a.ctypes.data_as(C.POINTER(C.c_double)), layout),
                  f"upload {name}")
        self.synchronize()

    def download(self, name: str, layout: int = capi.LAYOUT_REF) -> np.ndarray:
        n = field_planes(self.setup, name)
        out = np.empty((self.cfg.ncol, n) if layout == capi.LAYOUT_REF else (n, self.cfg.ncol),
                       np.complex128)
        self._chk(self.lib.cfd_download_field(self.ctx, capi.FIELDS[name],
                                              out.ctypes.data_as(C.POINTER(C.c_double)), layout),
                  f"download {name}")
        self.synchronize()
        return out

    def upload_state(self, state=None):
        st = state if state is not None else self.setup.state()
        for k in ("u1", "u2", "u3", "p"):
            self.upload(k, st[k])

    def download_state(self):
        return {k: self.download(k) for k in ("u1", "u2", "u3", "p")}

    def save_record_out(self, directory: str, tag: str, t: float = 0.0, it: int = 0, nband: int = 3):
        """Write the state in the reference's record_out format (cfd_b200.checkpoint)."""
        from .checkpoint import write_record_out
        return write_record_out(directory, tag, self.download_state(), self.setup, t=t, it=it,
                                mpgx=self.scalars()["mpgx"], nband=nband)

    def load_record_out(self, directory: str, tag: str) -> dict:
        """Upload a state from record_out files (read_in's role); returns their header."""
        from .checkpoint import read_record_out
        data = read_record_out(directory, tag, self.setup)
        self.upload_state({k: data[k] for k in ("u1", "u2", "u3", "p")})
        return data["header"]

    def synchronize(self):
        self._chk(self.lib.cfd_synchronize(self.ctx), "synchronize")

    def device_ptr(self, name: str) -> int:
        p = C.c_void_p()
        self._chk(self.lib.cfd_field_device_ptr(self.ctx, capi.FIELDS[name], C.byref(p)), "ptr")
        return p.value

    def set_stream(self, stream_handle: int):
        self._chk(self.lib.cfd_set_stream(self.ctx, C.c_void_p(stream_handle)), "set_stream")

    # -- the step (littleharsh.f90:163-196) -----------------------------------------------
    def rhs0(self, krk: int):
        self._chk(self.lib.cfd_rhs0(self.ctx, krk), "rhs0")

    def nonlinear(self, krk: int):
        self._chk(self.lib.cfd_nonlinear(self.ctx, krk), "nonlinear")

    def solve_uvw(self, krk: int):
        self._chk(self.lib.cfd_solve_uvw(self.ctx, krk), "solve_uvw")

    def meanflow(self, krk: int):
        self._chk(self.lib.cfd_meanflow(self.ctx, krk), "meanflow")

    def solve_p(self, krk: int):
        self._chk(self.lib.cfd_solve_p(self.ctx, krk), "solve_p")

    def vcorr(self, krk: int):
        self._chk(self.lib.cfd_vcorr(self.ctx, krk), "vcorr")

    def rk_substep(self, krk: int):
        self._chk(self.lib.cfd_rk_substep(self.ctx, krk), "rk_substep")

    def step(self, nsteps: int = 1):
        self._chk(self.lib.cfd_step(self.ctx, nsteps), "step")

    def scalars(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        self._chk(self.lib.cfd_get_scalars(self.ctx, C.byref(a), C.byref(b), C.byref(c)),
                  "scalars")
        return {"mpgx": a.value, "qx": b.value, "dgx": c.value}

    # -- statistics and CFL (stats.f90, dtc_calc) ------------------------------------------
    def stats_configure(self, jband: int, dnx: int, dnz: int, spectra: bool = True):
        """Configure and zero the FP64 statistics accumulators (bottom band up to v plane
        jband, tiles of dnx x dnz points; jband below the first v plane: plane sums only),
        and with spectra the spectra of spectra.f90, which the reference always takes."""
        sc = capi.CfdStatsConfig(int(jband), int(dnx), int(dnz), int(bool(spectra)))
        self._chk(self.lib.cfd_stats_configure(self.ctx, C.byref(sc)), "stats_configure")
        g = self.setup.grid
        self._stats_shape = capi.stats_band(g.nyu, g.nyv, g.nyp, int(jband), g.ju0, g.jv0, g.jp0) + \
            ((int(dnx), int(dnz)) if jband >= g.jv0 else (0, 0))

    def stats_accumulate(self):
        self._chk(self.lib.cfd_stats_accumulate(self.ctx), "stats_accumulate")

    def stats_reset(self):
        self._chk(self.lib.cfd_stats_reset(self.ctx), "stats_reset")

    def stats_read(self) -> dict:
        g = self.setup.grid
        nbu, nbv, nbp, dnx, dnz = self._stats_shape
        bufs = capi.stats_buffers(g.nyu, g.nyv, g.nyp, nbu, nbv, nbp, dnx, dnz)
        ist = C.c_int32()
        self._chk(self.lib.cfd_stats_read(self.ctx, *[b.ctypes.data for b in bufs], C.byref(ist)),
                  "stats_read")
        return capi.stats_dict(bufs, ist.value)

    def spectra_read(self) -> dict:
        """The accumulated spectra spU, spV, spW, spUV, spP as (columns, planes) arrays, the
        reference's sp(j,column) layout."""
        g = self.setup.grid
        bufs = capi.spectra_buffers(self.setup.cfg.ncol, g.nyu, g.nyv, g.nyp)
        self._chk(self.lib.cfd_spectra_read(self.ctx, *[b.ctypes.data for b in bufs.values()]), "spectra_read")
        return bufs

    def cfl(self):
        """(dtc, [u term, w term, v term]) of dtc_calc on the current state."""
        dtc = C.c_double()
        t = np.zeros(3)
        self._chk(self.lib.cfd_cfl(self.ctx, C.byref(dtc), t.ctypes.data), "cfl")
        return dtc.value, t

    def tuning(self) -> dict:
        """Launch shapes this context runs with (cfd_get_tuning)."""
        t = capi.CfdTuning()
        self._chk(self.lib.cfd_get_tuning(self.ctx, C.byref(t)), "get_tuning")
        return t.as_dict()

    def adapt_dt(self) -> float:
        """The reference's time-step rule (FOU3D.f90:178-181), dt = min(2.5 dtv, CFL dtc)
        with dtc from dtc_calc on the current state and dtv of start.f90:432; the new dt is
        set (the step graph is captured again) and returned.  The reference applies it at
        the start of every step; a caller that re-captures less often applies it every few
        steps."""
        dtc, _ = self.cfl()
        cfg = self.setup.cfg
        dt = min(2.5 * viscous_dt(cfg, self.setup.grid), cfg.cfl * dtc)
        self.set_dt(dt)
        return dt

    def set_dt(self, dt: float):
        """New time step for the following stages and steps (the graph is captured again)."""
        self._chk(self.lib.cfd_set_dt(self.ctx, float(dt)), "set_dt")

    def set_lastplane(self, on: bool):
        """Single-slab (bug-compatible) x/z advective term of the reference's ops_in_planes
        (on) or the per-plane term (off, the default)."""
        self._chk(self.lib.cfd_set_lastplane(self.ctx, int(bool(on))), "set_lastplane")

    def divergence_max(self) -> float:
        e = C.c_double()
        self._chk(self.lib.cfd_divergence_max(self.ctx, C.byref(e)), "divergence_max")
        return e.value

    def launch_count(self) -> int:
        n = C.c_int64()
        self._chk(self.lib.cfd_launch_count(self.ctx, C.byref(n)), "launch_count")
        return n.value
