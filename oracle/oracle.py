"""ctypes wrapper of the C++ FP64 oracle (oracle/cfd_oracle.cpp).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg, as the checker and the timed CPU baseline - never by the product.
Parity is unpinned by the reference's own tests (it has none and cannot be compiled
here); see cfd_oracle.cpp for how the oracle is pinned instead.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libcfd_oracle.so")
_dp = C.POINTER(C.c_double)


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "cfd_oracle.cpp")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE, "-B" if force else "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_last_error.restype = C.c_char_p
        for n in ("orc_set_field", "orc_get_field"):
            getattr(L, n).argtypes = [C.c_void_p, C.c_int, _dp]
        for n in ("orc_rhs0", "orc_nonlinear", "orc_solve_uvw", "orc_meanflow", "orc_solve_p",
                  "orc_vcorr", "orc_rk_substep", "orc_step", "orc_set_quirk"):
            getattr(L, n).argtypes = [C.c_void_p, C.c_int]
        L.orc_get_scalars.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_rft.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_cft.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_four_to_phys.argtypes = [C.c_void_p, _dp, C.c_int, C.c_int]
        L.orc_phys_to_four.argtypes = [C.c_void_p, _dp, C.c_int]
        L.orc_set_num_threads.argtypes = [C.c_int]
        L.orc_stats_configure.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_spectra_read.argtypes = [C.c_void_p] + [C.c_void_p] * 5
        L.orc_stats_accumulate.argtypes = [C.c_void_p]
        L.orc_stats_read.argtypes = [C.c_void_p] + [C.c_void_p] * 6 + [C.POINTER(C.c_int)]
        L.orc_cfl.argtypes = [C.c_void_p, _dp, C.c_void_p]
        L.orc_set_dt.argtypes = [C.c_void_p, C.c_double]
        _lib = L
    return _lib


FIELD_IDS = {"u1": 0, "u2": 1, "u3": 2, "p": 3, "nu1": 4, "nu2": 5, "nu3": 6, "div": 7,
             "psi": 8, "du1": 9, "du2": 10, "du3": 11}


def rft(c: np.ndarray, n: int, isa: int, m: int, iopt: int) -> np.ndarray:
    """The reference's rft on a flat float64 array (in place, returned)."""
    c = np.ascontiguousarray(c, dtype=np.float64)
    st = lib().orc_rft(c.ctypes.data_as(_dp), n, isa, m, iopt)
    assert st == 0, lib().orc_last_error()
    return c


def cft(c: np.ndarray, n: int, ise: int, isa: int, m: int, iopt: int) -> np.ndarray:
    c = np.ascontiguousarray(c, dtype=np.float64)
    st = lib().orc_cft(c.ctypes.data_as(_dp), n, ise, isa, m, iopt)
    assert st == 0, lib().orc_last_error()
    return c


def set_threads(n: int):
    lib().orc_set_num_threads(int(n))


class OracleChannel:
    """Same stage interface as cfd_b200.channel.Channel, computed on the CPU in FP64."""

    def __init__(self, setup, quirk_lastplane: bool = False):
        from cfd_b200 import capi
        self.setup = setup
        self._keep = []
        c = capi.make_config(setup.cfg.with_(precision="fp64"), setup.grid, setup.dt, self._keep)
        ibu = capi.make_iblist(setup.ibu, self._keep)
        ibv = capi.make_iblist(setup.ibv, self._keep)
        self._cfg = c
        self.h = lib().orc_create(C.addressof(c), C.addressof(ibu) if ibu else None,
                                  C.addressof(ibv) if ibv else None)
        if not self.h:
            raise RuntimeError(lib().orc_last_error().decode())
        if quirk_lastplane:
            lib().orc_set_quirk(self.h, 1)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _n(self, name):
        from cfd_b200.channel import field_planes
        return field_planes(self.setup, name)

    def upload(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.complex128)
        assert a.shape == (self.setup.cfg.ncol, self._n(name)), (name, a.shape)
        lib().orc_set_field(self.h, FIELD_IDS[name], a.ctypes.data_as(_dp))

    def download(self, name):
        out = np.empty((self.setup.cfg.ncol, self._n(name)), np.complex128)
        lib().orc_get_field(self.h, FIELD_IDS[name], out.ctypes.data_as(_dp))
        return out

    def upload_state(self, state=None):
        st = state if state is not None else self.setup.state()
        for k in ("u1", "u2", "u3", "p"):
            self.upload(k, st[k])

    def download_state(self):
        return {k: self.download(k) for k in ("u1", "u2", "u3", "p")}

    def rhs0(self, krk): lib().orc_rhs0(self.h, krk)
    def nonlinear(self, krk): lib().orc_nonlinear(self.h, krk)
    def solve_uvw(self, krk): lib().orc_solve_uvw(self.h, krk)
    def meanflow(self, krk): lib().orc_meanflow(self.h, krk)
    def solve_p(self, krk): lib().orc_solve_p(self.h, krk)
    def vcorr(self, krk): lib().orc_vcorr(self.h, krk)
    def rk_substep(self, krk): lib().orc_rk_substep(self.h, krk)
    def step(self, n=1): lib().orc_step(self.h, n)

    def scalars(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        lib().orc_get_scalars(self.h, C.byref(a), C.byref(b), C.byref(c))
        return {"mpgx": a.value, "qx": b.value, "dgx": c.value}

    # statistics (stats.f90) and dtc_calc, same interface as Channel
    def stats_configure(self, jband: int, dnx: int, dnz: int, spectra: bool = True):
        from cfd_b200 import capi
        st = lib().orc_stats_configure(self.h, int(jband), int(dnx), int(dnz), int(bool(spectra)))
        assert st == 0, "bad statistics tile"
        g = self.setup.grid
        self._stats_shape = capi.stats_band(g.nyu, g.nyv, g.nyp, int(jband), g.ju0, g.jv0, g.jp0) + \
            ((int(dnx), int(dnz)) if jband >= g.jv0 else (0, 0))

    def stats_accumulate(self):
        assert lib().orc_stats_accumulate(self.h) == 0

    def spectra_read(self) -> dict:
        from cfd_b200 import capi
        g = self.setup.grid
        bufs = capi.spectra_buffers(self.setup.cfg.ncol, g.nyu, g.nyv, g.nyp)
        assert lib().orc_spectra_read(self.h, *[b.ctypes.data for b in bufs.values()]) == 0, "spectra not configured"
        return bufs

    def stats_read(self) -> dict:
        from cfd_b200 import capi
        g = self.setup.grid
        nbu, nbv, nbp, dnx, dnz = self._stats_shape
        bufs = capi.stats_buffers(g.nyu, g.nyv, g.nyp, nbu, nbv, nbp, dnx, dnz)
        ist = C.c_int()
        lib().orc_stats_read(self.h, *[b.ctypes.data for b in bufs], C.byref(ist))
        return capi.stats_dict(bufs, ist.value)

    def set_dt(self, dt: float):
        assert lib().orc_set_dt(self.h, float(dt)) == 0

    def cfl(self):
        dtc = C.c_double()
        t = np.zeros(3)
        lib().orc_cfl(self.h, C.byref(dtc), t.ctypes.data)
        return dtc.value, t

    def four_to_phys(self, planes: np.ndarray, zero_oddball: bool = False) -> np.ndarray:
        p = np.ascontiguousarray(planes, dtype=np.float64)
        lib().orc_four_to_phys(self.h, p.ctypes.data_as(_dp), p.shape[0], int(zero_oddball))
        return p

    def phys_to_four(self, planes: np.ndarray) -> np.ndarray:
        p = np.ascontiguousarray(planes, dtype=np.float64)
        lib().orc_phys_to_four(self.h, p.ctypes.data_as(_dp), p.shape[0])
        return p
