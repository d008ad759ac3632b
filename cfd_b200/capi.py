"""ctypes binding of the C ABI declared in include/cfd_b200.h.

This is the binding a Python driver (or a test) uses; a Fortran driver binds the same
symbols with iso_c_binding.  The shared library is built in-tree by
``cfd_b200._build.build_library`` and must exist: there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libcfdb200.so")

CFD_OK = 0
ERRORS = {1: "CFD_ERR_ARG", 2: "CFD_ERR_SIZE", 3: "CFD_ERR_CUDA", 4: "CFD_ERR_NONFINITE",
          5: "CFD_ERR_STATE", 6: "CFD_ERR_NOMEM"}
PREC = {"fp64": 0, "mixed": 1}
FIELDS = {"u1": 0, "u2": 1, "u3": 2, "p": 3, "nu1": 4, "nu2": 5, "nu3": 6, "div": 7,
          "psi": 8, "du1": 9, "du2": 10, "du3": 11}
LAYOUT_REF, LAYOUT_PLANE = 0, 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class CfdConfig(C.Structure):
    _fields_ = [("ngal1", C.c_int32), ("ngal2", C.c_int32), ("ny", C.c_int32),
                ("dsty", C.c_int32), ("re", C.c_double), ("alp", C.c_double),
                ("bet", C.c_double), ("dt", C.c_double), ("mpgx", C.c_double),
                ("qxt", C.c_double), ("flag_ctpress", C.c_int32), ("precision", C.c_int32),
                ("yu", _dp), ("yv", _dp), ("dthdyu", _dp), ("dthdyv", _dp),
                ("dyu2i", _dp), ("dyv2i", _dp),
                ("ngal1_mid", C.c_int32), ("ngal2_mid", C.c_int32), ("band_vface", C.c_int32)]


class CfdIBList(C.Structure):
    _fields_ = [("n", C.c_int32), ("idx", _ip), ("w", _dp),
                ("jlo", C.c_int32 * 2), ("jhi", C.c_int32 * 2)]


class CfdTuning(C.Structure):
    _fields_ = [("xline_path", C.c_int32), ("xline_rows", C.c_int32), ("zlines", C.c_int32),
                ("solve_kind", C.c_int32), ("solve_cols", C.c_int32), ("rhs_chunk", C.c_int32),
                ("xsplit", C.c_int32), ("zsplit", C.c_int32)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class CfdStatsConfig(C.Structure):
    _fields_ = [("jband", C.c_int32), ("dnx", C.c_int32), ("dnz", C.c_int32), ("spectra", C.c_int32)]


def dptr(a):
    return a.ctypes.data_as(_dp)


# statistics quantities in the order of cfd_stats_read (stats.f90:1-106)
STATS_U = ("Um", "U2m", "Wm", "W2m", "UVm", "UWm")
STATS_V = ("Vm", "V2m", "wxm", "wx2m", "VWm")
STATS_P = ("Pm", "P2m")


def stats_buffers(nyu, nyv, nyp, nbu, nbv, nbp, dnx, dnz):
    """Host arrays for cfd_stats_read / orc_stats_read."""
    import numpy as np
    return (np.zeros((6, nyu)), np.zeros((5, nyv)), np.zeros((2, nyp)),
            np.zeros((6, nbu, dnz, dnx)), np.zeros((5, nbv, dnz, dnx)), np.zeros((2, nbp, dnz, dnx)))


SPECTRA = ("spU", "spV", "spW", "spUV", "spP")


def spectra_buffers(ncol, nyu, nyv, nyp):
    """Host arrays for cfd_spectra_read / orc_spectra_read, sp(j,column): [column][plane]."""
    import numpy as np
    return {"spU": np.zeros((ncol, nyu)), "spV": np.zeros((ncol, nyv)), "spW": np.zeros((ncol, nyu)),
            "spUV": np.zeros((ncol, nyu)), "spP": np.zeros((ncol, nyp))}


def stats_dict(bufs, istat):
    """Name the arrays of stats_buffers: plane sums by quantity, conditional sums as <name>C."""
    su, sv, sp, cu, cv, cp = bufs
    out = {"istat": istat}
    for names, a, c in ((STATS_U, su, cu), (STATS_V, sv, cv), (STATS_P, sp, cp)):
        for q, n in enumerate(names):
            out[n] = a[q].copy()
            out[n + "C"] = c[q].copy()
    return out


def stats_band(nyu, nyv, nyp, jband, j0u, j0v, j0p):
    """Planes of the bottom band (and of the mirrored top band) for a band ending at v plane
    jband: u planes j0u..jband+1, v planes j0v..jband, p planes j0p..jband."""
    if jband < j0v:
        return 0, 0, 0
    return jband + 1 - j0u + 1, jband - j0v + 1, jband - j0p + 1


def make_config(cfg, grid, dt, keep: list) -> CfdConfig:
    """Fill the C struct from a ChannelConfig and YGrid; `keep` holds the arrays alive."""
    import numpy as np
    arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in
            (grid.yu, grid.yv, grid.dthdyu, grid.dthdyv, grid.dyu2i, grid.dyv2i)]
    keep.extend(arrs)
    c = CfdConfig()
    c.ngal1, c.ngal2, c.ny, c.dsty = cfg.ngal1, cfg.ngal2, cfg.ny, grid.dny
    c.re, c.alp, c.bet, c.dt = cfg.re_b, cfg.alp, cfg.bet, dt
    c.mpgx, c.qxt, c.flag_ctpress = cfg.mpgx, cfg.qxt, cfg.flag_ctpress
    c.precision = PREC[cfg.precision]
    c.yu, c.yv, c.dthdyu, c.dthdyv, c.dyu2i, c.dyv2i = [dptr(a) for a in arrs]
    c.ngal1_mid = getattr(cfg, "ngal1_mid", 0) or cfg.ngal1
    c.ngal2_mid = getattr(cfg, "ngal2_mid", 0) or cfg.ngal2
    c.band_vface = getattr(cfg, "band_vface", 0)
    return c


def make_iblist(lst, keep: list):
    import numpy as np
    if lst is None:
        return None
    idx = np.ascontiguousarray(lst.idx, dtype=np.int32)
    w = np.ascontiguousarray(lst.w, dtype=np.float64)
    keep.extend([idx, w])
    s = CfdIBList()
    s.n = lst.n
    s.idx = idx.ctypes.data_as(_ip)
    s.w = dptr(w)
    s.jlo[0], s.jlo[1] = lst.jlo
    s.jhi[0], s.jhi[1] = lst.jhi
    return s


# exported symbols with their argument types (include/cfd_b200.h)
_VP = C.c_void_p
SIGNATURES = {
    "cfd_create": (C.c_int, [C.POINTER(CfdConfig), C.POINTER(CfdIBList), C.POINTER(CfdIBList),
                             C.c_int32, C.POINTER(_VP)]),
    "cfd_create_tuned": (C.c_int, [C.POINTER(CfdConfig), C.POINTER(CfdIBList), C.POINTER(CfdIBList),
                                   C.c_int32, C.POINTER(CfdTuning), C.POINTER(_VP)]),
    "cfd_get_tuning": (C.c_int, [_VP, C.POINTER(CfdTuning)]),
    "cfd_destroy": (C.c_int, [_VP]),
    "cfd_last_error": (C.c_char_p, [_VP]),
    "cfd_set_stream": (C.c_int, [_VP, _VP]),
    "cfd_synchronize": (C.c_int, [_VP]),
    "cfd_field_shape": (C.c_int, [_VP, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "cfd_upload_field": (C.c_int, [_VP, C.c_int32, _dp, C.c_int32]),
    "cfd_download_field": (C.c_int, [_VP, C.c_int32, _dp, C.c_int32]),
    "cfd_field_device_ptr": (C.c_int, [_VP, C.c_int32, C.POINTER(_VP)]),
    "cfd_rhs0": (C.c_int, [_VP, C.c_int32]),
    "cfd_nonlinear": (C.c_int, [_VP, C.c_int32]),
    "cfd_solve_uvw": (C.c_int, [_VP, C.c_int32]),
    "cfd_meanflow": (C.c_int, [_VP, C.c_int32]),
    "cfd_solve_p": (C.c_int, [_VP, C.c_int32]),
    "cfd_vcorr": (C.c_int, [_VP, C.c_int32]),
    "cfd_rk_substep": (C.c_int, [_VP, C.c_int32]),
    "cfd_step": (C.c_int, [_VP, C.c_int32]),
    "cfd_get_scalars": (C.c_int, [_VP, _dp, _dp, _dp]),
    "cfd_divergence_max": (C.c_int, [_VP, _dp]),
    "cfd_four_to_phys": (C.c_int, [_VP, _VP, C.c_int32, C.c_int32]),
    "cfd_phys_to_four": (C.c_int, [_VP, _VP, C.c_int32]),
    "cfd_rft": (C.c_int, [_VP, _VP, C.c_int32, C.c_int32, C.c_int32]),
    "cfd_cft": (C.c_int, [_VP, _VP, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "cfd_stats_configure": (C.c_int, [_VP, C.POINTER(CfdStatsConfig)]),
    "cfd_stats_accumulate": (C.c_int, [_VP]),
    "cfd_stats_reset": (C.c_int, [_VP]),
    "cfd_stats_read": (C.c_int, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, C.POINTER(C.c_int32)]),
    "cfd_spectra_read": (C.c_int, [_VP, _VP, _VP, _VP, _VP, _VP]),
    "cfd_cfl": (C.c_int, [_VP, _dp, _VP]),
    "cfd_set_dt": (C.c_int, [_VP, C.c_double]),
    "cfd_set_lastplane": (C.c_int, [_VP, C.c_int32]),
    "cfd_ensemble_create": (C.c_int, [C.POINTER(_VP), C.c_int32, C.POINTER(_VP)]),
    "cfd_ensemble_step": (C.c_int, [_VP, C.c_int32]),
    "cfd_ensemble_synchronize": (C.c_int, [_VP]),
    "cfd_ensemble_stream": (C.c_int, [_VP, C.POINTER(_VP)]),
    "cfd_ensemble_last_error": (C.c_char_p, [_VP]),
    "cfd_ensemble_destroy": (C.c_int, [_VP]),
    "cfd_launch_count": (C.c_int, [_VP, C.POINTER(C.c_int64)]),
    "cfd_profile": (C.c_int, [_VP, C.c_int32]),
    "cfd_profile_read": (C.c_int, [_VP, C.c_char_p, C.c_int32]),
    "cfd_lusol_u_noalloc": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                      _VP, _VP, _VP, _VP, _VP, _VP]),
    "cfd_version": (C.c_char_p, []),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library {path} is missing: run __graft_entry__.build() "
                           "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIB_PATH:
        _lib = lib
    return lib


class CfdError(RuntimeError):
    pass


def check(lib, ctx, status: int, what: str):
    if status != CFD_OK:
        msg = lib.cfd_last_error(ctx) if ctx else b""
        raise CfdError(f"{what}: {ERRORS.get(status, status)}: "
                       f"{msg.decode() if msg else ''}")
