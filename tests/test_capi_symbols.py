"""The C-ABI library loads and exports every function declared in include/cfd_b200.h
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from cfd_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "cfd_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cfd_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header():
    lib = ctypes.CDLL(capi.LIB_PATH)
    names = declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header():
    assert set(declared()) <= set(capi.SIGNATURES)


def test_version_string():
    lib = capi.load()
    assert lib.cfd_version().decode().startswith("cfd_b200")


def test_struct_layout_matches_header():
    # 4 int32 + 6 double + 2 int32 + 6 pointers on LP64
    # 4 ints, 6 doubles, 2 ints, 6 pointers, 3 ints (the band fields) + 4 bytes of tail padding
    assert ctypes.sizeof(capi.CfdConfig) == 16 + 48 + 8 + 48 + 12 + 4
    assert capi.CfdConfig.band_vface.offset == 16 + 48 + 8 + 48 + 8
    assert ctypes.sizeof(capi.CfdIBList) == 8 + 8 + 8 + 16
