"""The C-ABI library loads and exports every symbol include/uppe_b200.h declares (CPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, 'include', 'uppe_b200.h')).read()
    src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
    return sorted(set(re.findall(r'\b(uppe\w+)\s*\(', src)))


def test_library_exports_header_symbols():
    from project_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    names = declared_symbols()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_header():
    from project_b200 import _lib
    names = set(declared_symbols())
    assert names <= set(_lib.SIGNATURES), names - set(_lib.SIGNATURES)


def test_plan_rejects_bad_sizes_without_gpu_work():
    """Size validation happens before any CUDA call."""
    from project_b200 import _lib, build
    lib = ctypes.CDLL(build.build())
    for name, (res, args) in _lib.SIGNATURES.items():
        getattr(lib, name).restype = res
        getattr(lib, name).argtypes = args
    d = _lib.Desc3D()
    d.Nx, d.Ny, d.Nt, d.precision = 100, 128, 512, 0
    plan = ctypes.c_void_p()
    assert lib.uppe3d_plan_create(ctypes.byref(d), ctypes.byref(plan)) == -2
    assert b'power' in lib.uppe_last_error()
