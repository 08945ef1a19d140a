"""C-ABI: the library builds, loads without a GPU and exports every entry
point that include/psod.h declares."""

import ctypes as C
import os
import re

from psod_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "psod.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(psod_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header():
    path = build.build()
    lib = C.CDLL(path)
    names = header_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(capi.EXPORTS)


def test_abi_version_and_strings():
    lib = capi.load()
    assert lib.psod_abi_version() == 4
    assert b"nsel" in lib.psod_status_string(capi.ERR_NSEL)
    assert lib.psod_status_string(capi.OK) == b"ok"


def test_params_default_match_reference():
    p = capi.default_params(128)
    assert p.nmin == 100 and p.delta == 200.0 and p.delta2 == 800.0  # main:110-112
    assert p.ncut == 4 and p.nsel == 4000000 and p.nxbuffer == 0  # main:114
    assert p.nbins == 60 and p.rbin_lo == 0.01 and p.rbin_hi == 1.0  # main:1414, 2105


def test_create_without_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        return
    lib = capi.load()
    p = capi.default_params(16)
    h = C.c_void_p()
    assert lib.psod_ctx_create(C.byref(p), C.byref(h)) == capi.ERR_CUDA


def test_invalid_params_rejected():
    lib = capi.load()
    h = C.c_void_p()
    for kw in ({"ncut": 9}, {"nmin": 5}, {"nbins": 0}, {"nxbuffer": 2, "ncut": 4}, {"nxbuffer": 16}):
        p = capi.default_params(16, **kw)
        assert lib.psod_ctx_create(C.byref(p), C.byref(h)) == capi.ERR_ARG
