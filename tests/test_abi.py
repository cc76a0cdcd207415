"""The C-ABI library builds, loads and exports what include/euvl_b200.h declares
(CPU: no compute is launched)."""
import ctypes as C
import os
import re

import pytest

from euvlitho_b200 import _lib as L
from euvlitho_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return L.lib()


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "euvl_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(euv_[a-z0-9_]+)\s*\(", txt)))


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(L.EXPORTS)


def test_version_and_errors(lib):
    assert b"sm_100a" in lib.euv_version()
    rc = lib.euv_zgemm(4, 4, 4, L.c64(1, 0), None, None, 4, 0, None, 4, 0, L.c64(0, 0), None, 4, 0,
                       L.c64(0, 0), 1, None, 0, None)
    assert rc == L.EUV_ERR_BAD_ARG
    assert b"euv_zgemm" in lib.euv_last_error()


def test_invalid_descriptors_are_rejected(lib):
    d = L.AmpDesc()
    assert lib.euv_amp_workspace_bytes(C.byref(d)) == 0
    assert lib.euv_amp(C.byref(d), None, None, None, 0, None) == L.EUV_ERR_BAD_ARG
    a = L.AbbeDesc()
    assert lib.euv_abbe(C.byref(a), None, None, None) == L.EUV_ERR_BAD_ARG
    m = L.M3dDesc()
    assert lib.euv_m3d_fit(C.byref(m), None, None, None, None, None, None) == L.EUV_ERR_BAD_ARG
    assert lib.euv_lu_factor(-1, None, 1, 0, None, None, 1, None) == L.EUV_ERR_BAD_ARG
    assert lib.euv_matfun_cs(0, None, None, None, None, 1, 4, 0, None, 0, None) == L.EUV_ERR_BAD_ARG
    assert lib.euv_mask_spectrum(None, 1, 8, 8, 8, 8, 1, 1, 0, 0, None, None, 0, None) == L.EUV_ERR_BAD_ARG


def test_struct_sizes_match_c_layout():
    # natural C alignment of the descriptors (x86-64 ABI)
    assert C.sizeof(L.c64) == 16
    assert C.sizeof(L.Stack) == 6 * 16 + 6 * 8 + 8
