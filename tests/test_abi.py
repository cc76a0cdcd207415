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
    ld = L.LinearDesc()
    assert lib.euv_linear_amp(C.byref(ld), None, None, None, None, None, None) == L.EUV_ERR_BAD_ARG


def test_struct_sizes_match_c_layout():
    # natural C alignment of the descriptors (x86-64 ABI)
    assert C.sizeof(L.c64) == 16
    assert C.sizeof(L.Stack) == 6 * 16 + 6 * 8 + 8


def test_cnn_entry_points_reject_bad_arguments(lib):
    # validated before any launch or allocation: runs without a GPU
    assert lib.euv_cnn_blob_bytes(0, 1901) == 0
    assert lib.euv_cnn_blob_bytes(7, 1901) == 0
    assert lib.euv_cnn_blob_bytes(6, L.EUV_CNN_MAX_OUT + 1) == 0
    assert lib.euv_cnn_workspace_bytes(6, 0, 1901) == 0
    # 6 networks: the fp32 fc1 weights dominate (4096 x 65536 each)
    assert lib.euv_cnn_blob_bytes(6, 1901) > 6 * 4096 * 65536 * 4
    d = L.CnnDesc()
    d.n_models, d.n_masks, d.max_out = 1, 1, 10
    d.n_out[0] = 11  # above max_out
    d.d_factors = 256
    assert lib.euv_cnn_predict(C.byref(d), 1, 1, 1, 1, 1 << 30, None) == L.EUV_ERR_BAD_ARG
    assert b"n_out" in lib.euv_last_error()
    w = (L.CnnModelWeights * 1)()
    assert lib.euv_cnn_pack(1, w, 10, 1e-5, 256, 1 << 40, None) == L.EUV_ERR_BAD_ARG
    assert lib.euv_cnn_downsample(0, None, None, None) == L.EUV_ERR_BAD_ARG


def test_wait_probe_rejects_bad_arguments(lib):
    # validated before any launch, so this runs without a GPU
    assert lib.euv_wait_probe(None, 1000, None, None) == L.EUV_ERR_BAD_ARG
    assert lib.euv_wait_probe(None, -1, None, None) == L.EUV_ERR_BAD_ARG
    assert b"euv_wait_probe" in lib.euv_last_error()


def test_descriptor_layout_matches_the_header(tmp_path):
    """sizeof / offsetof of every descriptor, from the C compiler, against the
    ctypes mirrors."""
    import subprocess
    structs = {"euv_amp_desc": L.AmpDesc, "euv_abbe_desc": L.AbbeDesc, "euv_m3d_desc": L.M3dDesc,
               "euv_stack": L.Stack, "euv_linear_desc": L.LinearDesc, "euv_socs_desc": L.SocsDesc,
               "euv_cnn_desc": L.CnnDesc, "euv_cnn_model_weights": L.CnnModelWeights}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "euvl_b200.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for f, _ in py._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, f, cname, f))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln.strip():
            k1, k2, v = ln.split()
            got[(k1, k2)] = int(v)
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)

