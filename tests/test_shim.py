"""The C++ binding of the reference drivers (tests/shim): compiled with g++
against include/euvl_b200.h and libeuvl_b200.so, run without Python in the
loop, and checked against the FP64 oracle.

* ``ampS_shim.cpp`` is ampS with the reference's signature (header.h:1208-1213;
  std::vector<std::complex<double>> in place of Eigen::VectorXcd): the body a
  maintainer would put in the reference to call the library;
* ``plan_driver.cpp`` ports intensity.cpp / m3d.cpp main onto the plan API
  (euv_plan_create / _upload / _intensity / _m3d) and calls the ampS shim the
  way intensity.cpp:241-246 does.

The compile runs on the CPU; the runs need a GPU."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from euvlitho_b200 import _lib as L
from euvlitho_b200 import build
from euvlitho_b200.config import SimConfig, preset
from oracle import euv_oracle as O
from tests.helpers import flat_bits, packed, random_mask, rel_err, to_oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "tests", "shim")


def _cuda_home() -> str:
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and os.path.exists(os.path.join(c, "include", "cuda_runtime.h")):
            return c
    pytest.skip("CUDA toolkit headers not found")


def compile_driver(out_dir: str) -> str:
    build.build()
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    cuda = _cuda_home()
    libdir = os.path.join(ROOT, "euvlitho_b200")
    exe = os.path.join(out_dir, "plan_driver")
    cmd = [gxx, "-O2", "-std=c++17", "-Wall", "-Wno-unused-parameter",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"),
           os.path.join(SHIM, "plan_driver.cpp"), os.path.join(SHIM, "ampS_shim.cpp"),
           "-L", libdir, "-leuvl_b200", "-L", os.path.join(cuda, "lib64"), "-lcudart",
           "-Wl,-rpath," + libdir, "-Wl,-rpath," + os.path.join(cuda, "lib64"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def test_shim_and_driver_compile(tmp_path):
    exe = compile_driver(str(tmp_path))
    assert os.access(exe, os.X_OK)


def _run(exe, mode, cfg, pols, masks, tmp_path):
    c = L.config_struct(cfg, pols)
    (tmp_path / "config.bin").write_bytes(bytes(c))
    (tmp_path / "mask.bin").write_bytes(np.concatenate([packed(m) for m in masks]).tobytes())
    r = subprocess.run([exe, mode, str(tmp_path / "config.bin"), str(tmp_path / "mask.bin"),
                        str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_driver_intensity_matches_oracle(cuda, tmp_path):
    from euvlitho_b200 import io
    exe = compile_driver(str(tmp_path))
    cfg = preset("small")
    pols = ("X", "Y")
    masks = [random_mask(cfg.ndivx, cfg.ndivy, seed=s) for s in (61, 62)]
    _run(exe, "intensity", cfg, pols, masks, tmp_path)
    img = np.fromfile(tmp_path / "image.bin", np.float64).reshape(2, 2, cfg.xdiv, cfg.ydiv)
    for c, m in enumerate(masks):
        ref = O.intensity(to_oracle(cfg), flat_bits(m), polars=pols)
        for p, pol in enumerate(pols):
            assert rel_err(img[c, p], ref[pol]) < 1e-8, (c, pol)
    csv = io.read_emint(str(tmp_path / "emint.csv"))
    assert csv.shape == (cfg.xdiv, cfg.ydiv)
    assert np.max(np.abs(csv - img[0, 0])) <= 5e-6 * np.max(img[0, 0])  # 6 significant digits


@pytest.mark.gpu
def test_cpp_driver_m3d_matches_oracle(cuda, tmp_path):
    exe = compile_driver(str(tmp_path))
    cfg = SimConfig(ndivx=512, ndivy=512)  # reference m3d optics on a 512 nm clip
    m = random_mask(512, 512, seed=63)
    _run(exe, "m3d", cfg, ("X",), [m], tmp_path)
    ref = O.m3d(to_oracle(cfg), flat_bits(m))
    out = np.fromfile(tmp_path / "m3d.bin", np.complex128).reshape(3, -1)
    xin = ref["xinput"] == 1
    assert rel_err(out[0], ref["a0"]) < 1e-8
    assert rel_err(out[1][xin], ref["ax"]) < 1e-7
    assert rel_err(out[2][xin], ref["ay"]) < 1e-7
    assert np.all(out[1][~xin] == 0) and np.all(out[2][~xin] == 0)


@pytest.mark.gpu
def test_cpp_ampS_shim_matches_oracle(cuda, tmp_path):
    exe = compile_driver(str(tmp_path))
    cfg = SimConfig(ndivx=256, ndivy=256)  # reference optics and multilayer, 256 nm clip
    m = random_mask(256, 256, seed=64)
    _run(exe, "amps", cfg, ("X",), [m], tmp_path)
    Lm, Mm = cfg.order_limits()
    li, mi = O.order_set(cfg.order_kind, Lm, Mm)
    oc = to_oracle(cfg)
    ref = O.amp_s("X", flat_bits(m), oc, li, mi, Lm, Mm, oc.kx0, oc.ky0)
    from euvlitho_b200 import tables as T
    srcs = T.na_sources(cfg)
    got = np.fromfile(tmp_path / "ax.bin", np.complex128).reshape(len(srcs), len(li))
    for s, key in enumerate(srcs):
        assert rel_err(got[s], ref[key]) < 1e-8, key


def test_integration_doc_shows_the_compiled_shim_verbatim():
    """INTEGRATION.md prints the binding a maintainer adds to the reference;
    the files compiled above must be exactly those listings."""
    import re
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = [b.strip() for b in re.findall(r"```(?:cpp|c\+\+|c)\n(.*?)```", doc, re.S)]
    for name in ("ampS_shim.h", "ampS_shim.cpp"):
        with open(os.path.join(SHIM, name)) as f:
            assert f.read().strip() in blocks, name
