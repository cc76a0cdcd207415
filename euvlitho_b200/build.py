"""Build libeuvl_b200.so (sm_100a) in-tree with nvcc.

Usage: python -m euvlitho_b200.build [--verbose] [--ptxas-info]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libeuvl_b200.so")
SOURCES = ["api.cu", "zgemm.cu", "lu.cu", "rcwa.cu", "abbe.cu", "m3d.cu", "gemm_mixed.cu", "linear.cu", "raster.cu", "jacobi.cu", "socs.cu", "cnn.cu", "plan.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    p = shutil.which("nvcc")
    if p:
        return p
    cand = "/usr/local/cuda/bin/nvcc"
    if os.path.exists(cand):
        return cand
    raise RuntimeError("nvcc not found")


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in sorted(os.listdir(CSRC)) if h.endswith(".cuh")]
    deps.append(os.path.join(ROOT, "include", "euvl_b200.h"))
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps)):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    nvcc = nvcc_path()
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                    "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]
    if ptxas_info:
        flags += ["-Xptxas", "-v"]
    objs = []
    procs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        objs.append(o)
        cmd = [nvcc] + flags + ["-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for s, p in procs:
        out, _ = p.communicate()
        txt = out.decode(errors="replace")
        if p.returncode != 0 or verbose or ptxas_info:
            sys.stdout.write(txt)
        if p.returncode != 0:
            failed = True
            print("nvcc failed on", s, file=sys.stderr)
    if failed:
        raise RuntimeError("CUDA build failed")
    tmp = LIB + ".tmp"
    cmd = [nvcc] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas_info, a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
