"""Golden image of the reference's STCC-SOCS model (run once, in a container
that holds the reference checkout; writes tests/golden/ref_socs.npz).

The reference's ``cnn/intensity/stccsocs`` computes the three transmission
cross-coefficient matrices of the source and pupil (eigenfunction.py:5-163),
their eigenpairs sorted by |alpha|, and the SOCS image of a mask from its M3D
parameters (socs.py:12-151).  This script runs the reference's own
``eigenfunction`` and ``intsocs`` (NA 0.33 / 2048 nm constants of its
``elitho/const.py``) on the shipped ``mask.bin`` and ``inputxx.csv``.

Stand-ins, numerically transparent: CuPy is not installed, so a module whose
``asarray``, ``matmul``, ``fft.fft2``, ``linalg.eigh`` and ``.get()`` are
NumPy's takes its place (the scripts use nothing else of it); the vacuum /
absorber specular amplitudes of ``reflect_amplitude`` (CuPy eigensolver) come
from the oracle's narrow solves, as in make_linear_golden.py.  Stored: the
image (float32) and the leading eigenvalues of the three TCCs (float64).

Usage:  python tests/golden/make_socs_golden.py [REFERENCE_ROOT]   (~3 min)
"""
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)


class _HostArray(np.ndarray):
    def get(self):
        return np.asarray(self)


def _h(a):
    return np.asarray(a).view(_HostArray)


def _install_stand_ins() -> None:
    cp = types.ModuleType("cupy")
    cp.asarray = lambda a, *args, **kw: _h(np.asarray(a, *args, **kw))
    cp.matmul = lambda a, b: _h(np.matmul(np.asarray(a), np.asarray(b)))
    cp.fft = types.SimpleNamespace(fft2=lambda a: _h(np.fft.fft2(np.asarray(a))))

    def eigh(a):
        w, v = np.linalg.eigh(np.asarray(a))
        return _h(w), _h(v)
    cp.linalg = types.SimpleNamespace(eigh=eigh)
    sys.modules["cupy"] = cp
    sys.modules["bitarray"] = types.ModuleType("bitarray")  # imported, unused here


def main() -> int:
    from make_linear_golden import uniform_amplitudes
    from refroot import reference_root
    ref = reference_root()
    d = os.path.join(ref, "cnn", "intensity", "stccsocs")
    _install_stand_ins()
    sys.path.insert(0, d)
    import eigenfunction as E  # the reference's eigenfunction.py
    import socs as R           # the reference's socs.py
    from oracle import euv_oracle as O
    const = R.const
    p = O.read_inputxx(os.path.join(d, "inputxx.csv"))
    t0 = time.perf_counter()
    ampvc, ampab = uniform_amplitudes()
    t1 = time.perf_counter()
    eig = E.eigenfunction(0)
    t2 = time.perf_counter()
    mask2d = O.read_mask_bin(os.path.join(d, "mask.bin"), const.NDIVX, const.NDIVY)
    pattern = np.asarray(mask2d, np.float64) * (ampvc - ampab) + ampab  # socs.py:197-206
    pattern = np.flipud(pattern.reshape(const.NDIVY, const.NDIVX)).T.astype(np.complex128)
    img = R.intsocs(_h(pattern.copy()), p["a0"], p["ax"], p["ay"], ampvc / abs(ampvc), *eig)
    t3 = time.perf_counter()
    out = os.path.join(HERE, "ref_socs.npz")
    np.savez_compressed(out, intsocs=np.asarray(np.real(img), np.float32),
                        alpha_s0=np.asarray(eig[0][:128]), alpha_sx=np.asarray(eig[2][:32]),
                        alpha_sy=np.asarray(eig[4][:32]),
                        ampvc=np.complex128(ampvc), ampab=np.complex128(ampab))
    print("eigenfunction %.0f s, intsocs %.0f s (amplitudes %.0f s); max %.6g -> %s"
          % (t2 - t1, t3 - t2, t1 - t0, np.max(np.real(img)), out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
