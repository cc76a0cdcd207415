"""Golden images of the reference's linear Abbe model (run once, in a container
that holds the reference checkout; writes tests/golden/ref_linear.npz).

The reference's ``cnn/intensity/linear/linear.py`` computes, from a mask and
its M3D parameters (``inputxx.csv``), the linear-model image ``intlinear`` and
the thin-mask (Kirchhoff) image ``intft``.  This script runs the reference's
own ``int_linear`` (linear.py:45-188, with the NA 0.33 / 2048 nm constants of
its ``elitho/const.py``) on the shipped ``mask.bin`` and ``inputxx.csv``, so
the oracle's restatement and the GPU kernels can be checked against the
reference's code rather than against a re-reading of it.

Two stand-ins, both numerically transparent:
* CuPy is not installed: a module whose ``asarray`` / ``fft.fft2`` / ``.get()``
  are NumPy's takes its place (linear.py uses nothing else of it);
* ``reflect_amplitude`` (the vacuum / absorber specular amplitudes ampvc, ampab
  and phase0 = ampvc/|ampvc|) needs CuPy's eigensolver, so those three numbers
  come from the oracle's narrow solves on the all-vacuum / all-absorber masks
  (the same quantities m3d.cpp:240-258 uses, ``vcxx``/``abxx`` at the centre
  source), and are stored beside the images.

Usage:  python tests/golden/make_linear_golden.py [REFERENCE_ROOT]   (~5 min)
"""
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


class _HostArray(np.ndarray):
    def get(self):
        return np.asarray(self)


def _install_stand_ins() -> None:
    cp = types.ModuleType("cupy")
    cp.asarray = lambda a, *args, **kw: np.asarray(a, *args, **kw)
    cp.fft = types.SimpleNamespace(fft2=lambda a: np.fft.fft2(np.asarray(a)).view(_HostArray))
    sys.modules["cupy"] = cp
    sys.modules["bitarray"] = types.ModuleType("bitarray")  # imported, unused by int_linear


def uniform_amplitudes():
    """ampvc, ampab: specular amplitude of the centre source on the all-vacuum
    and all-absorber masks (oracle narrow solves, reference configuration)."""
    from oracle import euv_oracle as O
    cfg = O.SimConfig()
    ln, mn = O.order_limits(cfg, "ellipse", 1.5)
    li, mi = O.order_set("ellipse", ln, mn)
    LMAX, MMAX = O.order_limits(cfg, cfg.order_kind, cfg.cut)
    n = cfg.ndivx * cfg.ndivy
    pos = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(li, mi))}
    vc = O.amp_s("X", np.ones(n, np.int32), cfg, li, mi, LMAX, MMAX, cfg.kx0, cfg.ky0)
    ab = O.amp_s("X", np.zeros(n, np.int32), cfg, li, mi, LMAX, MMAX, cfg.kx0, cfg.ky0)
    return vc[(0, 0)][pos[(0, 0)]], ab[(0, 0)][pos[(0, 0)]]


def main() -> int:
    from refroot import reference_root
    ref = reference_root()
    lin_dir = os.path.join(ref, "cnn", "intensity", "linear")
    _install_stand_ins()
    sys.path.insert(0, lin_dir)
    import linear as R  # the reference's linear.py
    from oracle import euv_oracle as O
    const = R.const
    p = O.read_inputxx(os.path.join(lin_dir, "inputxx.csv"))
    a0, ax, ay = p["a0"], p["ax"], p["ay"]  # ax, ay: the xinput points only, as in the file
    t0 = time.perf_counter()
    ampvc, ampab = uniform_amplitudes()
    t1 = time.perf_counter()
    mask2d = O.read_mask_bin(os.path.join(lin_dir, "mask.bin"), const.NDIVX, const.NDIVY)
    # linear.py:208-216: pattern on the mask grid, y flipped, transposed to [x][y]
    pattern = np.asarray(mask2d, np.float64) * (ampvc - ampab) + ampab
    pattern = np.flipud(pattern.reshape(const.NDIVY, const.NDIVX)).T.astype(np.complex128)
    phase0 = ampvc / abs(ampvc)
    intlinear, intft = R.int_linear(0, pattern.copy(), a0, ax, ay, phase0)
    t2 = time.perf_counter()
    out = os.path.join(HERE, "ref_linear.npz")
    np.savez_compressed(out, intlinear=np.asarray(intlinear, np.float32),
                        intft=np.asarray(intft, np.float32),
                        ampvc=np.complex128(ampvc), ampab=np.complex128(ampab),
                        max_intlinear=np.float64(np.max(intlinear)),
                        max_intft=np.float64(np.max(intft)))
    print("ampvc", ampvc, "ampab", ampab, "(%.0f s)" % (t1 - t0))
    print("int_linear %.0f s; max intlinear %.6g intft %.6g -> %s"
          % (t2 - t1, np.max(intlinear), np.max(intft), out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
