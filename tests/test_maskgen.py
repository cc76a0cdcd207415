"""The reference's mask generator (cnn/intensity/mask/mask.cpp, mVBF.h), CPU
side: the oracle's restatement and the host layout against the shipped mask
(which is that program's first draw) and against the program itself when it
has been built under oracle/_ref (make -C oracle ref)."""
import gzip
import os
import subprocess

import numpy as np
import pytest

from euvlitho_b200 import masks as MK
from oracle import euv_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
REF_BIN = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "maskgen")


def _golden_bits():
    with gzip.open(os.path.join(GOLDEN, "ref_mask.bin.gz")) as fh:
        return np.frombuffer(fh.read(), np.uint8)


def test_oracle_generator_reproduces_the_shipped_mask():
    m = O.vbf_mask(2048, 2048, MK.LibcRand(1))
    assert np.array_equal(MK.pack(m.reshape(2048, 2048)), _golden_bits())


@pytest.mark.parametrize("nx,ny,seed", [(2048, 2048, 1), (1024, 1024, 7), (1024, 256, 3), (512, 2048, 11)])
def test_layout_rectangles_match_the_oracle_over_consecutive_masks(nx, ny, seed):
    # one libc generator per process: seed it again before the second sequence
    r = MK.LibcRand(seed)
    rects = [MK.vbf_rectangles(nx, ny, r) for _ in range(3)]
    r = MK.LibcRand(seed)
    want = [O.vbf_mask(nx, ny, r) for _ in range(3)]
    for rs, w in zip(rects, want):
        assert np.array_equal(MK.paint(rs, nx, ny).reshape(-1), w)


def test_shipped_mask_is_the_reference_programs_first_draw(tmp_path):
    if not os.path.exists(REF_BIN):
        pytest.skip("reference generator not built (make -C oracle ref)")
    subprocess.run([REF_BIN], cwd=tmp_path, check=True)
    got = np.fromfile(tmp_path / "mask.bin", np.uint8)
    assert np.array_equal(got, _golden_bits())


def test_sidewall_radii_follow_the_slice_rule():
    assert MK.sidewall_erosion(8, 7.5) == [int(round((7 - n) * 7.5 * np.tan(np.deg2rad(6.0))))
                                           for n in range(8)]
    assert MK.sidewall_erosion(1, 60.0) == [0]
