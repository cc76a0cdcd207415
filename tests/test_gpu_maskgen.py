"""Device mask rasteriser (euv_mask_raster through the C ABI): the reference
generator's masks bit for bit, and sidewall slices equal to the host erosion."""
import gzip
import os

import numpy as np
import pytest

from euvlitho_b200 import masks as MK
from oracle import euv_oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_reference_generator_on_the_device(cuda):
    got = MK.vbf_batch(3, 2048, 2048, seed=1, device=cuda).cpu().numpy()
    r = MK.LibcRand(1)
    for k in range(3):
        want = MK.pack(O.vbf_mask(2048, 2048, r).reshape(2048, 2048))
        assert np.array_equal(got[k, 0], want), k
    with gzip.open(os.path.join(GOLDEN, "ref_mask.bin.gz")) as fh:
        assert np.array_equal(got[0, 0], np.frombuffer(fh.read(), np.uint8))


@pytest.mark.parametrize("nx,ny", [(1024, 1024), (1024, 256), (256, 512)])
def test_sidewall_slices_match_the_host_erosion(cuda, nx, ny):
    rng = np.random.default_rng(nx + ny)
    rects = []
    for _ in range(2):
        rs = []
        for _ in range(40):  # overlapping rectangles, some touching the edges
            x0, y0 = int(rng.integers(-20, nx)), int(rng.integers(-20, ny))
            rs.append((x0, x0 + int(rng.integers(1, 90)), y0, y0 + int(rng.integers(1, 90))))
        rs.append((0, 3, 0, ny))   # a column on the wrap-around edge
        rects.append(rs)
    radii = MK.sidewall_erosion(8, 7.5)
    got = MK.rasterize(rects, nx, ny, radii, device=cuda).cpu().numpy()
    for m, rs in enumerate(rects):
        host = MK.sidewall_slices(MK.paint(rs, nx, ny), 8, 7.5)
        for s in range(8):
            assert np.array_equal(got[m, s], MK.pack(host[s])), (m, s, radii[s])


def test_empty_rectangle_list_gives_vacuum(cuda):
    got = MK.rasterize([[], []], 64, 64, (0, 2), device=cuda).cpu().numpy()
    assert (got == 255).all()
