"""A step split over GPUs, emulated on one GPU: the partial images of the
ranks' unit ranges (run one after the other) sum to the whole step's image.
The ranks' kernels never wait on one another, so running them in sequence is
the same computation."""
import numpy as np
import pytest

from euvlitho_b200 import masks as MK
from euvlitho_b200.config import preset
from euvlitho_b200.engine import unit_range

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("world", [2, 3])
def test_partial_images_sum_to_the_step(cuda, precision, world):
    import torch
    from euvlitho_b200.engine import Plan
    cfg = preset("small")
    plan = Plan(cfg, device=cuda, pols=("X", "Y"), precision=precision)
    b = plan.intensity_batch(3)
    b.masks.copy_(torch.from_numpy(MK.batch(cfg.ndivx, cfg.ndivy, [4, 5, 6])))
    b.run()
    whole = b.image.clone()
    acc = torch.zeros_like(whole)
    for r in range(world):
        b.run_units(*unit_range(b.U, world, r))
        acc += b.image
    b.check()
    err = float((acc - whole).abs().max() / whole.abs().max())
    assert err < 1e-13, err
