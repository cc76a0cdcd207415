"""The autotuner on the device: its picks change launch shapes only, never the
results, and a second use reads them from the cache."""
import numpy as np
import pytest

from euvlitho_b200 import _lib as L
from euvlitho_b200 import autotune as A
from euvlitho_b200 import masks as MK
from euvlitho_b200.config import preset

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_tuned_picks_keep_the_results(cuda, tmp_path, precision):
    import torch
    from euvlitho_b200.engine import Plan
    L.lib().euv_tune_clear()
    cfg = preset("small")
    plan = Plan(cfg, device=cuda, pols=("X", "Y"), precision=precision)
    b = plan.intensity_batch(3)
    b.masks.copy_(torch.from_numpy(MK.batch(cfg.ndivx, cfg.ndivy, [1, 2, 3])))
    b.run()
    ref = b.image.clone()
    path = str(tmp_path / "tuning.json")
    res = A.ensure(b, path=path, reps=1)
    assert res["tuned"] and res["tuned_ms"] <= res["base_ms"]
    for (name, k0, k1), v in res["picks"].items():
        assert L.lib().euv_tune_get(A.KNOBS[name], k0, k1) == v
    # every candidate of every knob ran the whole step; results do not move
    for name in A.shapes(b):
        for k0, k1 in A.shapes(b)[name]:
            for v in A.CANDIDATES[name]:
                L.lib().euv_tune_set(A.KNOBS[name], k0, k1, v)
                b.run()
                b.check()
                err = float((b.image - ref).abs().max() / ref.abs().max())
                assert err < 1e-12, (name, v, err)
            L.lib().euv_tune_set(A.KNOBS[name], k0, k1, res["picks"][(name, k0, k1)])
    L.lib().euv_tune_clear()
    again = A.ensure(b, path=path, reps=1)
    assert again["tuned"] is False and again["picks"] == res["picks"]
    L.lib().euv_tune_clear()
