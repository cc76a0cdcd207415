"""Failure detection on the GPU without a fault: a bounded device wait that
runs out comes back as a status bit with the context still usable, the
pipeline's status word stays clear on healthy runs, and a solver-failure flag
(set from the host, standing in for the device) surfaces as an error of the
batch and of the served requests."""
import numpy as np
import pytest

from euvlitho_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


def test_expired_wait_sets_the_timeout_bit_and_the_context_survives(cuda):
    import torch
    flag = torch.zeros(1, dtype=torch.int32, device=cuda)      # nothing ever sets it
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    L.call("euv_wait_probe", flag.data_ptr(), 2_000_000, status.data_ptr(), _stream())  # 2 ms
    torch.cuda.synchronize()
    assert status.item() == L.EUV_STATUS_TIMEOUT
    status.zero_()
    flag.fill_(1)
    L.call("euv_wait_probe", flag.data_ptr(), 2_000_000, status.data_ptr(), _stream())
    torch.cuda.synchronize()
    assert status.item() == 0
    # the context still computes
    a = torch.randn(64, 64, dtype=torch.complex128, device=cuda)
    c = torch.empty_like(a)
    L.call("euv_zgemm", 64, 64, 64, L.c64.of(1), None, a.data_ptr(), 64, 0, a.data_ptr(), 64, 0,
           L.c64.of(0), c.data_ptr(), 64, 0, L.c64.of(0), 1, None, 0, _stream())
    torch.cuda.synchronize()
    ref = (a.T @ a.T).T  # column-major product
    assert torch.allclose(c, ref, rtol=1e-12, atol=1e-10)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_healthy_batch_leaves_the_status_clear(cuda, precision):
    import torch
    from euvlitho_b200 import masks as MK
    from euvlitho_b200.config import preset
    from euvlitho_b200.engine import Plan
    cfg = preset("small")
    plan = Plan(cfg, device=cuda, pols=("X", "Y"), precision=precision)
    b = plan.intensity_batch(2)
    b.masks.copy_(torch.from_numpy(MK.batch(cfg.ndivx, cfg.ndivy, [1, 2])))
    b.run()
    b.check()
    assert b.status.item() == 0


def test_solver_failure_flag_fails_the_batch(cuda):
    import torch
    from euvlitho_b200 import masks as MK
    from euvlitho_b200.config import preset
    from euvlitho_b200.engine import Plan
    cfg = preset("small")
    plan = Plan(cfg, device=cuda, pols=("X",))
    b = plan.intensity_batch(1)
    b.masks.copy_(torch.from_numpy(MK.batch(cfg.ndivx, cfg.ndivy, [3])))
    b.status.fill_(L.EUV_STATUS_SINGULAR)   # stands in for a zero pivot found on the device
    b.run()
    with pytest.raises(L.EuvError) as e:
        b.check()
    assert e.value.code == L.EUV_ERR_SINGULAR
    b.check()  # the word was cleared by the failed check


def test_served_requests_carry_the_failure_instead_of_an_image(cuda):
    from euvlitho_b200 import serving as S
    reqs = S.workload(6, rate=1000.0, seed=11, periods=(256,), boxes=(5,), source_counts=(50,))
    srv = S.Server(device=cuda, precision="mixed", max_batch=1, n_streams=1)
    key = reqs[0].key
    srv.warm([key])
    srv.slots[0].status.fill_(L.EUV_STATUS_TIMEOUT)  # the next launch of this slot fails
    stats = srv.serve(reqs)
    assert stats["failed"] == 1
    bad = [r for r in reqs if r.error is not None]
    assert len(bad) == 1 and bad[0].image is None and "gave up" in bad[0].error
    assert all(r.image is not None and np.isfinite(r.image).all() for r in reqs if r.error is None)


def test_bad_mask_size_is_rejected_on_the_host(cuda):
    import torch
    from euvlitho_b200.config import preset
    from euvlitho_b200.engine import Plan
    plan = Plan(preset("small"), device=cuda)
    with pytest.raises(ValueError):
        plan.intensity(torch.zeros(1, 17, dtype=torch.uint8))
