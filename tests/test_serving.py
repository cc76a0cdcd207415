"""Serving: continuous batching returns, for every request, the image the same
clip gets when it is computed alone (CPU checks of the workload generator, GPU
check of the results)."""
import numpy as np
import pytest

from euvlitho_b200 import serving as S


def test_workload_is_poisson_and_propagating():
    reqs = S.workload(400, rate=50.0, seed=3)
    t = np.array([r.arrival for r in reqs])
    gaps = np.diff(np.r_[0.0, t])
    assert abs(gaps.mean() - 1 / 50.0) < 0.2 / 50.0          # mean rate
    assert all(S.propagating(r.key.period, r.key.box) for r in reqs)
    assert {r.key.period for r in reqs} == set(S.PERIODS)
    assert {r.key.n_src for r in reqs} <= set(S.SOURCE_COUNTS)


def test_config_for_gives_the_requested_source_count():
    from euvlitho_b200 import tables as T
    for key in (S.ClipKey(256, 5, 50), S.ClipKey(1024, 15, 200), S.ClipKey(512, 10, 100)):
        cfg = S.config_for(key)
        n = sum(len(f.pts) for f in T.sources(cfg)[1])
        assert n == key.n_src
        assert (cfg.ndivx, cfg.lbox) == (key.period, key.box)


@pytest.mark.gpu
def test_each_result_same_alone_and_in_the_mix(cuda):
    """Requests of two periods and two source counts with the same order box
    share launches (one ampS of all their units, each with its own period);
    every request's image equals the image the server returns for that clip
    served alone (1e-13: the launch's other clips do not reach a clip's
    result), and the engine's own single-configuration image to 1e-5 (the
    group fixes the Euler factor count of the mixed form, which the engine
    derives per configuration: the two differ by the product's truncation,
    below 1e-7 of G^-1)."""
    import torch
    # arrivals within a fraction of a millisecond: the requests queue up while
    # the first launches run, so later launches mix periods and source counts
    reqs = S.workload(24, rate=1e5, seed=5, periods=(256, 512), boxes=(5,),
                      source_counts=(50, 100))
    assert len({r.key for r in reqs}) > 1
    keys = sorted({r.key for r in reqs}, key=lambda k: (k.period, k.box, k.n_src))
    srv = S.Server(device=cuda, precision="mixed", max_batch=8, n_streams=3)
    srv.warm(keys)
    stats = srv.serve(reqs)
    assert stats["requests"] == len(reqs) and stats["failed"] == 0
    assert stats["mean_batch"] > 1.5
    assert any(len({r.key for r in gl}) > 1 for gl in srv.launched_groups)
    alone_srv = S.Server(device=cuda, precision="mixed", max_batch=1, n_streams=1)
    alone_srv.warm(keys)
    for r in reqs:
        one = S.Request(r.rid, r.key, r.mask, 0.0)
        alone_srv.serve([one])
        err = np.max(np.abs(r.image - one.image)) / np.max(np.abs(one.image))
        assert err < 1e-13, (r.rid, err)
        plan = srv.plan(r.key)
        eng = plan.intensity(torch.from_numpy(r.mask[None])).cpu().numpy()[0]
        err = np.max(np.abs(r.image - eng)) / np.max(np.abs(eng))
        assert err < 1e-5, (r.rid, err)
