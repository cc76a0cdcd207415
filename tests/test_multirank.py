"""The multi-GPU paths of bench.py, checked with world_size 2 on CPU (gloo):
replicas (each rank images its own clips; the only collectives are a barrier
and the max of the timings) and the unit split (the ranks share the same
clips' units and an all-reduce sums the partial images; the oracle computes
each rank's share here)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    local_ms = 100.0 + 50.0 * rank          # rank 1 is the slowest
    ms = bench.max_over_ranks_on(local_ms, world, torch.device("cpu"))
    dist.barrier()
    out[rank] = (ms, bench.whole_job_rate(4, world, ms), tuple(bench.rank_seeds(rank, 4)))
    dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0][0] == out[1][0] == 150.0                    # max over ranks
    assert out[0][1] == pytest.approx(8 / 0.150)              # all ranks' clips / slowest time
    assert not set(out[0][2]) & set(out[1][2])                 # disjoint clips per rank


def _split_worker(rank, world, port, out):
    """One rank of a step split over GPUs, with the oracle standing in for the
    device: the rank solves and images its range of the (clip, polarisation,
    family) units in the engine's unit order, then the images are summed by
    an all-reduce."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import numpy as np
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    from euvlitho_b200.config import preset
    from euvlitho_b200.engine import unit_range
    from oracle import euv_oracle as O
    from tests.helpers import flat_bits, random_mask, to_oracle
    cfg = preset("small")
    oc = to_oracle(cfg)
    pols = ("X", "Y")
    masks = [flat_bits(random_mask(cfg.ndivx, cfg.ndivy, seed=s)) for s in (71, 72)]
    Lm, Mm = cfg.order_limits()
    li, mi = O.order_set(cfg.order_kind, Lm, Mm)
    nd, fams = O.source(oc)
    fams = [(k, v) for k, v in fams.items() if v]
    lin, mn, _, _ = O.pupil_set(oc)
    sdivsum = sum(len(v) for _, v in fams)
    ntab = len(pols) * len(fams)
    U = len(masks) * ntab
    u0, u1 = unit_range(U, world, rank)
    part = np.zeros((len(masks), len(pols), cfg.xdiv, cfg.ydiv))
    for u in range(u0, u1):
        c, t = divmod(u, ntab)
        p, f = divmod(t, len(fams))
        (nsx, nsy), pts = fams[f]
        sx0 = 2 * O.PI / oc.dx * nsx / nd + oc.kx0
        sy0 = 2 * O.PI / oc.dy * nsy / nd + oc.ky0
        Ax = O.amp_s(pols[p], masks[c], oc, li, mi, Lm, Mm, sx0, sy0, source_orders=pts)
        for F in O.abbe_family_fields(oc, pols[p], Ax, li, mi, nsx, nsy, nd, pts, lin, mn, 0):
            g = np.fft.ifft2(F, axes=(1, 2)) * (cfg.xdiv * cfg.ydiv)
            part[c, p] += np.sum(g.real ** 2 + g.imag ** 2, axis=0) / sdivsum
    img = torch.from_numpy(part)
    dist.all_reduce(img)
    out[rank] = (img.numpy(), (u0, u1))
    dist.destroy_process_group()


def test_two_rank_unit_split_sums_to_the_full_image():
    """bench.py --split-units: the ranks' unit ranges cover every unit once and
    the all-reduced partial images equal the whole image of each clip."""
    import numpy as np
    from euvlitho_b200.config import preset
    from oracle import euv_oracle as O
    from tests.helpers import flat_bits, random_mask, to_oracle
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_split_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    (a, ra), (b, rb) = out[0], out[1]
    assert ra[0] == 0 and ra[1] == rb[0] and rb[1] > rb[0]
    assert np.array_equal(a, b)
    cfg = preset("small")
    for c, seed in enumerate((71, 72)):
        ref = O.intensity(to_oracle(cfg), flat_bits(random_mask(cfg.ndivx, cfg.ndivy, seed=seed)),
                          polars=("X", "Y"))
        for p, pol in enumerate(("X", "Y")):
            assert np.max(np.abs(a[c, p] - ref[pol])) <= 1e-12 * np.max(ref[pol])


def test_unit_ranges_cover_every_unit_once():
    from euvlitho_b200.engine import unit_range
    for U in (1, 5, 24, 97):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                u0, u1 = unit_range(U, world, r)
                seen += list(range(u0, u1))
                assert abs((u1 - u0) - U / world) < 1
            assert seen == list(range(U))
