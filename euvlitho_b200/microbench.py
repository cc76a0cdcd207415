"""Kernel microbenchmarks at the shapes of the measured workloads.

  python -m euvlitho_b200.microbench mixed  --n 961 --batch 4
  python -m euvlitho_b200.microbench zgemm  --n 961 --batch 4
  python -m euvlitho_b200.microbench lu     --n 961 --batch 24 --nrhs 96
  python -m euvlitho_b200.microbench step   --precision mixed --clips 4
  python -m euvlitho_b200.microbench linear --preset reference --clips 1
  python -m euvlitho_b200.microbench raster --clips 64 --slices 8
  python -m euvlitho_b200.microbench socs   --preset reference --clips 4
  python -m euvlitho_b200.microbench cnn    --clips 64
  python -m euvlitho_b200.microbench summarize launches.csv

Times each library entry point with CUDA events on the launching stream after
warm-up and prints one JSON line (the commands the ncu summaries in profiles/
are taken from).  `step` runs one pipeline step of a preset's workload (the
batched one by default: 1024 nm clips, N = 961, 3 Bloch families x 2
polarisations = 6 units per clip) untimed, then `--reps` steps between
cudaProfilerStart/Stop, so that `ncu --profile-from-start off` lists exactly
those steps' launches; `--compare` adds the FP64 form's image and the mixed
form's intensity error against it.
`linear` times the linear Abbe model (M3D-parameter amplitudes + two fused
Abbe images per clip) with tables resident, on seeded masks and parameters.
`raster` times the device mask rasteriser on the reference generator's
2048^2 masks (layouts drawn on the host beforehand), with sidewall slices.
`socs` times the STCC-SOCS tables (TCC GEMMs + three Jacobi eigensolves, once
per configuration) and the per-clip SOCS images.
`cnn` times the CNN predict (six networks, random weights) on --clips random
mask rasters, tables resident.
`summarize` folds an ncu `--csv` launch list of gpu__time_duration.sum into
launches, total time and share per kernel.
"""
from __future__ import annotations

import argparse
import collections
import csv
import json
import sys

import torch

from . import _lib as L


def summarize(path: str) -> str:
    hdr, agg = None, collections.defaultdict(lambda: [0, 0.0])
    for r in csv.reader(open(path)):
        if r and r[0] == "ID":
            hdr = r
            continue
        if not hdr or len(r) != len(hdr):
            continue
        d = dict(zip(hdr, r))
        if d.get("Metric Name") != "gpu__time_duration.sum":
            continue
        v = float(d["Metric Value"].replace(",", ""))
        u = d["Metric Unit"]
        v = v / 1e3 if u in ("ns", "nsecond") else (v * 1e3 if u in ("ms", "msecond") else v)
        k = d["Kernel Name"].split("(")[0].replace("euv::", "")
        if k.startswith("void at::"):
            k = "torch " + k[len("void at::"):].split("<")[0]
        agg[k][0] += 1
        agg[k][1] += v
    tot = sum(v[1] for v in agg.values()) or 1.0
    lines = ["| kernel | launches | total us | share |", "|---|---:|---:|---:|"]
    for k, v in sorted(agg.items(), key=lambda x: -x[1][1]):
        lines.append("| %s | %d | %.1f | %.1f%% |" % (k, v[0], v[1], 100 * v[1] / tot))
    lines.append("| total | %d | %.1f | 100%% |" % (sum(v[0] for v in agg.values()), tot))
    return "\n".join(lines)


def _step(a) -> dict:
    from . import masks as MK
    from .config import preset
    from .engine import Plan
    cfg = preset(a.preset)
    plan = Plan(cfg, device=torch.device("cuda"), pols=("X", "Y"), precision=a.precision)
    b = plan.intensity_batch(a.clips)
    b.masks.copy_(torch.from_numpy(MK.batch(cfg.ndivx, cfg.ndivy, range(a.clips))))
    b.run()
    torch.cuda.synchronize()
    n0 = L.lib().euv_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.profiler.start()
    e0.record()
    for _ in range(a.reps):
        b.run()
    e1.record()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    out = {"preset": a.preset, "precision": a.precision, "clips": a.clips, "units": b.U,
           "orders": plan.orders.n, "slices": cfg.nabs,
           "ms_per_step": e0.elapsed_time(e1) / a.reps,
           "launches_per_step": (L.lib().euv_kernel_launches() - n0) // a.reps}
    if a.compare and a.precision != "fp64":
        img = b.image.clone()
        del b
        p64 = Plan(cfg, device=torch.device("cuda"), pols=("X", "Y"), precision="fp64")
        b64 = p64.intensity_batch(a.clips)
        b64.masks.copy_(torch.from_numpy(MK.batch(cfg.ndivx, cfg.ndivy, range(a.clips))))
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        b64.run()
        t1.record()
        torch.cuda.synchronize()
        out["fp64_ms_per_step"] = t0.elapsed_time(t1)
        out["intensity_err_vs_fp64"] = float((img - b64.image).abs().max() / b64.image.abs().max())
    return out


def _linear(a) -> dict:
    import numpy as np
    from . import masks as MK
    from .config import preset
    from .engine import Plan
    cfg = preset(a.preset)
    plan = Plan(cfg, device=torch.device("cuda"))
    tb = plan.linear_tables()
    rng = np.random.default_rng(0)
    par = [torch.from_numpy((rng.standard_normal((a.clips, plan.ncut))
                             + 1j * rng.standard_normal((a.clips, plan.ncut))) * 1e-3).cuda()
           for _ in range(3)]
    bits = torch.from_numpy(MK.batch(cfg.ndivx, cfg.ndivy, range(a.clips))).cuda()
    ms = _time(lambda: plan.linear(bits, *par), a.reps)
    S, ncut, bx = tb["n_src"], plan.ncut, 2 * cfg.lpmaxX + 1
    by = 2 * cfg.lpmaxY + 1
    # Abbe per image: per source, 3 components x (stage y: YDIV x ncut + stage x: XDIV x YDIV x bx)
    flop = 2 * a.clips * S * 3 * 8.0 * (cfg.ydiv * ncut + cfg.xdiv * cfg.ydiv * bx)
    return {"preset": a.preset, "clips": a.clips, "sources": S, "ncut": ncut, "pupil_box": [bx, by],
            "ms_per_call": ms, "clips_per_s": a.clips / (ms / 1e3),
            "abbe_fp64_tflops": flop / (ms / 1e3) / 1e12}


def _raster(a) -> dict:
    from . import masks as MK
    n, nx = a.clips, 2048
    r = MK.LibcRand(1)
    rects = [MK.vbf_rectangles(nx, nx, r) for _ in range(n)]
    radii = MK.sidewall_erosion(a.slices, 60.0 / a.slices)
    out = torch.empty((n, a.slices, nx * nx // 8), dtype=torch.uint8, device="cuda")
    ms = _time(lambda: MK.rasterize(rects, nx, nx, radii, out=out), a.reps)
    steps = max(radii)
    # bytes per mask: fill + paint (~1 B/pixel each), erosion 2 B/pixel per step, pack 1 B/pixel + bits
    moved = n * nx * nx * (2 + 2 * steps + a.slices * (1 + 1.0 / 8))
    return {"masks": n, "slices": a.slices, "erosion_steps": steps, "ms_per_call": ms,
            "masks_per_s": n / (ms / 1e3), "gb_per_s_algorithmic": moved / (ms / 1e3) / 1e9}


def _socs(a) -> dict:
    import time
    import numpy as np
    from . import masks as MK
    from .config import preset
    from .engine import Plan
    cfg = preset(a.preset)
    plan = Plan(cfg, device=torch.device("cuda"))
    plan.uniform_solves()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tb = plan.socs_tables()
    torch.cuda.synchronize()
    t_tab = time.perf_counter() - t0
    rng = np.random.default_rng(0)
    par = [torch.from_numpy((rng.standard_normal((a.clips, plan.ncut))
                             + 1j * rng.standard_normal((a.clips, plan.ncut))) * 1e-3).cuda()
           for _ in range(3)]
    bits = torch.from_numpy(MK.batch(cfg.ndivx, cfg.ndivy, range(a.clips))).cuda()
    ms = _time(lambda: plan.socs(bits, *par), a.reps)
    return {"preset": a.preset, "clips": a.clips, "ncut": plan.ncut, "sources": tb["n_src"],
            "tables_s": t_tab, "ms_per_call": ms, "clips_per_s": a.clips / (ms / 1e3)}


def cnn_random_weights(n_outs, seed: int = 0):
    """Random state_dicts of the CNN predict networks (default-init scales),
    drawn on the device."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    ch = (1, 16, 32, 64, 128, 256)

    def u(shape, fan_in):
        b = 1.0 / fan_in ** 0.5
        return (torch.rand(shape, generator=g, device="cuda") * 2 - 1) * b
    sds = []
    for n in n_outs:
        sd = {}
        for l in range(5):
            sd["conv%d.weight" % (l + 1)] = u((ch[l + 1], ch[l], 3, 3), 9 * ch[l])
            sd["conv%d.bias" % (l + 1)] = u((ch[l + 1],), 9 * ch[l])
            c = ch[l + 1]
            sd["norm%d.weight" % (l + 1)] = 1 + 0.2 * torch.randn(c, generator=g, device="cuda")
            sd["norm%d.bias" % (l + 1)] = 0.2 * torch.randn(c, generator=g, device="cuda")
            sd["norm%d.running_mean" % (l + 1)] = 0.2 * torch.randn(c, generator=g, device="cuda")
            sd["norm%d.running_var" % (l + 1)] = 0.5 + torch.rand(c, generator=g, device="cuda")
        sd["fc1.weight"] = u((4096, 65536), 65536)
        sd["fc1.bias"] = u((4096,), 65536)
        sd["fc2.weight"] = u((n, 4096), 4096)
        sd["fc2.bias"] = u((n,), 4096)
        sds.append(sd)
    return sds


# FP32-equivalent FLOP per mask and network: conv1..conv5 (2 x pixels x cout x
# 9 cin) + fc1 + fc2
def cnn_flop_per_mask(n_out: int) -> float:
    conv = sum(2.0 * (512 >> l) ** 2 * (16 << l) * 9 * (1 if l == 0 else 8 << l) for l in range(5))
    return conv + 2.0 * 65536 * 4096 + 2.0 * 4096 * n_out


def _cnn(a) -> dict:
    from . import cnn
    n_outs = (1901, 1901, 1749, 1749, 1749, 1749)[:a.networks]
    pred = cnn.CnnPredictor(cnn_random_weights(n_outs),
                            [torch.ones(n).numpy() for n in n_outs], torch.device("cuda"))
    torch.cuda.empty_cache()  # the fp32 weights are packed: release them
    g = torch.Generator(device="cuda").manual_seed(1)
    bits = torch.randint(0, 256, (a.clips, cnn.MASK_BYTES), generator=g, device="cuda",
                         dtype=torch.uint8)
    out = torch.empty((len(n_outs), a.clips, pred.max_out), dtype=torch.float64, device="cuda")
    ms = _time(lambda: pred.predict_device(bits, out), a.reps)
    pred.check()
    flop = a.clips * sum(cnn_flop_per_mask(n) for n in n_outs)
    conv1 = a.clips * len(n_outs) * 2.0 * 512 ** 2 * 16 * 9
    return {"masks": a.clips, "networks": len(n_outs), "ms_per_call": ms,
            "masks_per_s": a.clips / (ms / 1e3),
            "fp32_equiv_tflops": flop / (ms / 1e3) / 1e12,
            "tf32_tensor_tflops": 3 * (flop - conv1) / (ms / 1e3) / 1e12,
            "fc1_weight_gb": len(n_outs) * 4096 * 65536 * 4 / 1e9}


def _time(fn, reps: int) -> float:
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.profiler.start()
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    return e0.elapsed_time(e1) / reps


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("kernel", choices=["mixed", "zgemm", "lu", "step", "linear", "raster",
                                       "socs", "cnn", "summarize"])
    ap.add_argument("--slices", type=int, default=8)
    ap.add_argument("csv", nargs="?", help="ncu --csv launch list (summarize)")
    ap.add_argument("--n", type=int, default=961)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--nrhs", type=int, default=96)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--preset", default="batched")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--clips", type=int, default=4)
    ap.add_argument("--networks", type=int, default=6, help="cnn: networks (1..6)")
    ap.add_argument("--compare", action="store_true",
                    help="step: also run the FP64 form and report the intensity error")
    a = ap.parse_args(argv)
    if a.kernel == "summarize":
        print(summarize(a.csv))
        return 0
    if a.kernel == "step":
        print(json.dumps(_step(a)))
        return 0
    if a.kernel == "linear":
        print(json.dumps(_linear(a)))
        return 0
    if a.kernel == "raster":
        print(json.dumps(_raster(a)))
        return 0
    if a.kernel == "socs":
        print(json.dumps(_socs(a)))
        return 0
    if a.kernel == "cnn":
        print(json.dumps(_cnn(a)))
        return 0
    n, b = a.n, a.batch
    s = torch.cuda.current_stream().cuda_stream
    g = torch.Generator(device="cuda").manual_seed(0)
    A = torch.randn(b, n, n, dtype=torch.complex128, device="cuda", generator=g)
    out = {"kernel": a.kernel, "n": n, "batch": b}
    if a.kernel in ("mixed", "zgemm"):
        B = torch.randn(b, n, n, dtype=torch.complex128, device="cuda", generator=g)
        C = torch.empty_like(A)
        if a.kernel == "mixed":
            wb = L.lib().euv_zgemm_mixed_workspace_bytes(n, n, n, b)
            ws = torch.empty(wb, dtype=torch.uint8, device="cuda")

            def fn():
                L.call("euv_zgemm_mixed", n, n, n, L.c64(1, 0), None, A.data_ptr(), n, n * n,
                       B.data_ptr(), n, n * n, L.c64(0, 0), C.data_ptr(), n, n * n, L.c64(0, 0),
                       b, None, 0, ws.data_ptr(), wb, None, s)
        else:
            def fn():
                L.call("euv_zgemm", n, n, n, L.c64(1, 0), None, A.data_ptr(), n, n * n,
                       B.data_ptr(), n, n * n, L.c64(0, 0), C.data_ptr(), n, n * n, L.c64(0, 0),
                       b, None, 0, s)
        ms = _time(fn, a.reps)
        out.update(ms=ms, complex_tflops=8.0 * n ** 3 * b / (ms / 1e3) / 1e12)
    else:
        A += n * torch.eye(n, dtype=torch.complex128, device="cuda")
        W = torch.empty_like(A)
        R = torch.randn(b, a.nrhs, n, dtype=torch.complex128, device="cuda", generator=g)
        X = torch.empty_like(R)
        piv = torch.empty(b * n, dtype=torch.int32, device="cuda")
        info = torch.empty(b, dtype=torch.int32, device="cuda")

        def fn():
            W.copy_(A)
            X.copy_(R)
            L.call("euv_lu_factor", n, W.data_ptr(), n, n * n, piv.data_ptr(), info.data_ptr(), b, s)
            L.call("euv_lu_solve", n, a.nrhs, W.data_ptr(), n, n * n, piv.data_ptr(), X.data_ptr(),
                   n, n * a.nrhs, b, s)
        ms = _time(fn, a.reps)
        out.update(ms=ms, nrhs=a.nrhs)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
