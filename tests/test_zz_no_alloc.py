"""euv_matfun_cs_noalloc: the entry point for callers that cannot allocate
device memory (plug-ins whose host owns all device memory, hosts with a fixed
device-memory budget, latency-critical loops that must avoid the device-wide
synchronisation of cudaMalloc/cudaFree).  It uses a fixed 16 MiB
scratch array inside the library instead of a caller workspace.

Checked through the C ABI against the workspace entry point euv_matfun_cs on
two calls in a row (the shared array keeps the previous call's contents).
Named so that pytest collects it after every other test file."""
import numpy as np
import pytest

from euvlitho_b200 import _lib as L

pytestmark = pytest.mark.gpu

TOL = 1e-13  # same kernels and arithmetic as euv_matfun_cs: equal to rounding


def _slice_matrix(n, seed):
    rng = np.random.default_rng(seed)
    k = 2 * np.pi / 13.5
    D = np.diag(k * k * (0.93 + 0.05j) - rng.uniform(0, 0.01, n)) + \
        0.004 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    return np.ascontiguousarray(D.T)  # column-major


def _reference(cuda, Dcm, thick, n, batch):
    import torch
    dD = torch.from_numpy(Dcm).to(cuda)
    th = torch.from_numpy(thick).to(cuda)
    c, s = torch.empty_like(dD), torch.empty_like(dD)
    wb = L.lib().euv_matfun_workspace_bytes(n, batch)
    ws = torch.empty(wb, dtype=torch.uint8, device=cuda)
    L.call("euv_matfun_cs", n, dD.data_ptr(), th.data_ptr(), c.data_ptr(), s.data_ptr(), batch, 12,
           L.EUV_PREC_FP64, ws.data_ptr(), wb, torch.cuda.current_stream().cuda_stream)
    return c, s


@pytest.mark.parametrize("n,batch", [(121, 3), (200, 2)])
def test_noalloc_matches_workspace_entry_on_two_calls(cuda, n, batch):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    for call, seed in enumerate((n, n + 1)):  # two calls in a row, different inputs
        D = np.stack([_slice_matrix(n, seed * 10 + b) for b in range(batch)])
        thick = np.array([60.0, 7.5, 30.0][:batch] if batch <= 3 else [60.0] * batch)
        c_ref, s_ref = _reference(cuda, D, thick, n, batch)
        dD = torch.from_numpy(D).to(cuda)
        th = torch.from_numpy(thick).to(cuda)
        c = torch.full_like(dD, float("nan"))
        s = torch.full_like(dD, float("nan"))
        L.call("euv_matfun_cs_noalloc", n, dD.data_ptr(), th.data_ptr(), c.data_ptr(),
               s.data_ptr(), batch, 12, stream)
        torch.cuda.synchronize()
        for got, ref in ((c, c_ref), (s, s_ref)):
            g, r = got.cpu().numpy(), ref.cpu().numpy()
            assert np.all(np.isfinite(g)), "call %d" % call
            assert np.max(np.abs(g - r)) / np.max(np.abs(r)) < TOL, "call %d" % call


def test_noalloc_rejects_requests_above_the_fixed_scratch(cuda):
    n = 1024  # 5 * n^2 * 16 bytes = 80 MiB > 16 MiB
    rc = L.lib().euv_matfun_cs_noalloc(n, 16, 16, 16, 16, 1, 8, None)
    assert rc == L.EUV_ERR_BAD_ARG
    assert b"scratch" in L.lib().euv_last_error()
