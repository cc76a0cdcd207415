"""STCC-SOCS on the GPU: the Jacobi eigensolver (euv_heev) against LAPACK, the
SOCS image (euv_socs_image) against the oracle, and at the reference
configuration against the reference's own intsocs."""
import gzip
import os

import numpy as np
import pytest

from euvlitho_b200 import _lib as L
from euvlitho_b200 import io
from euvlitho_b200.config import SimConfig
from oracle import euv_oracle as O
from tests.helpers import packed, random_mask, to_oracle

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


@pytest.mark.parametrize("n,kind", [(1, "rand"), (2, "rand"), (5, "rand"), (64, "rand"),
                                    (129, "rand"), (96, "repeated"), (200, "psd")])
def test_jacobi_matches_lapack(cuda, n, kind):
    import torch
    rng = np.random.default_rng(n)
    X = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    if kind == "rand":
        H = (X + X.conj().T) / 2
    elif kind == "psd":
        H = X @ X.conj().T / n
    else:  # eigenvalues with multiplicity
        Q, _ = np.linalg.qr(X)
        lam = np.repeat(rng.standard_normal(n // 4), 4)
        H = (Q * lam) @ Q.conj().T
        H = (H + H.conj().T) / 2
    a = torch.from_numpy(np.ascontiguousarray(H.T)).to(cuda)  # column-major
    w = torch.empty(n, dtype=torch.float64, device=cuda)
    v = torch.empty((n, n), dtype=torch.complex128, device=cuda)
    st = torch.zeros(1, dtype=torch.int32, device=cuda)
    wb = L.lib().euv_heev_workspace_bytes(n)
    ws = torch.empty(wb, dtype=torch.uint8, device=cuda)
    L.call("euv_heev", n, a.data_ptr(), n, w.data_ptr(), v.data_ptr(), n, 30, 1e-14, ws.data_ptr(),
           wb, st.data_ptr(), _stream())
    torch.cuda.synchronize()
    assert st.item() == 0
    wh, V = w.cpu().numpy(), v.cpu().numpy().T   # V[:, j] = eigenvector j
    scale = np.max(np.abs(np.linalg.eigvalsh(H)))
    assert np.max(np.abs(np.sort(wh) - np.linalg.eigvalsh(H))) < 1e-12 * scale
    assert np.max(np.abs(V.conj().T @ V - np.eye(n))) < 1e-12
    assert np.max(np.abs(H @ V - V * wh)) < 1e-11 * scale


def _socs_oracle(cfg, masks, par, tb, plan):
    oc = to_oracle(cfg)
    e = (tb["alpha_s0"].cpu().numpy(), tb["phi_s0"].cpu().numpy(), tb["alpha_sx"].cpu().numpy(),
         tb["phi_sx"].cpu().numpy(), tb["alpha_sy"].cpu().numpy(), tb["phi_sy"].cpu().numpy())
    return [O.socs_image(oc, masks[c].reshape(-1), par[0][c], par[1][c], par[2][c], tb["amp_vc"],
                         tb["amp_ab"], e, tb["nsocs"], tb["nsocsxy"], tb["nout"]) for c in range(len(masks))]


def test_socs_image_matches_the_oracle(cuda):
    """Same kernels (the device eigenpairs) in both: checks the SOCS sum, the
    64-point DFTs and the Fourier interpolation; the eigenvalues themselves are
    checked against LAPACK on the oracle's TCC."""
    import torch
    from euvlitho_b200.engine import Plan
    cfg = SimConfig(ndivx=512, ndivy=512)
    plan = Plan(cfg, device=cuda)
    tb = plan.socs_tables(nsocs=60, nsocsxy=12)
    oc = to_oracle(cfg)
    tcc = O.socs_tcc(oc, 0.0)
    z, copies = O.socs_padding(oc)
    assert (z, copies) == plan.socs_padding()
    for t, name in zip(tcc, ("s0", "sx", "sy")):
        # TCC_sx / TCC_sy have +-lambda pairs (the source grid is symmetric):
        # their order within |alpha| ties is set by rounding, so compare spectra
        lam = np.sort(O.socs_eigen(t, z, copies)[0])
        got = np.sort(tb["eig_" + name])
        assert np.max(np.abs(got - lam)) < 1e-12 * np.max(np.abs(lam)), name
    rng = np.random.default_rng(3)
    masks = [random_mask(512, 512, s) for s in (4, 5)]
    par = [(rng.standard_normal((2, plan.ncut)) + 1j * rng.standard_normal((2, plan.ncut))) * 1e-3
           for _ in range(3)]
    par[1][:, plan.xinput == 0] = 0
    par[2][:, plan.xinput == 0] = 0
    img = plan.socs(torch.from_numpy(np.stack([packed(m) for m in masks])), *par,
                    nsocs=60, nsocsxy=12).cpu().numpy()
    want = _socs_oracle(cfg, masks, par, tb, plan)
    for c in range(2):
        err = np.max(np.abs(img[c] - want[c])) / np.max(np.abs(want[c]))
        assert err < 1e-10, (c, err)


@pytest.mark.slow
def test_reference_config_matches_the_reference_socs(cuda):
    import torch
    from euvlitho_b200.engine import Plan
    p = os.path.join(GOLDEN, "ref_socs.npz")
    if not os.path.exists(p):
        pytest.skip("ref_socs.npz not generated")
    g = np.load(p)
    plan = Plan(SimConfig(), device=cuda)
    tb = plan.socs_tables()
    for name in ("s0", "sx", "sy"):
        ref = np.abs(g["alpha_" + name])    # |alpha|: the sign order of +- ties is rounding
        got = np.abs(tb["eig_" + name][:len(ref)])
        assert np.max(np.abs(got - ref)) < 1e-12 * np.max(ref), name
    with gzip.open(os.path.join(GOLDEN, "ref_mask.bin.gz")) as fh:
        bits = np.frombuffer(fh.read(), np.uint8).copy()
    with gzip.open(os.path.join(GOLDEN, "ref_inputxx.csv.gz"), "rt") as fh:
        xx = io.read_inputxx(fh)
    img = plan.socs(torch.from_numpy(bits)[None], xx["a0"][None],
                    io.expand_xinput(xx["ax"], plan.xinput)[None],
                    io.expand_xinput(xx["ay"], plan.xinput)[None])[0].cpu().numpy()
    ref = g["intsocs"].astype(np.float64)
    assert np.max(np.abs(img - ref)) / np.max(ref) < 2e-7
