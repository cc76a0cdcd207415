"""The cluster LU panel's bookkeeping (csrc/lu.cu, lu_panel_cluster_kernel),
restated in NumPy and checked on CPU against an unblocked LU with whole-row
swaps (LAPACK getf2 order).

The kernel keeps a block of LC_BLK columns at fixed register indices and
stores a block's columns when the block ends; the row swap at column c
exchanges only the columns from c on, and the laswp launch after the panel
(sub = 1) then gives every panel column c the swaps of the pivots c+1.. that it
missed.  The pivot is the first maximum of |re| + |im| (izamax)."""
import numpy as np
import pytest


def _getf2(A):
    A = A.copy()
    n, nb = A.shape
    piv = []
    for c in range(nb):
        col = np.abs(A[c:, c].real) + np.abs(A[c:, c].imag)
        p = c + int(np.argmax(col))
        piv.append(p)
        A[[c, p], :] = A[[p, c], :]
        if A[c, c] != 0:
            A[c + 1:, c] /= A[c, c]
            A[c + 1:, c + 1:] -= np.outer(A[c + 1:, c], A[c, c + 1:])
    return A, piv


def _cluster_panel(A, blk):
    n, nb = A.shape
    reg = A.copy()           # the rows as the threads hold them
    out = np.zeros_like(A)   # the panel as stored to global memory
    piv = []
    for c0 in range(0, nb, blk):
        for c in range(c0, min(c0 + blk, nb)):
            col = np.abs(reg[c:, c].real) + np.abs(reg[c:, c].imag)
            p = c + int(np.argmax(col))
            piv.append(p)
            reg[[c, p], c:] = reg[[p, c], c:]        # columns from c on only
            if reg[c, c] != 0:
                reg[c + 1:, c] /= reg[c, c]
                reg[c + 1:, c + 1:] -= np.outer(reg[c + 1:, c], reg[c, c + 1:])
        out[:, c0:c0 + blk] = reg[:, c0:c0 + blk]   # the block leaves the registers
    for c in range(nb):                              # laswp, sub = 1
        for jj in range(c + 1, nb):
            p = piv[jj]
            if p != jj:
                out[[jj, p], c] = out[[p, jj], c]
    return out, piv


@pytest.mark.parametrize("n,nb,blk", [(40, 32, 4), (100, 32, 4), (33, 1, 4), (70, 13, 4), (64, 32, 8)])
def test_cluster_panel_matches_getf2(n, nb, blk):
    rng = np.random.default_rng(n * 100 + nb)
    A = rng.standard_normal((n, nb)) + 1j * rng.standard_normal((n, nb))
    ref, pref = _getf2(A)
    got, pgot = _cluster_panel(A, blk)
    assert pgot == pref
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12)
