"""The four-way split sums of the Abbe kernel's DFT stages (csrc/abbe.cu, R4
path), restated in NumPy and checked against the direct sums on CPU.

x stage: f(x) = sum_lx G(lx) e^(2 pi i (lx - lpx) x / X).  With t = lx - lpx
and the sum started at lx0 = (lpx mod 4) - 4 over zero pad rows, the four
partial sums P_s(g) over t = s (mod 4) give f(g + q X/4) = sum_s i^(q s) P_s(g)
(radix-4 butterfly).  y stage: for the rows y0 + q Y/4 of one CTA, every pupil
point's product u = E e^(2 pi i m y0 / Y) adds i^(m q) u to row q."""
import numpy as np
import pytest


def _direct_x(G, lpx, X):
    lx = np.arange(G.shape[0])
    x = np.arange(X)
    W = np.exp(2j * np.pi * np.outer(x, lx - lpx) / X)
    return np.tensordot(W, G, axes=(1, 0))


def _split_x(G, lpx, X):
    bx = G.shape[0]
    pad = 4
    Gp = np.concatenate([np.zeros((pad,) + G.shape[1:], complex), G,
                         np.zeros((pad,) + G.shape[1:], complex)])
    lx0 = (lpx & 3) - 4
    nj = (bx - lx0 + 3) // 4
    out = np.zeros((X,) + G.shape[1:], complex)
    for g in range(X // 4):
        P = np.zeros((4,) + G.shape[1:], complex)
        w = np.exp(2j * np.pi * ((lx0 - lpx) * g % X) / X)
        r = np.exp(2j * np.pi * g / X)
        for j in range(nj):
            for k in range(4):
                P[k] += Gp[pad + lx0 + 4 * j + k] * w
                w *= r
        A, B = P[0] + P[2], P[0] - P[2]
        S, D = P[1] + P[3], P[1] - P[3]
        for q, f in enumerate((A + S, B + 1j * D, A - S, B - 1j * D)):
            out[g + q * X // 4] = f
    return out


@pytest.mark.parametrize("lpx,X", [(5, 64), (6, 76), (7, 88), (8, 100), (20, 256)])
def test_x_stage_split_sums(lpx, X):
    rng = np.random.default_rng(lpx * 1000 + X)
    G = rng.standard_normal((2 * lpx + 1, 4, 3)) + 1j * rng.standard_normal((2 * lpx + 1, 4, 3))
    np.testing.assert_allclose(_split_x(G, lpx, X), _direct_x(G, lpx, X), rtol=0, atol=1e-10)


@pytest.mark.parametrize("lpy,Y", [(2, 32), (3, 40), (4, 52), (5, 64), (10, 256)])
def test_y_stage_rows_a_quarter_apart(lpy, Y):
    rng = np.random.default_rng(lpy * 1000 + Y)
    m = np.arange(-lpy, lpy + 1)
    E = rng.standard_normal(m.size) + 1j * rng.standard_normal(m.size)
    for y0 in range(Y // 4):
        direct = [np.sum(E * np.exp(2j * np.pi * m * (y0 + q * Y // 4) / Y)) for q in range(4)]
        g = np.zeros(4, complex)
        for mm, e in zip(m, E):
            u = e * np.exp(2j * np.pi * mm * y0 / Y)
            k = mm % 4
            for q in range(4):
                g[q] += (1j ** ((k * q) % 4)) * u
        np.testing.assert_allclose(g, direct, rtol=0, atol=1e-10)
