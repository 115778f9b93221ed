"""CPU restatement of the covariance-form grid (csrc/grid_cov.cu), checked
against the FP64 oracle: the Gram of the 16 x int4 components in the kernel's
component order, E from the Gram by the partner rule, V = [Re w ; -Im w] in
the same order, and I_b = v_b^T E v_b equal to the window sum of
|sum_a w_a x_a|^2 (the reference's float order, src/cpu_beamformer.cpp:56-78,
computed here exactly)."""
from __future__ import annotations

import numpy as np

from conftest import grid_weights, random_voltage

F, A = 336, 64


def _components(v: np.ndarray) -> np.ndarray:
    """[T][F][A] packed bytes -> [T][F][128] int64 components in the kernel's
    order: component m = 16c + 4h + k is antenna 8c + 4(h >> 1) + k, the real
    part for even h; each is 16 x the signed nibble, as the unpack stores it."""
    lo = (v & 0x0F).astype(np.int64)
    hi = (v >> 4).astype(np.int64)
    re = np.where(lo >= 8, lo - 16, lo) * 16
    im = np.where(hi >= 8, hi - 16, hi) * 16
    m = np.arange(128)
    ant = 8 * (m >> 4) + 4 * (((m >> 2) & 3) >> 1) + (m & 3)
    part = (m >> 2) & 1
    return np.where(part[None, None, :] == 0, re[:, :, ant], im[:, :, ant])


def _e_from_gram(G: np.ndarray) -> np.ndarray:
    """E_mn = (G_mn +- G_{m^4, n^4}) / 256, + when m and n are the same part."""
    m = np.arange(128)
    part = (m >> 2) & 1
    sign = np.where(part[:, None] == part[None, :], 1, -1)
    partner = G[..., m ^ 4, :][..., :, m ^ 4]
    E2 = G + sign * partner
    assert np.all(E2 % 256 == 0)
    return E2 // 256


def _v(w: np.ndarray) -> np.ndarray:
    """canonical [B][F][A][2] weights -> V [F][128][B] in the component order."""
    m = np.arange(128)
    ant = 8 * (m >> 4) + 4 * (((m >> 2) & 3) >> 1) + (m & 3)
    part = (m >> 2) & 1
    wr, wi = w[..., 0].astype(np.float64), w[..., 1].astype(np.float64)  # [B][F][A]
    v = np.where(part[None, None, :] == 0, wr[:, :, ant], -wi[:, :, ant])  # [B][F][128]
    return np.transpose(v, (1, 2, 0))


def test_covariance_form_equals_window_power(orc):
    T, B, S = 192, 5, 64
    v = random_voltage(T, F, A, seed=3)
    w = grid_weights(A, F, B, seed=4)
    y = _components(v)                                   # [T][F][128]
    V = _v(w)                                            # [F][128][B]
    out = np.zeros((T // S, F, B))
    for win in range(T // S):
        ys = y[win * S:(win + 1) * S]                    # [S][F][128]
        G = np.einsum("tfm,tfn->fmn", ys, ys)            # exact int64
        E = _e_from_gram(G).astype(np.float64)           # [F][128][128]
        Y = np.einsum("fmn,fnb->fmb", E, V)
        out[win] = np.einsum("fmb,fmb->fb", V, Y)
    ref = orc.beamform_integrated(v, w, T, F, A, B, S, f64=True)
    assert np.allclose(out, ref, rtol=1e-9, atol=1e-6), float(np.max(np.abs(out - ref)))


def test_e_is_the_real_form_of_the_hermitian_covariance():
    """E = [[Rr, -Ri], [Ri, Rr]] of R = sum_t x x^H, arranged in the
    component order (checked entry by entry on one channel)."""
    T = 40
    v = random_voltage(T, 1, A, seed=9)
    y = _components(v)[:, 0, :]
    E = _e_from_gram(np.einsum("tm,tn->mn", y, y))
    lo = (v[:, 0, :] & 0x0F).astype(np.int64)
    hi = (v[:, 0, :] >> 4).astype(np.int64)
    x = np.where(lo >= 8, lo - 16, lo) + 1j * np.where(hi >= 8, hi - 16, hi)
    R = np.einsum("ta,tb->ab", x, np.conj(x))
    m = np.arange(128)
    ant = 8 * (m >> 4) + 4 * (((m >> 2) & 3) >> 1) + (m & 3)
    part = (m >> 2) & 1
    for i in range(128):
        for j in range(128):
            a, b = ant[i], ant[j]
            if part[i] == part[j]:
                want = R[a, b].real
            elif part[i] == 0:
                want = -R[a, b].imag
            else:
                want = R[a, b].imag
            assert E[i, j] == want, (i, j)
