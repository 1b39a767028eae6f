"""The index arithmetic of the fused Greenwood row stage (fftcheb.cu,
greenwood_fused_kernel) replayed on the host: the 16 x 16 x 16 plan of the
4096-point transform with its exchange-plane layout, the 4 x 4 16-point DFT
with its output order, and the twiddle powers formed from two table reads,
against the oracle's DCT-III (the RowFFTWorkspace::dct_type3_batch
restatement, rsatb/calc/fft.hpp:125-154, pinned in test_oracle_golden.py).
The CUDA kernel itself is checked against the cuFFT row stage and the oracle
in test_transport_gpu.py."""
from __future__ import annotations

import numpy as np

import oracle

M, N, PLANE = 2048, 4096, 257
C8, S8, R2 = np.cos(np.pi / 8), np.sin(np.pi / 8), np.cos(np.pi / 4)
# v[j0 + 4 c] *= e^{2 pi i j0 c / 16} between the two radix-4 passes
INNER = {5: C8 + 1j * S8, 6: R2 + 1j * R2, 7: S8 + 1j * C8, 9: R2 + 1j * R2, 10: 1j,
         11: -R2 + 1j * R2, 13: S8 + 1j * C8, 14: -R2 + 1j * R2, 15: -C8 - 1j * S8}


def _dft4(a0, a1, a2, a3):
    s02, d02 = a0 + a2, a0 - a2
    s13, d13 = a1 + a3, 1j * (a1 - a3)
    return s02 + s13, d02 + d13, s02 - s13, d02 - d13


def _dft16(v):
    """dft16_inv on columns v[:, 0..15]; output k lands in column 4 (k % 4) + k // 4."""
    v = v.copy()
    for j0 in range(4):
        v[:, j0], v[:, j0 + 4], v[:, j0 + 8], v[:, j0 + 12] = _dft4(
            v[:, j0], v[:, j0 + 4], v[:, j0 + 8], v[:, j0 + 12])
    for i, f in INNER.items():
        v[:, i] *= f
    for c in range(4):
        v[:, 4 * c], v[:, 4 * c + 1], v[:, 4 * c + 2], v[:, 4 * c + 3] = _dft4(
            v[:, 4 * c], v[:, 4 * c + 1], v[:, 4 * c + 2], v[:, 4 * c + 3])
    return v


def _at(k):
    return 4 * (k % 4) + k // 4


QTW = np.exp(2j * np.pi * np.arange(1024) / N)


def _twiddle(n):
    return QTW[n & 1023] * (1j ** ((n >> 10) & 3))


def _pow16(b, b4):
    """w-powers b^k, k = 0..15, as b4^(k // 4) b^(k % 4) (Pow16)."""
    lo = [np.ones_like(b), b, b * b]
    lo.append(lo[2] * b)
    hi = [np.ones_like(b), b4, b4 * b4]
    hi.append(hi[2] * b4)
    return np.stack([hi[k // 4] * lo[k % 4] for k in range(16)], axis=1)


def _fused_plan(x, w):
    """The kernel's transform of one sequence x (length M) with weights w,
    returning the outputs k < M and the exchange slots each pass wrote."""
    t = np.arange(256)
    ph = w * np.exp(1j * np.pi * np.arange(M) / (2 * M))
    v = np.zeros((256, 16), complex)
    for j in range(16):
        n = t + 256 * j
        if j < 8:
            v[:, j] = ph[n] * x[n]
        else:
            m = 2 * M - n
            ok = n != M
            v[ok, j] = np.conj(ph[m[ok]]) * x[m[ok]]
    v = _dft16(v)
    xch = np.full(16 * PLANE, np.nan, complex)
    n0, n1 = t & 15, t >> 4
    tw = _pow16(_twiddle(t), _twiddle(4 * t))
    slots_a = []
    for k0 in range(16):
        idx = n0 * PLANE + k0 * 16 + n1
        xch[idx] = v[:, _at(k0)] * tw[:, k0]
        slots_a.append(idx)
    # pass B: thread (n0, k0)
    n0, k0 = t & 15, t >> 4
    v = np.stack([xch[n0 * PLANE + k0 * 16 + j] for j in range(16)], axis=1)
    v = _dft16(v)
    xch2 = np.full(16 * PLANE, np.nan, complex)
    tw = _pow16(_twiddle(16 * n0), _twiddle(64 * n0))
    slots_b = []
    for k1 in range(16):
        idx = k0 * PLANE + k1 * 16 + n0
        xch2[idx] = v[:, _at(k1)] * tw[:, k1]
        slots_b.append(idx)
    # pass C: thread (k0, k1)
    k0, k1 = t & 15, t >> 4
    v = _dft16(np.stack([xch2[k0 * PLANE + k1 * 16 + j] for j in range(16)], axis=1))
    out = np.zeros(M, complex)
    for k2 in range(8):
        out[k0 + 16 * k1 + 256 * k2] = v[:, _at(k2)]
    return out, np.concatenate(slots_a), np.concatenate(slots_b)


def test_fused_plan_equals_oracle_dct3():
    rng = np.random.default_rng(11)
    for _ in range(2):
        x = rng.standard_normal(M) + 1j * rng.standard_normal(M)
        w = rng.random(M)
        got, slots_a, slots_b = _fused_plan(x, w)
        want = oracle.dct3((w * x)[None, :])[0]
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
        # every exchange slot is written once per pass, inside the 16 planes
        for s in (slots_a, slots_b):
            assert s.size == N and np.unique(s).size == N and s.max() < 16 * PLANE


def test_dft16_output_order():
    rng = np.random.default_rng(3)
    z = rng.standard_normal((4, 16)) + 1j * rng.standard_normal((4, 16))
    d = _dft16(z)
    want = np.fft.ifft(z, axis=1) * 16
    assert np.allclose(np.stack([d[:, _at(k)] for k in range(16)], axis=1), want,
                       rtol=0, atol=1e-13)
