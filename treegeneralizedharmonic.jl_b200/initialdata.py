"""Seeded synthetic initial data: the analytic background plus Fourier modes.

The perturbation of every one of the 20 evolved components is a sum of 8 modes
A sin(pi (k . x) + phi) with integer wavenumbers k in {1..4}^3 (periodic on a box of side 2)
and uniform phases. The generator is xoshiro256** seeded through SplitMix64; per component,
per mode it draws k_x, k_y, k_z (the top two bits of one draw each, plus one) and the phase
(the top 53 bits of one draw, times 2 pi / 2^53), in that order.
"""
import math

import numpy as np

_M64 = (1 << 64) - 1


def _rotl(x, k):
    return ((x << k) | (x >> (64 - k))) & _M64


class Xoshiro256ss:
    def __init__(self, seed):
        x = seed & _M64
        s = []
        for _ in range(4):
            x = (x + 0x9E3779B97F4A7C15) & _M64
            z = x
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
            s.append(z ^ (z >> 31))
        self.s = s

    def next(self):
        s = self.s
        r = (_rotl((s[1] * 5) & _M64, 7) * 9) & _M64
        t = (s[1] << 17) & _M64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = _rotl(s[3], 45)
        return r


def fourier_modes(seed=20261203, nvars=20, nmodes=8, kmax=4):
    """[nvars, nmodes] wavenumbers (int, 3) and phases."""
    assert kmax == 4
    g = Xoshiro256ss(seed)
    ks = np.zeros((nvars, nmodes, 3), dtype=np.int64)
    ph = np.zeros((nvars, nmodes))
    for v in range(nvars):
        for m in range(nmodes):
            for d in range(3):
                ks[v, m, d] = 1 + (g.next() >> 62)
            ph[v, m] = (g.next() >> 11) * (2.0 * math.pi / 2.0 ** 53)
    return ks, ph


def perturbation(forest, amplitude=1e-4, seed=20261203, scale=None):
    """The perturbation at every owned point, in state layout (float64 numpy, flat).
    `scale[v, m]` optionally multiplies mode m of component v."""
    ks, ph = fourier_modes(seed)
    N1 = forest.N + 1
    out = np.zeros((forest.nblocks, 20, N1, N1, N1))
    for b in range(forest.nblocks):
        x, y, z = forest.block_positions(b)
        for v in range(20):
            acc = np.zeros_like(x)
            for m in range(ks.shape[1]):
                a = amplitude if scale is None else amplitude * scale[v, m]
                acc += a * np.sin(math.pi * (ks[v, m, 0] * x + ks[v, m, 1] * y + ks[v, m, 2] * z) + ph[v, m])
            out[b, v] = acc
    return out.reshape(-1)
