"""The oracle's stencil sums are the reference's term by term (src/evolution.jl:192-219):
`axis_stencil` writes w[1] u[-r] + w[2] u[-r+1] + ... + w[n] u[r] as a left fold from the lowest
offset to the highest, and `mixed_stencil` folds the first-derivative rows of the second axis
(inner) and then the rows along the first axis (outer) the same way. Julia contracts none of
these products and sums (no `muladd`), so every product and every sum is rounded on its own:
Python floats do exactly that. The device's second differences are pinned to the oracle's at a
spacing where any other order shows (test_gpu_parity.py), so this closes the chain to the
reference."""
import numpy as np
import pytest


def _left_fold(w, u, base, stride):
    r = (len(w) - 1) // 2
    s = float(w[0]) * float(u[base - r * stride])
    for k in range(1, len(w)):
        s = s + float(w[k]) * float(u[base + (k - r) * stride])
    return s


def _mixed_fold(w, u, base, s1, s2):
    r = (len(w) - 1) // 2
    outer = None
    for a in range(len(w)):
        inner = float(w[0]) * float(u[base + (a - r) * s1 - r * s2])
        for e in range(1, len(w)):
            inner = inner + float(w[e]) * float(u[base + (a - r) * s1 + (e - r) * s2])
        outer = float(w[0]) * inner if a == 0 else outer + float(w[a]) * inner
    return outer


def _data(seed, n=24):
    rng = np.random.default_rng(seed)
    # values of order one with small variations, where the summation order shows in the last bits
    return np.ascontiguousarray(1.0 + 1e-3 * rng.standard_normal(n * n * n))


@pytest.mark.parametrize("q", [2, 4, 6, 8])
def test_axis_stencils_are_the_references_left_folds(oracle, q):
    n = 24
    u = _data(q)
    tables = {1: oracle.weights_double(q, 1), 2: oracle.weights_double(q, 2), 0: oracle.weights_double(q // 2 + 1, 0)}
    base = 12 + n * (12 + n * 12)
    paired_differs = False
    for which, w in tables.items():
        for stride in (1, n, n * n):
            for shift in range(8):
                b = base + shift * (1 + n)
                got = oracle.axis_stencil(q, which, u, b, stride)
                assert got == _left_fold(w, u, b, stride), (q, which, stride, shift)
                if which == 2:
                    # the control: taps paired at +-k, summed from the centre out, is another rounding
                    r = (len(w) - 1) // 2
                    p = float(w[r]) * float(u[b])
                    for k in range(1, r + 1):
                        p = p + float(w[r + k]) * (float(u[b + k * stride]) + float(u[b - k * stride]))
                    paired_differs |= p != got
    assert paired_differs


@pytest.mark.parametrize("q", [2, 4, 6, 8])
def test_mixed_stencils_are_the_references_folds(oracle, q):
    n = 24
    u = _data(100 + q)
    w = oracle.weights_double(q, 1)
    base = 12 + n * (12 + n * 12)
    for s1, s2 in ((1, n), (1, n * n), (n, n * n)):
        for shift in range(8):
            b = base + shift * (1 + n + n * n)
            assert oracle.mixed_stencil(q, u, b, s1, s2) == _mixed_fold(w, u, b, s1, s2), (q, s1, s2, shift)
