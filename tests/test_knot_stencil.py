"""The split form's derivative near the knots of DD05's piecewise cubics.

The reference's derivative tables hold the seven-point central difference
with step dx = x/1000 (potential_CPU.cpp:159-170).  For a sum of terms
a_i (k_i - x)^3_+ that stencil is exact for every term whose knot lies 3 dx
or more from x; the kernels (sld_pot32.cuh, knot_stencil32 / knot_stencil64)
therefore take the exact derivative and add, for the knot within 3 dx, the
stencil's difference from that term's exact derivative.  Here the same
identity is checked in numpy against the stencil of the whole function, at
distances spread around every knot.
"""
import numpy as np

DENS_A = [0.9332056681088162, -1.162558782567700, -0.3502026949249225,
          0.4287820835430028, 4.907925057809273, -5.307049068415304]
DENS_K = [3.0, 2.8666666666666666, 2.7333333333333333, 2.6, 2.4, 2.3]
PAIR_A = [-0.1960674387419232, 0.3687525935422963, -1.505333614924853,
          4.948907078156191, -4.894613262753399, 3.468897724782442,
          -1.792218099820337, 80.22069592246987]
PAIR_K = [4.1, 3.8, 3.5, 3.2, 2.9, 2.6, 2.4, 2.3]


def cube_pos(x):
    return np.where(x > 0, x ** 3, 0.0)


def fn(a, k, x):
    return sum(ai * cube_pos(ki - x) for ai, ki in zip(a, k))


def stencil(a, k, x):
    dx = x / 1000.0
    return (45 * (fn(a, k, x + dx) - fn(a, k, x - dx)) - 9 * (fn(a, k, x + 2 * dx) - fn(a, k, x - 2 * dx))
            + (fn(a, k, x + 3 * dx) - fn(a, k, x - 3 * dx))) / (60 * dx)


def knot_stencil(u, dx):
    s = (45 * (cube_pos(u - dx) - cube_pos(u + dx)) - 9 * (cube_pos(u - 2 * dx) - cube_pos(u + 2 * dx))
         + (cube_pos(u - 3 * dx) - cube_pos(u + 3 * dx)))
    return s / (60 * dx) + 3 * np.maximum(u, 0.0) ** 2


def corrected(a, k, x):
    d = sum(-3 * ai * np.where(ki - x > 0, (ki - x) ** 2, 0.0) for ai, ki in zip(a, k))
    dx = x / 1000.0
    for ai, ki in zip(a, k):
        u = ki - x
        d = d + np.where(np.abs(u) < 3 * dx, ai * knot_stencil(u, dx), 0.0)
    return d


def test_knot_stencil_reproduces_the_tables_derivative():
    rng = np.random.default_rng(3)
    for a, k in ((DENS_A, DENS_K), (PAIR_A, PAIR_K)):
        x = np.concatenate([ki + rng.uniform(-0.015, 0.015, 4000) for ki in k])
        x = x[(x > 2.05) & (x < 4.1001)]
        ref = stencil(a, k, x)
        exact = sum(-3 * ai * np.where(ki - x > 0, (ki - x) ** 2, 0.0) for ai, ki in zip(a, k))
        got = corrected(a, k, x)
        scale = np.max(np.abs(ref))
        # without the stencil terms the exact derivative misses by ~1e-4
        assert np.max(np.abs(exact - ref)) / scale > 1e-5
        assert np.max(np.abs(got - ref)) / scale < 1e-12


def test_exchange_knot():
    a, k = [0.870 / 3.75 ** 3], [3.75]
    x = np.linspace(3.72, 3.7501, 3001)
    ref = stencil(a, k, x)
    got = corrected(a, k, x)
    assert np.max(np.abs(got - ref)) < 1e-14
