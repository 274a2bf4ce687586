"""The oracle's differentiators against a numpy restatement, on grids where
optimalfilter (src/elastic3d.f90:846-907) picks the 7-point FIR filter of
src/kernel7.inc along x1 (5 <= sx1 <= 14), x2 (5 <= sx2 <= 14) and x3
(5 <= sx3/2 <= 14, where every layer is a boundary layer of the filter and
the finite differences of localstrain_ani apply), and the central
difference elsewhere.

numpy's roll gives the periodic neighbours, so sx2 = 6 also checks the
wrap-around of a 7-tap filter on an axis shorter than 2 x 7 + 1 samples.
FP64 oracle, relative error <= 1e-12.
"""
import numpy as np
import pytest

FIR7 = np.array([8.77856e-01, -2.81913e-01, +6.22696e-02, +2.82441e-02,
                 -5.09029e-02, +4.20471e-02, -1.59409e-02], np.float32).astype(np.float64)

NAMES = ("s11", "s12", "s13", "s22", "s23", "s33")


def d_periodic(a, axis, n, dx):
    """derivative along a periodic axis of n samples (localstrain_ani loops
    over len1 / len2 taps)"""
    if 5 <= n <= 14:
        return sum(FIR7[l - 1] / dx * (np.roll(a, -l, axis) - np.roll(a, l, axis)) for l in range(1, 8))
    return 0.5 / dx * (np.roll(a, -1, axis) - np.roll(a, 1, axis))


def d_depth(a, dx3):
    """axis 0: central differences inside, one-sided at the top and the
    bottom layers (src/elastic3d.f90:977-1002)"""
    d = np.empty_like(a)
    d[1:-1] = (a[2:] - a[:-2]) / (2 * dx3)
    d[0] = (a[1] - a[0]) / dx3
    d[-1] = (a[-1] - a[-2]) / dx3
    return d


def grad(a, dx, sx1, sx2):
    """(d/dx1, d/dx2, d/dx3) of a (sx3h, sx2, sx1) field"""
    return (d_periodic(a, 2, sx1, dx[0]), d_periodic(a, 1, sx2, dx[1]), d_depth(a, dx[2]))


GRIDS = [(32, 8, 8), (32, 6, 6), (48, 12, 12), (16, 9, 9), (32, 4, 6), (32, 16, 16), (16, 14, 5),
         (8, 32, 8), (12, 8, 6), (8, 6, 12), (12, 4, 9)]


@pytest.mark.parametrize("sx1,sx2,sx3h", GRIDS)
def test_stressupdate_matches_numpy(oracle64, sx1, sx2, sx3h):
    o = oracle64
    rng = np.random.default_rng(sx2 * 100 + sx3h)
    dx = (0.5, 0.4, 0.25)
    lam, mu = 1.3, 0.8
    u = np.zeros((3, sx3h, sx2, sx1 + 2))
    u[..., :sx1] = rng.standard_normal((3, sx3h, sx2, sx1))
    sig = np.zeros((sx3h, sx2, sx1), o.tensor)
    o.stressupdate(u, lam, mu, dx, sx1, sx2, sx3h, sig)
    g = [grad(u[k, ..., :sx1], dx, sx1, sx2) for k in range(3)]
    e = {"s11": g[0][0], "s22": g[1][1], "s33": g[2][2],
         "s12": 0.5 * (g[1][0] + g[0][1]), "s13": 0.5 * (g[2][0] + g[0][2]), "s23": 0.5 * (g[2][1] + g[1][2])}
    tr = e["s11"] + e["s22"] + e["s33"]
    for n in NAMES:
        want = 2 * mu * e[n] + (lam * tr if n in ("s11", "s22", "s33") else 0.0)
        err = np.abs(sig[n] - want).max() / np.abs(want).max()
        assert err < 1e-12, (n, err)


@pytest.mark.parametrize("sx1,sx2,sx3h", GRIDS)
def test_bodyforce_matches_numpy(oracle64, sx1, sx2, sx3h):
    o = oracle64
    rng = np.random.default_rng(sx2 * 10 + sx3h)
    dx = (0.5, 0.4, 0.25)
    sig = np.zeros((sx3h, sx2, sx1), o.tensor)
    for n in NAMES:
        sig[n] = rng.standard_normal((sx3h, sx2, sx1))
    c = np.zeros((3, sx3h, sx2, sx1 + 2))
    t = np.zeros((3, sx2, sx1 + 2))
    o.bodyforce(sig, dx, sx1, sx2, sx3h, c, t)
    rows = (("s11", "s12", "s13"), ("s12", "s22", "s23"), ("s13", "s23", "s33"))
    for i, (a, b, d) in enumerate(rows):
        want = -(d_periodic(sig[a], 2, sx1, dx[0]) + d_periodic(sig[b], 1, sx2, dx[1]) + d_depth(sig[d], dx[2]))
        err = np.abs(c[i, ..., :sx1] - want).max() / np.abs(want).max()
        assert err < 1e-12, (i, err)
        assert np.array_equal(t[i, :, :sx1], sig[d][0])


def test_fir7_differentiates_a_band_limited_signal():
    """The filter's purpose: on 12 samples, the derivative of the lowest
    harmonics is closer to the analytic one than the central difference."""
    n, dx = 12, 1.0
    x = np.arange(n) * dx
    for k in (1, 2, 3):
        w = 2 * np.pi * k / (n * dx)
        f = np.sin(w * x)[:, None]
        exact = w * np.cos(w * x)
        fir = d_periodic(f, 0, n, dx)[:, 0]
        cd = 0.5 / dx * (np.roll(f, -1, 0) - np.roll(f, 1, 0))[:, 0]
        assert np.abs(fir - exact).max() < np.abs(cd - exact).max()
