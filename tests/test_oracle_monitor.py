"""The oracle's observation-plane sampler (monitorstressfield / monitorfield,
src/elastic3d.f90:3404-3762): grid size, node values on grid-aligned planes,
a constant field kept by the normalised sinc window, zero outside the box,
and the plane's points on the rotated plane."""
import math

import numpy as np
import pytest

from relax_b200.config import relax_obsplane

from cases import oracle_monitor_plane

SX, DX = (32, 32, 16), (1.0, 1.0, 1.0)


def _field(nc, seed=0):
    rng = np.random.default_rng(seed)
    shape = (SX[2], SX[1], SX[0]) if nc == 1 else (nc, SX[2], SX[1], SX[0])
    return rng.normal(0, 1, shape).astype(np.float32)


def _fix(x):
    f, c = math.floor(x), math.ceil(x)
    return c if x - f > 0.5 else f


@pytest.mark.parametrize("nc", [1, 6])
def test_grid_aligned_plane_reads_nodes(oracle32, nc):
    f = _field(nc)
    # internal strike 0, dip 0: the plane x1 = 3, along x2 and down x3
    op = relax_obsplane(x=3.0, y=-2.0, z=6.0, length=8.0, width=6.0, strike=0.0, dip=0.0)
    out = oracle_monitor_plane(oracle32.lib, f, SX, DX, op)
    assert out.shape[:2] == (_fix(6.0) + 1, _fix(8.0) + 1)
    for j3 in range(out.shape[0]):
        for j2 in range(out.shape[1]):
            x1, x2, x3 = out[j3, j2, :3]
            assert x1 == 3.0 and x2 == -2.0 + (j2 - 4) and x3 == 6.0 + (j3 - 3)
            i1, i2, i3 = int(x1) % SX[0], int(x2) % SX[1], int(x3)
            want = f[i3, i2, i1] if nc == 1 else f[:, i3, i2, i1]
            np.testing.assert_array_equal(out[j3, j2, 5:], np.atleast_1d(want).astype(np.float64))


@pytest.mark.parametrize("nc", [1, 6])
def test_constant_field_is_kept(oracle32, nc):
    f = np.full((SX[2], SX[1], SX[0]) if nc == 1 else (nc, SX[2], SX[1], SX[0]), 2.5, np.float32)
    op = relax_obsplane(x=0.3, y=1.7, z=5.2, length=7.3, width=4.1, strike=0.4, dip=0.7)
    out = oracle_monitor_plane(oracle32.lib, f, SX, DX, op)
    inside = (out[..., 2] >= 0) & (out[..., 2] <= SX[2] - 1)
    assert inside.any()
    np.testing.assert_allclose(out[inside][:, 5:], 2.5, rtol=2e-6)


def test_points_lie_on_the_plane_and_outside_reads_zero(oracle32):
    f = _field(6, seed=2)
    op = relax_obsplane(x=2.0, y=-3.0, z=2.0, length=10.0, width=16.0, strike=0.6, dip=0.9)
    out = oracle_monitor_plane(oracle32.lib, f, SX, DX, op)
    cs, ss, cd, sd = math.cos(op.strike), math.sin(op.strike), math.cos(op.dip), math.sin(op.dip)
    xr = cd * (cs * op.x - ss * op.y) - sd * op.z
    for p in out.reshape(-1, 11):
        # the local x coordinate (out of plane) of every sample is the centre's
        x = cd * (cs * p[0] - ss * p[1]) - sd * p[2]
        assert abs(x - xr) < 1e-5
    below = out[..., 2] < 0
    assert below.any()
    assert (out[below][:, 5:] == 0).all()


def test_sizes_follow_the_taper(oracle32):
    f = _field(1)
    op = relax_obsplane(x=0.0, y=0.0, z=4.0, length=5.0, width=3.0, strike=0.0, dip=0.0)
    out = oracle_monitor_plane(oracle32.lib, f, SX, DX, op, beta=0.25)
    assert out.shape[:2] == (_fix(3.0 * 1.5) + 1, _fix(5.0 * 1.5) + 1)
