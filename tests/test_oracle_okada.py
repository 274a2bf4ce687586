"""The half-space dislocation of Okada (1992) that RELAX adds for small
coseismic sources (okada, src/okada/green_space.f90:29-105): the oracle's
restatement is pinned by the properties that determine the solution
uniquely -- equilibrium away from the fault, a traction-free surface, a
displacement jump across the fault equal to the dislocation, decay far
away -- and the library's host evaluation (relax_okada_point, the same
code the GPU runs) agrees with it.  CPU only."""
import ctypes as C
import math

import numpy as np
import pytest

from relax_b200 import _lib
from relax_b200.config import relax_source

LAM, MU = 1.0, 1.0


def _oracle(oracle64, src, p):
    d = (C.c_double * 3)()
    oracle64.lib.orc_okada(LAM, MU, src["slip"], src["opening"], src["x"], src["y"], src["z"], src["width"],
                           src["length"], src["strike"], src["dip"], src["rake"], p[0], p[1], p[2], d)
    return np.array(d[:])


def _lib_point(src, p):
    lib = _lib.load()
    s = relax_source(**src)
    d = (C.c_double * 3)()
    _lib.check(lib.relax_okada_point(C.byref(s), LAM, MU, p[0], p[1], p[2], d))
    return np.array(d[:])


def _source(kind, dip, strike=30.0):
    src = dict(slip=0.0, opening=0.0, x=1.0, y=-2.0, z=3.0, width=4.0, length=6.0, strike=strike, dip=dip,
               rake=0.0, period=0.0, phase=0.0, beta=0.0)
    if kind == "strike":
        src.update(slip=1.0, rake=0.0)
    elif kind == "dip":
        src.update(slip=1.0, rake=90.0)
    else:
        src.update(opening=1.0)
    return src


def _frame(src):
    """Strike, down-dip and normal unit vectors in RELAX's (north, east, down) frame."""
    st, dp = math.radians(src["strike"]), math.radians(src["dip"])
    s = np.array([math.cos(st), math.sin(st), 0.0])
    d = np.array([-math.sin(st) * math.cos(dp), math.cos(st) * math.cos(dp), math.sin(dp)])
    return s, d, np.cross(s, d)


def _stress(f, p, h):
    g = np.zeros((3, 3))
    for j in range(3):
        e = np.zeros(3)
        e[j] = h
        g[:, j] = (f(p + e) - f(p - e)) / (2 * h)
    eps = 0.5 * (g + g.T)
    return LAM * np.trace(eps) * np.eye(3) + 2 * MU * eps


KINDS = ["strike", "dip", "tensile"]
DIPS = [90.0, 60.0, 25.0]


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("dip", DIPS)
def test_displacement_jump_equals_the_dislocation(oracle64, kind, dip):
    src = _source(kind, dip)
    s, d, n = _frame(src)
    top = np.array([src["x"], src["y"], src["z"]])
    f = lambda p: _oracle(oracle64, src, p)
    for a, b in [(0.5, 0.5), (0.2, 0.7), (0.8, 0.3)]:
        p = top + a * src["length"] * s + b * src["width"] * d
        jump = f(p + 1e-4 * n) - f(p - 1e-4 * n)
        want = {"strike": s, "dip": -d, "tensile": n}[kind]
        # the jump is the unit dislocation along strike, up dip or along the normal
        assert abs(abs(np.dot(jump, want)) - 1.0) < 1e-3, (jump, want)
        assert np.linalg.norm(jump - np.dot(jump, want) * want) < 1e-3


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("dip", DIPS)
def test_traction_free_surface_and_equilibrium(oracle64, kind, dip):
    src = _source(kind, dip)
    f = lambda p: _oracle(oracle64, src, p)
    rng = np.random.default_rng(7)
    for _ in range(6):
        # sigma_i3 vanishes at x3 = 0: one-sided points converge linearly in depth
        p0 = np.array([rng.uniform(-12, 12), rng.uniform(-12, 12), 0.0])
        scale = np.abs(_stress(f, p0 + [0, 0, 0.5], 1e-3)).max()
        t1 = np.abs(_stress(f, p0 + [0, 0, 1e-3], 5e-5)[:, 2]).max()
        t2 = np.abs(_stress(f, p0 + [0, 0, 1e-4], 5e-6)[:, 2]).max()
        assert t1 < 1e-2 * scale + 1e-9 and t2 < 0.2 * t1 + 1e-9
        # div sigma = 0 inside the medium, away from the fault
        p = np.array([rng.uniform(-12, 12), rng.uniform(-12, 12), rng.uniform(0.5, 12)])
        if np.linalg.norm(p - np.array([src["x"], src["y"], src["z"]])) < 9.0:
            p[0] += 12.0
        h = 1e-3
        terms = np.zeros((3, 3))
        for j in range(3):
            e = np.zeros(3)
            e[j] = h
            terms[:, j] = (_stress(f, p + e, h)[:, j] - _stress(f, p - e, h)[:, j]) / (2 * h)
        # the terms d_j sigma_ij cancel to finite-difference accuracy
        assert np.abs(terms.sum(axis=1)).max() < 1e-4 * np.abs(terms).sum(axis=1).max()


def test_decay_and_the_library_agrees(oracle64):
    rng = np.random.default_rng(3)
    for kind in KINDS:
        for dip in (90.0, 45.0, 10.0):
            src = _source(kind, dip, strike=rng.uniform(0, 360))
            far = [np.linalg.norm(_oracle(oracle64, src, [r, 0.3 * r, 0.0])) for r in (100.0, 200.0)]
            assert 3.5 < far[0] / far[1] < 8.5          # 1/r^2, or 1/r^3 near a nodal direction
            for _ in range(20):
                p = np.array([rng.uniform(-15, 15), rng.uniform(-15, 15), rng.uniform(0, 10)])
                a, b = _oracle(oracle64, src, p), _lib_point(src, p)
                np.testing.assert_allclose(b, a, rtol=1e-11, atol=1e-13)
    # on a fault edge both return zero
    src = _source("strike", 90.0, strike=0.0)
    edge = [src["x"] + 2.0, src["y"], src["z"]]
    assert not _oracle(oracle64, src, edge).any() and not _lib_point(src, edge).any()


def _dc3d(oracle64, src, p):
    d = (C.c_double * 3)()
    oracle64.lib.orc_okada_dc3d(LAM, MU, src["slip"], src["opening"], src["x"], src["y"], src["z"], src["width"],
                                src["length"], src["strike"], src["dip"], src["rake"], p[0], p[1], p[2], d)
    return np.array(d[:])


@pytest.mark.parametrize("kind", ["strike", "dip", "tensile"])
@pytest.mark.parametrize("dip", [90.0, 60.0, 25.0, 10.0])
def test_okada_matches_the_references_dc3d(oracle64, kind, dip):
    """Against a restatement of the reference's own routine: DC3D
    (src/okada/dc3d.f, displacement rows of UA, UB, UC over the four
    corners of the real source and its image) behind green_space.f90's
    okada, with its REAL*4 arguments.  Receivers on a grid around the
    source, at the surface and at depth; the FP32 arguments bound the
    agreement at 2e-5 of the displacement scale (points within 0.05 of a
    fault edge excluded)."""
    src = _source(kind, dip)
    rng = np.random.default_rng(int(dip) + len(kind))
    pts = [np.array([rng.uniform(-12, 14), rng.uniform(-14, 10), z]) for z in (0.0, 0.0, 1.5, 4.0, 7.5)
           for _ in range(40)]
    ref = np.array([_dc3d(oracle64, src, p) for p in pts])
    scale = np.abs(ref).max()
    assert scale > 1e-3
    for p, r in zip(pts, ref):
        ours = _oracle(oracle64, src, p)
        lib = _lib_point(src, p)
        assert np.abs(ours - r).max() <= 2e-5 * scale, (p, ours, r)
        assert np.abs(lib - r).max() <= 2e-5 * scale, (p, lib, r)
