"""The space-domain solution for small coseismic sources on the GPU
(dislocations_disp, src/relax.f90:1298-1349; grnfct_okada,
src/okada/green_space.f90:114-144): the relax_op_okada kernel against the
oracle's Okada (1992) restatement point by point, and the coseismic solve of
an event with sources below the Nyquist length against the oracle run, with
the origin shifted and the grid rotated (the sources go back to the
input-file convention for this term).

Tolerance: FP64 arithmetic rounded to FP32 per source, so 1e-6 of the
field's maximum point by point; the coseismic fields to relative L2 1e-5."""
import ctypes as C

import numpy as np
import pytest

from relax_b200 import _lib
from relax_b200.api import Relax
from relax_b200.config import Event, Fault, Tensile, relax_source

from cases import linear_small, rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _src(**kw):
    base = dict(slip=0.0, opening=0.0, x=0.0, y=0.0, z=0.0, width=1.0, length=1.0, strike=0.0, dip=90.0, rake=0.0,
                period=0.0, phase=0.0, beta=0.0)
    base.update(kw)
    return relax_source(**base)


def test_okada_op_matches_oracle(oracle64):
    lib = _lib.load()
    sx1, sx2, sx3h = 64, 48, 16
    dx = (0.7, 0.5, 0.6)
    srcs = (relax_source * 3)(_src(slip=1.3, x=-2.0, y=1.5, z=0.0, width=1.0, length=1.2, strike=25.0, dip=70.0,
                                   rake=30.0),
                              _src(opening=0.8, x=3.0, y=-4.0, z=2.0, width=0.9, length=0.8, strike=100.0, dip=40.0),
                              _src(slip=-0.5, x=5.0, y=6.0, z=1.0, width=0.6, length=0.9, strike=300.0, dip=90.0,
                                   rake=-90.0))
    u = [torch.zeros((sx3h, sx2, sx1 + 2), dtype=torch.float32, device="cuda") for _ in range(3)]
    _lib.check(lib.relax_op_okada(C.cast(srcs, C.c_void_p), 3, 1.0, 1.0, sx1, sx2, sx3h, *dx,
                                  *[C.c_void_p(t.data_ptr()) for t in u], None))
    torch.cuda.synchronize()
    got = np.stack([t.cpu().numpy()[..., :sx1] for t in u])
    rng = np.random.default_rng(0)
    scale = np.abs(got).max()
    assert scale > 1e-3
    d = (C.c_double * 3)()
    for _ in range(1500):
        i1, i2, i3 = int(rng.integers(sx1)), int(rng.integers(sx2)), int(rng.integers(sx3h))
        x1 = (i1 if i1 < sx1 // 2 else i1 - sx1) * dx[0]
        x2 = (i2 if i2 < sx2 // 2 else i2 - sx2) * dx[1]
        want = np.zeros(3, np.float32)
        for s in srcs:
            oracle64.lib.orc_okada(1.0, 1.0, s.slip, s.opening, s.x, s.y, s.z, s.width, s.length, s.strike, s.dip,
                                   s.rake, x1, x2, i3 * dx[2], d)
            want += np.array(d[:], np.float32)
        np.testing.assert_allclose(got[:, i3, i2, i1], want, rtol=0, atol=1e-6 * scale)


def _small_sources(rotated):
    sim = linear_small(sx=64, sz=32, steps=2)
    sim.events = [Event(0.0, [Fault(1.0, -10.0, 0.0, 0.0, 20.0, 6.0, 0.0, 90.0, 0.0),
                              Fault(2.0, 4.0, 6.0, 1.0, 1.5, 1.2, 40.0, 60.0, 120.0)],
                        tensile=[Tensile(0.7, -6.0, -8.0, 2.0, 1.0, 3.0, 10.0, 80.0)])]
    if rotated:
        sim.x0, sim.y0, sim.rot = 1.5, -2.0, 20.0
    return sim


@pytest.mark.parametrize("rotated", [False, True])
def test_coseismic_with_small_sources_matches_oracle(oracle32, rotated):
    sim = _small_sources(rotated)
    with Relax(sim) as r:
        r.coseismic()
        u = r.field("u")
        for _ in range(2):
            r.step()
        u2 = r.field("u")
    _, rf0 = oracle32.run(sim, 0)
    assert rel_l2(u[..., :sim.sx1], rf0["u"][..., :sim.sx1]) < 1e-5
    logs, rf = oracle32.run(sim, 2)
    assert rel_l2(u2[..., :sim.sx1], rf["u"][..., :sim.sx1]) < 1e-4
    # the small sources contribute: without them the fields differ
    big = _small_sources(rotated)
    big.events[0].faults = big.events[0].faults[:1]
    big.events[0].tensile = []
    with Relax(big) as r:
        r.coseismic()
        ub = r.field("u")
    assert rel_l2(u[..., :sim.sx1], ub[..., :sim.sx1]) > 1e-3
