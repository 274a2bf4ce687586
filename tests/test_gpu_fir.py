"""Time steps on narrow and shallow boxes, where optimalfilter
(src/elastic3d.f90:846-907) picks the 7-point FIR differentiator of
src/kernel7.inc along x1 (5 <= sx1 <= 14) or x2 (5 <= sx2 <= 14) and the
finite differences of localstrain_ani through the whole depth
(5 <= sx3/2 <= 14), against both oracle builds with the GPU's Dt sequence
replayed.

On these grids the stress kernel reads the x1 and x2 derivatives from
k_fir_xy and the x-forward pass of the Green's function takes the generic
kernel with the filters in its divergence.  Tolerances as in test_gpu_step: relative L2
<= 1e-4 of every field after the run, the logs to 1e-3.
"""
import dataclasses

import pytest

from cases import linear_small, powerlaw_small
from test_gpu_step import check_logs, compare, gpu_run

pytestmark = pytest.mark.gpu


def _narrow(builder, sx2, **kw):
    sim = builder(**kw)
    sim.sx2 = sx2
    sim.name += f"-sx2-{sx2}"
    return sim


def _narrow_x1(builder, sx1, sx2=None, **kw):
    """a box of sx1 samples along x1 (the fault shortened to fit it)"""
    sim = builder(**kw)
    sim.sx1 = sx1
    if sx2:
        sim.sx2 = sx2
    f = sim.events[0].faults[0]
    half = 0.25 * sx1 * sim.dx1
    sim.events[0].faults[0] = dataclasses.replace(f, x=-half, length=2.0 * half)
    sim.name += f"-sx1-{sx1}"
    return sim


CASES = {
    "linear sx2=8 sx3/2=8": (lambda: _narrow(linear_small, 8, sx=32, sz=16), 4),
    "linear sx2=6 sx3/2=9": (lambda: _narrow(linear_small, 6, sx=32, sz=18), 4),
    "power-law sx2=12 sx3/2=12": (lambda: _narrow(powerlaw_small, 12, sx=32, sz=24), 3),
    "power-law sx2=9 sx3/2=16": (lambda: _narrow(powerlaw_small, 9, sx=48, sz=32), 3),
    "linear sx1=8": (lambda: _narrow_x1(linear_small, 8, sx=32, sz=16), 4),
    "linear sx1=12 sx2=8": (lambda: _narrow_x1(linear_small, 12, sx2=8, sx=32, sz=16), 4),
    "power-law sx1=12": (lambda: _narrow_x1(powerlaw_small, 12, sx=32, sz=24, afterslip=False), 3),
}


@pytest.mark.parametrize("name", list(CASES))
def test_fir_grids_match_oracles(oracle32, oracle64, name):
    builder, nsteps = CASES[name]
    sim = builder()
    glogs, gf, _ = gpu_run(sim, nsteps)
    assert len(glogs) == nsteps + 1
    dts = [lg[1] for lg in glogs[1:]]
    rlogs, rf = oracle32.run(sim, nsteps, dt_schedule=dts)
    check_logs(glogs, rlogs, 1e-3)
    compare(gf, rf, 1e-4)
    _, df = oracle64.run(sim, nsteps, dt_schedule=dts)
    compare(gf, df, 1e-4)

