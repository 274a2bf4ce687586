"""Surface loads (traction, src/elastic3d.f90:2517-2590) on the GPU against
the oracle.

A step load enters the coseismic solve of event 0; a periodic load enters
every step as a traction rate -- the predictor's with Dt/2e8 as the
reference passes it (src/relax.f90:685), the corrector's with Dt (:806) --
and makes the step take the host's Dt before its first Green's function, so
it runs without the captured graph; a second event at t = 1.0 brings its
own loads through the event branch.  The oracle replays the GPU's Dt
sequence.  Tolerances: relative L2 <= 1e-4 of every field after the run
against both oracle builds; the logs to 1e-3 (test_gpu_step.check_logs).
"""
import numpy as np
import pytest

from cases import loads_small, rel_l2
from test_gpu_step import check_logs, compare, gpu_run

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("periodic,second_event,nsteps", [(False, False, 3), (True, False, 3), (True, True, 5)])
def test_loads_match_oracles(oracle32, oracle64, periodic, second_event, nsteps):
    sim = loads_small(periodic=periodic, second_event=second_event)
    glogs, gf, _ = gpu_run(sim, nsteps)
    assert len(glogs) == nsteps + 1
    dts = [lg[1] for lg in glogs[1:]]
    if second_event:
        assert any(abs(lg[5] - 1.0) < 1e-9 for lg in glogs), [lg[5] for lg in glogs]
    rlogs, rf = oracle32.run(sim, nsteps, dt_schedule=dts)
    check_logs(glogs, rlogs, 1e-3)
    compare(gf, rf, 1e-4)
    _, df = oracle64.run(sim, nsteps, dt_schedule=dts)
    compare(gf, df, 1e-4)


def test_loads_change_the_solution():
    """The loads are not silently dropped: the surface displacement with
    loads differs from the same deck without them by far more than the
    parity tolerance."""
    with_loads = loads_small(periodic=True, second_event=False)
    without = loads_small(periodic=False, second_event=False)
    without.events[0].loads = []
    _, ga, _ = gpu_run(with_loads, 2)
    _, gb, _ = gpu_run(without, 2)
    assert rel_l2(ga["u"][:, 0, :, :-2], gb["u"][:, 0, :, :-2]) > 1e-2
    # and the periodic load's rate moves the solution between steps: the
    # difference to a deck with the step load alone grows with time
    step_only = loads_small(periodic=False, second_event=False)
    _, gc, _ = gpu_run(step_only, 2)
    assert np.abs(ga["u"] - gc["u"]).max() > 0
