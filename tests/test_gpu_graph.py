"""The step as a CUDA graph: after one plain step a context replays its
step's kernels from a captured graph (steps without surface loads).  The
replayed steps equal the plain ones bit for bit -- logs, fields, afterslip
patches and kernel counts -- across afterslip planes, a coseismic event in
the middle of the run, prescribed time steps and the tracked relaxation
fields.  Per-launch profiling turns the graph off, which gives the plain
reference run."""
import numpy as np
import pytest

from relax_b200.api import Relax

from cases import linear_small, powerlaw_small, two_events

pytestmark = pytest.mark.gpu


def _run(sim, nsteps, plain, track=False, dts=None):
    with Relax(sim) as r:
        if plain:
            r.profile(True)
        if track:
            r.track_relaxation(vel_planes=3, ur_planes=2, inter_i3=4)
        r.coseismic()
        n0 = r.launch_count()
        logs = [r.step(dts[k] if dts else None) for k in range(nsteps)]
        launches = r.launch_count() - n0
        fields = {n: r.field(n) for n in ("u", "sig", "tau", "moment", "gamma")}
        patches = [np.ctypeslib.as_array(r.patches(k)).copy() for k in range(r.cfg.np)]
        extra = [r.plane("v", 1), r.plane("ur", 1), r.plane("ur", 4)] if track else []
    return logs, fields, patches, launches, extra


CASES = {
    "powerlaw-afterslip": (lambda: powerlaw_small(sx=64, sz=32), 5, False, None),
    "two-events": (lambda: two_events(), 6, False, None),
    "prescribed-dt": (lambda: linear_small(steps=8), 4, False, [0.3, 0.2, 0.25, 0.1]),
    "tracked": (lambda: linear_small(steps=8), 4, True, None),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_graph_replay_equals_plain_steps(name):
    make, nsteps, track, dts = CASES[name]
    a = _run(make(), nsteps, plain=False, track=track, dts=dts)
    b = _run(make(), nsteps, plain=True, track=track, dts=dts)
    assert a[0] == b[0]
    for n in a[1]:
        assert a[1][n].tobytes() == b[1][n].tobytes(), n
    for x, y in zip(a[2], b[2]):
        assert x.tobytes() == y.tobytes()
    assert a[3] == b[3]
    for x, y in zip(a[4], b[4]):
        assert x.tobytes() == y.tobytes()
