"""Batches (relax_batch_*): every member stepped in a batch matches the same
deck stepped alone through relax_step, bit for bit (the batched launches run
the same kernels on per-member argument tables), including afterslip planes,
a second coseismic event, members that finish early and grids without the
batched instantiation.  No reference counterpart: RELAX runs one simulation
per process."""
import copy
import dataclasses

import numpy as np
import pytest

from relax_b200 import _lib
from relax_b200.api import Batch, Relax
from cases import linear_small, powerlaw_small, two_events

pytestmark = pytest.mark.gpu


def _variant(sim, k):
    """member k: its own slip, rheology and plane position"""
    s = copy.deepcopy(sim)
    s.name = f"{sim.name}-{k}"
    f = s.events[0].faults[0]
    s.events[0].faults[0] = dataclasses.replace(f, slip=f.slip * (1.0 + 0.25 * k), x=f.x + 2.0 * k)
    s.nonlinear = [(z, g0 * (1.0 + 0.5 * k), n + 0.25 * k, c) for (z, g0, n, c) in s.nonlinear]
    s.linear = [(z, g0 * (1.0 + 0.5 * k)) for (z, g0) in s.linear]
    if s.planes:
        p = s.planes[0]
        s.planes[0] = dataclasses.replace(p, x=p.x + 3.0 * k, length=p.length - 2.0 * k)
    return s


def _alone(sim, nsteps):
    with Relax(sim) as r:
        logs = [r.coseismic()] + [r.step() for _ in range(nsteps)]
        out = {"logs": logs, "u": r.field("u"), "tau": r.field("tau"), "gamma": r.field("gamma")}
        if sim.planes:
            out["patches"] = np.array([(p.slip, p.v, p.taus) for p in r.patches(0)])
    return out


def _batched(sims, nsteps):
    with Batch(sims) as b:
        logs = [[l] for l in b.coseismic()]
        n0 = b.launch_count()
        for _ in range(nsteps):
            for k, l in enumerate(b.step()):
                logs[k].append(l)
        launches = b.launch_count() - n0
        outs = []
        for k in range(len(sims)):
            m = b.member(k)
            o = {"logs": logs[k], "u": m.field("u"), "tau": m.field("tau"), "gamma": m.field("gamma")}
            if sims[k].planes:
                o["patches"] = np.array([(p.slip, p.v, p.taus) for p in m.patches(0)])
            outs.append(o)
    return outs, launches


def _same(a, b):
    assert a["logs"] == b["logs"]
    for key in ("u", "gamma", "patches"):
        if key in a:
            assert np.array_equal(a[key], b[key]), key
    for name in a["tau"].dtype.names:
        assert np.array_equal(a["tau"][name], b["tau"][name]), name


def test_batch_matches_members_alone():
    base = powerlaw_small(sx=128, sz=64, dx=1.0)
    sims = [_variant(base, k) for k in range(3)]
    outs, launches = _batched(sims, 3)
    for k, s in enumerate(sims):
        _same(outs[k], _alone(s, 3))
    # one launch per stage for all members: 2 friction + dt + 5 + corr + friction + monitor + 5 + end
    # (the tuner's first three steps are batched)
    assert launches == 3 * 16


def test_batch_linear_members_finish_at_their_interval():
    base = linear_small(sx=128, sz=64, steps=3)
    sims = [_variant(base, k) for k in range(3)]
    sims[1].interval = 4.0
    outs, _ = _batched(sims, 8)
    for k, s in enumerate(sims):
        ref = _alone(s, 8)
        # members past their interval report i = 0 (as relax_step does) and stay put
        if k != 1:
            assert ref["logs"][-1][0] == 0
        _same(outs[k], ref)


def test_batch_event_fires_in_one_member():
    ev = two_events(sx=128, sz=64)
    plain = linear_small(sx=128, sz=64, steps=8)
    plain.tscale = 3.0
    sims = [ev, plain]
    outs, _ = _batched(sims, 5)
    assert any(l[1] for l in outs[0]["logs"][1:]), "the second event fires within 5 steps"
    for k, s in enumerate(sims):
        _same(outs[k], _alone(s, 5))


def test_batch_without_batched_passes_steps_members_in_turn():
    # x1 length 96 has no register instantiation
    base = linear_small(sx=96, sz=64, steps=3)
    sims = [_variant(base, k) for k in range(2)]
    outs, _ = _batched(sims, 3)
    for k, s in enumerate(sims):
        _same(outs[k], _alone(s, 3))


@pytest.mark.parametrize("sx,sz", [(64, 64), (192, 96), (64, 128)])
def test_batch_ensemble_shapes(sx, sz):
    """the grid shapes of the uneven ensemble that need the 8 x 4 and 24 x 4 / 24 x 8 passes, and
    the 128-deep z pass"""
    base = powerlaw_small(sx=sx, sz=sz, dx=1.0, afterslip=False)
    sims = [_variant(base, k) for k in range(2)]
    outs, launches = _batched(sims, 2)
    for k, s in enumerate(sims):
        _same(outs[k], _alone(s, 2))
    assert launches == 2 * 13   # dt + 5 + corr + 5 + end per step


def test_batch_rejects_mismatched_members():
    a = linear_small(sx=128, sz=64)
    b = linear_small(sx=128, sz=64)
    b.mu = 2.0
    with pytest.raises(_lib.RelaxError) as e:
        Batch([a, b])
    assert e.value.code == 1


def test_ensemble_of_uneven_grids_matches_members_alone():
    """relax_ensemble_*: members of three shapes (two batched groups and a
    grid stepped in turn), interleaved in the member list, each equal to
    its deck stepped alone; one host synchronisation per ensemble step."""
    from relax_b200.api import Ensemble
    a = powerlaw_small(sx=64, sz=64, dx=1.0, afterslip=False)
    b = powerlaw_small(sx=128, sz=64, dx=1.0)
    c = linear_small(sx=96, sz=64, steps=3)
    sims = [_variant(a, 0), _variant(b, 0), _variant(c, 0), _variant(a, 1), _variant(b, 1)]
    with Ensemble(sims) as e:
        assert e.groups() == 3
        logs = [[l] for l in e.coseismic()]
        for _ in range(3):
            for k, l in enumerate(e.step()):
                logs[k].append(l)
        outs = []
        for k in range(len(sims)):
            m = e.member(k)
            o = {"logs": logs[k], "u": m.field("u"), "tau": m.field("tau"), "gamma": m.field("gamma")}
            if sims[k].planes:
                o["patches"] = np.array([(p.slip, p.v, p.taus) for p in m.patches(0)])
            outs.append(o)
    for k, s in enumerate(sims):
        _same(outs[k], _alone(s, 3))


def test_batch_tuner_chooses_a_form_and_keeps_members_exact():
    """The batch's tuner: steps 1-3 batched (the third timed), 4-6 with the
    members in turn (the sixth timed), then the faster form; every step of
    either form leaves each member equal to its deck stepped alone."""
    base = powerlaw_small(sx=64, sz=64, dx=1.0)
    sims = [_variant(base, k) for k in range(3)]
    with Batch(sims) as b:
        logs = [[l] for l in b.coseismic()]
        states = []
        for step in range(8):
            for k, l in enumerate(b.step()):
                logs[k].append(l)
            states.append(b.tuning())
        outs = []
        for k in range(len(sims)):
            m = b.member(k)
            o = {"logs": logs[k], "u": m.field("u"), "tau": m.field("tau"), "gamma": m.field("gamma"),
                 "patches": np.array([(p.slip, p.v, p.taus) for p in m.patches(0)])}
            outs.append(o)
    assert [s["mode"] for s in states[:5]] == ["measuring"] * 5
    assert states[2]["batched_ms"] > 0 and states[4]["in_turn_ms"] < 0
    final = states[-1]
    assert final["mode"] in ("batched", "in turn")
    assert final["batched_ms"] > 0 and final["in_turn_ms"] > 0
    assert final["mode"] == ("batched" if final["batched_ms"] <= final["in_turn_ms"] else "in turn")
    for k, s in enumerate(sims):
        _same(outs[k], _alone(s, 8))


def test_ensemble_reports_each_group_tuning():
    from relax_b200.api import Ensemble
    a = powerlaw_small(sx=64, sz=64, dx=1.0, afterslip=False)
    c = linear_small(sx=96, sz=64, steps=8)
    sims = [_variant(a, 0), _variant(c, 0), _variant(a, 1)]
    with Ensemble(sims) as e:
        e.coseismic()
        for _ in range(7):
            e.step()
        t = e.tuning()
    assert [g["grid"] for g in t] == [(64, 64, 64), (96, 96, 64)]
    assert [g["members"] for g in t] == [2, 1]
    assert t[0]["mode"] in ("batched", "in turn") and t[0]["batched_ms"] > 0 and t[0]["in_turn_ms"] > 0
    assert t[1]["mode"] == "in turn"   # one member: nothing to batch


def test_batch_of_transient_members_matches_members_alone():
    """Members with the transient (Burgers) rheology and a viscous layer:
    the batched TRANS instantiations of the corrector and END passes (the
    tuner's first three steps are batched, the fourth in turn)."""
    from cases import transient_small
    base = transient_small(linear=True, nonlinear=True, viscous=True, sx=64, sz=64)
    sims = [_variant(base, k) for k in range(2)]
    outs, _ = _batched(sims, 4)
    for k, s in enumerate(sims):
        _same(outs[k], _alone(s, 4))
