"""Checkpoint and restart (no counterpart in the reference): a context
restored from a checkpoint continues bit for bit -- the same log lines and
fields -- as the context that wrote it, across afterslip planes, transient
rheology, a later coseismic event and the tracked relaxation fields; files
of another configuration, truncated or corrupted, are rejected."""
import numpy as np
import pytest

from relax_b200 import _lib
from relax_b200.api import Relax

from cases import linear_small, powerlaw_small, transient_small, two_events

pytestmark = pytest.mark.gpu


def _fields(r, transient):
    names = ["u", "sig", "tau", "moment", "gamma"] + (["eps"] if transient else [])
    return {n: r.field(n) for n in names}


CASES = {
    "powerlaw-afterslip": (lambda: powerlaw_small(sx=64, sz=32), 3, 3, False),
    "transient": (lambda: transient_small(linear=True, nonlinear=True, viscous=True), 2, 3, False),
    "two-events": (lambda: two_events(), 2, 3, False),     # the event at t = 1 fires after the restart
    "tracked": (lambda: linear_small(steps=8), 2, 3, True),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_restart_continues_bit_for_bit(tmp_path, name):
    make, before, after, track = CASES[name]
    sim = make()
    transient = bool(sim.ltransient or sim.nltransient)
    path = tmp_path / "state.ckpt"
    with Relax(sim) as r:
        if track:
            r.track_relaxation(vel_planes=4, ur_planes=3, inter_i3=5)
        r.coseismic()
        for _ in range(before):
            r.step()
        r.save(path)
        logs_a = [r.step() for _ in range(after)]
        fa = _fields(r, transient)
        pa = [np.ctypeslib.as_array(r.patches(k)).copy() for k in range(sim_np(r))]
        va = [r.plane("v", 1), r.plane("ur", 2), r.plane("ur", 5)] if track else []
        ta = r.time()
    with Relax(sim) as r:
        if track:
            r.track_relaxation(vel_planes=4, ur_planes=3, inter_i3=5)
        r.load(path)
        logs_b = [r.step() for _ in range(after)]
        fb = _fields(r, transient)
        pb = [np.ctypeslib.as_array(r.patches(k)).copy() for k in range(sim_np(r))]
        vb = [r.plane("v", 1), r.plane("ur", 2), r.plane("ur", 5)] if track else []
        tb = r.time()
    assert logs_a == logs_b
    assert ta == tb
    for n in fa:
        assert fa[n].tobytes() == fb[n].tobytes(), n
    for a, b in zip(pa, pb):
        assert a.tobytes() == b.tobytes()
    for a, b in zip(va, vb):
        assert a.tobytes() == b.tobytes()


def sim_np(r):
    return r.cfg.np


def test_bad_checkpoints_are_rejected(tmp_path):
    sim = linear_small()
    path = tmp_path / "a.ckpt"
    with Relax(sim) as r:
        r.coseismic()
        r.step()
        r.save(path)
    # another grid
    with Relax(linear_small(sx=32, sz=32)) as r:
        with pytest.raises(_lib.RelaxError) as e:
            r.load(path)
        assert e.value.code == 5
    raw = path.read_bytes()
    bad = tmp_path / "b.ckpt"
    with Relax(sim) as r:
        bad.write_bytes(raw[:-100])                    # truncated
        with pytest.raises(_lib.RelaxError, match="truncated or corrupt"):
            r.load(bad)
        flipped = bytearray(raw)
        flipped[len(raw) // 2] ^= 0x40                 # one bit of the payload
        bad.write_bytes(bytes(flipped))
        with pytest.raises(_lib.RelaxError, match="truncated or corrupt"):
            r.load(bad)
        bad.write_bytes(b"not a checkpoint at all" * 10)
        with pytest.raises(_lib.RelaxError, match="not a checkpoint"):
            r.load(bad)
        r.load(path)                                   # the good file still loads
        assert r.time()[1] == 1
