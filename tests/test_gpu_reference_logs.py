"""The GPU time loop against the reference's own captured runs.

examples/tutorials/output2.param (power law n = 3, 120 steps),
output3.param (afterslip, 26 steps) and output4.param (linear Maxwell with
a weak zone, 30 steps) log Dt, the Maxwell times, t, the power and C:E^i of
every step to 3 significant figures (src/relax.f90:1100-1105).  Their echoed
input decks (tests/golden/reference_output{2,3,4}.input) are read by the
library's input reader and run on the GPU at their full 256^3 size for
every logged step; each printed value must agree with the log to one unit
in its 3rd digit or RTOL of the value.

The logs come from older builds of the reference than its current source:

* output4's weak zone was smoothed with the input's beta (0.2): its
  tm(ve) = 0.667 = 1/(1 + 0.5) is the layer's fluidity 1 plus half the
  zone's 1 at the zone's lower edge (2 km), the value of the taper there.
  The current source builds the zone with beta = 0 (src/relax.f90:487),
  which gives the full 1 at that edge and tm(ve) = 0.5.  The test runs
  both: the log with the zone built at beta = 0.2 (Dt, tm(ve) and t then
  agree with every line to 0.05 %), and the current source's field, whose
  tm(ve) must be exactly 0.5.  The log's power (the amplitude of the
  moment-density rate) decays 0.08 % per step faster than here (0.14 %
  apart at step 1, 2.4 % at step 30) and its C:E^i grows 0.02 % per step
  slower (0.6 % apart at step 30): bounds RTOL4_POWER and RTOL4_CEI.
* output2 (an MKL build) differs from step 1 by 0.2 % in Dt and tm(pl) (a
  minimum over the grid of 1/gammadot, i.e. of the peak stress; the FP32
  and FP64 oracles agree with the GPU there to 1e-5).  With the adaptive
  time step that difference is carried along the nonlinear relaxation;
  the bound is RTOL2_EARLY over the first 10 steps and RTOL2 after.
"""
import ctypes as C
import json
import math
import os

import numpy as np
import pytest

from relax_b200 import _lib
from relax_b200.api import Relax
from relax_b200.config import relax_weakzone

from test_reference_decks import read_deck

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_logs.json")
RTOL = 5e-3
RTOL2_EARLY = 3e-3
RTOL2 = 2.5e-2
RTOL4_POWER = 3e-2
RTOL4_CEI = 1e-2


def _close(ours, ref, rtol):
    if ref == 0.0:
        return abs(ours) < 1e-12
    ulp3 = 10.0 ** (math.floor(math.log10(abs(ref))) - 2)
    return abs(ours - ref) <= max(1.01 * ulp3, rtol * abs(ref))


def _run(relax, nsteps):
    logs = [relax.coseismic()]
    for _ in range(nsteps):
        lg = relax.step()
        if lg[0] == 0:
            break
        logs.append(lg)
    return logs


def _weakzone_field(inp, beta):
    """The deck's linear weak zones built on the device with smoothing beta
    (relax_op_dgammadot0), as a host array in the layout of relax_config."""
    c = inp.config
    zones = inp.weakzones(0)
    arr = (relax_weakzone * len(zones))(*zones)
    nh = c.sx1 * c.sx2 * (c.sx3 // 2)
    d = torch.zeros(nh, dtype=torch.float32, device="cuda")
    _lib.check(_lib.load().relax_op_dgammadot0(C.cast(arr, C.c_void_p), len(zones), c.sx1, c.sx2, c.sx3 // 2,
                                               c.dx1, c.dx2, c.dx3, beta, C.c_void_p(d.data_ptr()), None))
    torch.cuda.synchronize()
    return d.cpu().numpy()


def _compare(name, logs, ref, rtol_of_step, rtol_of_col=None):
    assert len(logs) == len(ref), (len(logs), len(ref))
    worst = {}
    bad = []
    for ours, theirs in zip(logs, ref):
        assert ours[0] == theirs[0]
        cols = (7,) if ours[0] == 0 else (1, 2, 3, 4, 5, 6, 7)
        for c in cols:
            if theirs[c] != 0:
                worst[c] = max(worst.get(c, 0.0), abs(ours[c] - theirs[c]) / abs(theirs[c]))
            rtol = rtol_of_step(ours[0]) if rtol_of_col is None else rtol_of_col(ours[0], c)
            if not _close(ours[c], theirs[c], rtol):
                bad.append((ours[0], c, ours[c], theirs[c]))
    print(name, "largest relative deviation per column", worst)
    for ours, theirs in zip(logs, ref):
        print(name, ours[0], " ".join(f"{a:.4e}/{b:.2e}" for a, b in zip(ours[1:], theirs[1:])))
    assert not bad, bad[:10]


def _ref(name):
    with open(GOLDEN) as f:
        return json.load(f)[name]


def test_gpu_reproduces_output3():
    ref = _ref("output3")
    inp = read_deck("output3")
    with Relax.from_input(inp) as r:
        logs = _run(r, len(ref) - 1)
    _compare("output3", logs, ref, lambda i: RTOL)


def test_gpu_reproduces_output2():
    ref = _ref("output2")
    inp = read_deck("output2")
    with Relax.from_input(inp) as r:
        logs = _run(r, len(ref) - 1)
    _compare("output2", logs, ref, lambda i: RTOL2_EARLY if i <= 10 else RTOL2)


def test_gpu_reproduces_output4_with_the_logs_weak_zone_smoothing():
    ref = _ref("output4")
    inp = read_deck("output4")
    field = _weakzone_field(inp, inp.config.beta)
    cfg = inp.config
    cfg.lineardgammadot0 = field.ctypes.data_as(C.POINTER(C.c_float))
    with Relax(inp.simulation(), config=cfg, keep=(inp, field)) as r:
        logs = _run(r, len(ref) - 1)
    _compare("output4", logs, ref, None, lambda i, c: RTOL4_POWER if c == 6 else RTOL4_CEI if c == 7 else RTOL)


def test_output4_current_source_weak_zone():
    """beta = 0 (src/relax.f90:487): fluidity 1 + 1 at the zone's lower edge."""
    inp = read_deck("output4")
    with Relax.from_input(inp) as r:
        r.coseismic()
        lg = r.step()
    assert lg[2] == 0.5, lg
