"""The input decks echoed in the reference's captured runs, read by the
library's input reader (src/input.f90:43-1767).

tests/golden/reference_output{2,3,4}.input are the inputs that
examples/tutorials/output{2,3,4}.param echo, turned back into input files by
tests/golden/make_reference_logs.py.  The decks of output2 (power law n = 3)
and output3 (afterslip) read back to the same relax_config as the
transcriptions reference_output2/3 in relax_b200.config; output4 (linear
Maxwell between 2 and 3 km, a linear weak zone, five stress observation
segments) has no transcription and is checked record by record.  Host code
only: runs on the CPU."""
import math
import os

import pytest

from relax_b200 import _lib
from relax_b200.api import Input
from relax_b200.config import reference_output2, reference_output3

from test_input import compare

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def read_deck(run):
    with open(os.path.join(GOLDEN, f"reference_{run}.input")) as f:
        return Input.parse(f.read())


@pytest.mark.parametrize("run,builder", [("output2", reference_output2), ("output3", reference_output3)])
def test_echoed_deck_reads_to_the_transcription(run, builder):
    inp = read_deck(run)
    sim = builder()
    want, _keep = sim.to_c(_lib.structure_fn)
    compare(inp.config, want, sim.sx3h)
    assert inp.info.wdir == run.encode()


def test_output4_deck_records():
    inp = read_deck("output4")
    c = inp.config
    assert (c.sx1, c.sx2, c.sx3) == (256, 256, 256)
    assert (c.dx1, c.beta, c.nyquist) == (0.05, 0.2, 1.0)
    assert (c.lambda_, c.mu, c.gam) == (1.0, 1.0, 8.33e-4)
    assert (c.interval, c.odt, c.tscale, c.skip) == (2.0, -1.0, 1.0, 1)
    # viscoelasticstructure of (2, 1), (3, 1), (3, 0): gammadot0 = 1 from
    # 2 km to 3 km, 0 below (the layers hold the depth of their top)
    lin = c.linearstruc
    for k in range(c.sx3 // 2):
        z = k * c.dx3
        want = 1.0 if 2.0 <= z < 3.0 else 0.0
        if abs(z - 2.0) > 1e-9 and abs(z - 3.0) > 1e-9:
            assert lin[k].gammadot0 == pytest.approx(want, abs=1e-12), (k, z, lin[k].gammadot0)
    assert not c.nonlinearstruc and not c.faultcreepstruc
    assert list(inp.info.nwz) == [1, 0, 0, 0]
    wz = inp.weakzones(0)
    assert len(wz) == 1 and wz[0].dgammadot0 == 1.0 and wz[0].thickness == 1.0
    seg = inp.segments()
    assert len(seg) == 5 and all(s.friction == 0.6 for s in seg)
    # strikes 0 and 90 degrees in the deck: 90 degrees apart after the convention
    d = math.degrees(seg[1].strike - seg[0].strike)
    assert abs(abs(d) % 180.0 - 90.0) < 1e-9, d
    ev = c.events[0]
    assert (ev.ns, ev.nt, ev.nm, ev.nl) == (1, 0, 0, 0)
    # wangconvention: slip -1 -> +1 (src/input.f90:1780-1800)
    assert ev.s[0].slip == 1.0
