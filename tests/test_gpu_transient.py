"""Transient (Burgers) rheology on the GPU against the oracle: the
predictor's and corrector's transienteigenstress calls fused into the stress
passes (including the corrector's in-place reading of epsilonikdot,
src/relax.f90:768-786), the two extra Maxwell times and the 5-mechanism time
step (src/relax.f90:660-664)."""
import pytest

from relax_b200.api import Relax

from cases import transient_small
from test_gpu_step import check_logs, compare

pytestmark = pytest.mark.gpu


def _gpu(sim, nsteps):
    with Relax(sim) as r:
        logs, tmt = [r.coseismic()], []
        for _ in range(nsteps):
            lg = r.step()
            if lg[0] == 0:
                break
            logs.append(lg)
            tmt.append((r.last_log.tm_tl, r.last_log.tm_tnl))
        fields = {k: r.field(k) for k in ("u", "sig", "tau", "gamma")}
    return logs, tmt, fields


@pytest.mark.parametrize("kind", ["linear", "nonlinear", "both+viscous"])
@pytest.mark.parametrize("nsteps", [1, 4])
def test_transient_run_matches_oracle(oracle32, oracle64, kind, nsteps):
    sim = transient_small(linear=kind != "nonlinear", nonlinear=kind != "linear",
                          viscous=kind == "both+viscous")
    glogs, gtm, gf = _gpu(sim, nsteps)
    dts = [l[1] for l in glogs[1:]]
    rlogs, rf = oracle32.run(sim, nsteps, dt_schedule=dts)
    tol = 1e-5 if nsteps == 1 else 1e-4
    check_logs(glogs, rlogs, 10 * tol)
    for g, o in zip(gtm, rf["tm_transient"][1:]):
        for a, b in zip(g, o):
            assert abs(a - b) <= 1e-5 * abs(b), (g, o)
    compare(gf, rf, tol)
    _, df = oracle64.run(sim, nsteps, dt_schedule=dts)
    compare(gf, df, tol)
    # the adaptive step of the oracle agrees with the GPU's
    alogs, _ = oracle32.run(sim, 1, fields=False)
    assert abs(alogs[1][1] - glogs[1][1]) <= 1e-5 * alogs[1][1]
