"""Parity on the benchmarked grids: the kernel instantiations that the
benchmark lines time, run against both oracle builds.

* C2 -- power law n = 3 under a 20-degree thrust with one afterslip plane on
  the 256 x 256 x 128 box (dx = 0.5 km): the x passes run with M = sx1/2 =
  128 (k_xfwd_reg<DIV, 16, 8>, k_xinv_reg<16, 8>), the y pass with 16 x 16,
  the z pass with 16 x 8.  One step (<= 1e-5) and four steps (<= 1e-4).
* C1 -- linear Maxwell on the 128^2 x 128 box for its full 20 steps at
  Dt = 0.5 (<= 1e-4 after the run).
* C3 shape -- three seeded faults with gravity and n = 3.5 below a 25 km lid
  on a box of the large instance's x1 length (sx1 = 512: the M = 256 x
  passes), narrowed along x2 and x3 so that the oracle finishes in seconds;
  and on a box of its depth (sx3 = 256: the pruned z pass with 16 x 16),
  narrowed along x1 and x2.

The GPU run is adaptive; the oracles replay its Dt sequence (a fixed dt
schedule).  Tolerances: relative L2 of u, sig, tau (gamma 3x, see
test_gpu_step.compare) against the FP32 oracle and against the FP64 oracle.
"""
import pytest

from relax_b200.config import linear_maxwell, powerlaw_thrust, random_faults

from test_gpu_step import check_logs, compare, gpu_run

pytestmark = pytest.mark.gpu


def _replay(oracle32, oracle64, sim, nsteps, tol):
    glogs, gf, _ = gpu_run(sim, nsteps)
    assert len(glogs) == nsteps + 1
    dts = [lg[1] for lg in glogs[1:]]
    rlogs, rf = oracle32.run(sim, nsteps, dt_schedule=dts)
    check_logs(glogs, rlogs, 10 * tol)
    e32 = compare(gf, rf, tol)
    _, df = oracle64.run(sim, nsteps, dt_schedule=dts)
    e64 = compare(gf, df, tol)
    return glogs, e32, e64


@pytest.mark.parametrize("nsteps", [1, 4])
def test_c2_benchmark_grid_matches_oracles(oracle32, oracle64, nsteps):
    sim = powerlaw_thrust(sx=256, sz=128, dx=0.5)
    tol = 1e-5 if nsteps == 1 else 1e-4
    glogs, e32, e64 = _replay(oracle32, oracle64, sim, nsteps, tol)
    # the adaptive step of the oracle itself agrees with the GPU's
    alogs, _ = oracle32.run(sim, 1, fields=False)
    assert abs(alogs[1][1] - glogs[1][1]) <= 2e-5 * alogs[1][1]


def test_c1_full_run_matches_oracles(oracle32, oracle64):
    sim = linear_maxwell(sx=128, sz=128, dx=0.8, steps=20)
    glogs, _, _ = _replay(oracle32, oracle64, sim, 20, 1e-4)
    assert all(lg[1] == 0.5 for lg in glogs[1:])
    assert abs(glogs[-1][5] - 10.0) < 1e-12


def test_c3_shape_matches_oracles(oracle32, oracle64):
    sim = random_faults(1, sx=512, sx2=64, sz=64, dx=1.0, lmax=40.0)
    _replay(oracle32, oracle64, sim, 3, 1e-4)


def test_c3_depth_matches_oracles(oracle32, oracle64):
    sim = random_faults(1, sx=64, sx2=64, sz=256, dx=1.0, lmax=40.0)
    _replay(oracle32, oracle64, sim, 3, 1e-4)
