"""Tensile cracks and dilatation point sources on the GPU against the
oracle: the coseismic solve over the whole box (their images lie below the
surface, so the x3 transform is not pruned), the moment densities removed
from tau, and interseismic shear and tensile loading in the corrector."""
import pytest

from cases import sources_small
from test_gpu_step import check_logs, compare, gpu_run

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nsteps,interseismic", [(0, False), (3, False), (3, True)])
def test_sources_match_oracle(oracle32, oracle64, nsteps, interseismic):
    sim = sources_small(interseismic=interseismic)
    glogs, gf, _ = gpu_run(sim, nsteps)
    dts = [l[1] for l in glogs[1:]]
    rlogs, rf = oracle32.run(sim, nsteps, dt_schedule=dts)
    tol = 1e-5 if nsteps <= 1 else 1e-4
    check_logs(glogs, rlogs, 10 * tol)
    compare(gf, rf, tol)
    _, df = oracle64.run(sim, nsteps, dt_schedule=dts)
    compare(gf, df, tol)


@pytest.mark.parametrize("nsteps", [0, 3])
def test_eigenstrain_sources_match_oracle(oracle32, oracle64, nsteps):
    """Cuboid (dipping, and vertical with the method of images) and
    tetrahedral eigenstrain: body forces and the moment densities removed
    from tau (cuboidSource, tetrahedronSource, momentDensityCuboid,
    momentDensityTetrahedron, src/elastic3d.f90:1680-2039, 2788-3029)."""
    from cases import eigenstrain_small
    sim = eigenstrain_small()
    glogs, gf, _ = gpu_run(sim, nsteps)
    dts = [l[1] for l in glogs[1:]]
    rlogs, rf = oracle32.run(sim, nsteps, dt_schedule=dts)
    tol = 1e-5 if nsteps <= 1 else 1e-4
    check_logs(glogs, rlogs, 10 * tol)
    compare(gf, rf, tol)
    _, df = oracle64.run(sim, nsteps, dt_schedule=dts)
    compare(gf, df, tol)
