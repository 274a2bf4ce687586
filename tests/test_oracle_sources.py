"""The oracle's tensile cracks and dilatation point sources
(tensilesource / mogisource, src/elastic3d.f90:2315-2509, and their moment
densities :3137-3286) in the coseismic solve and the interseismic loading."""
import numpy as np

from relax_b200.config import Event, Point

from cases import linear_small, rel_l2, tensor_array, sources_small


def test_point_source_field_is_symmetric(oracle32):
    """a point source on the box axis: u3 even in x2 (exactly) and in x1, u1 odd
    in x1.  Along x1 the symmetry holds to the Nyquist mode: the R2C axis
    takes its Nyquist wavenumber as +1/(2 dx1) (src/fourier.f90:64-113)
    and the Cerruti terms odd in k1 see that sign."""
    s = linear_small(64, 32)
    s.events = [Event(0.0, [], points=[Point(1.0, 0.0, 0.0, 6.0)])]
    _, f = oracle32.run(s, 0)
    u = f["u"][..., :64]
    u1, u3 = u[0], u[2]
    flip = lambda a, ax: np.roll(np.flip(a, axis=ax), 1, axis=ax)   # index i -> -i
    assert np.abs(u3).max() > 0
    assert np.allclose(u3, flip(u3, 1), atol=1e-6 * np.abs(u3).max())
    assert np.allclose(u3, flip(u3, 2), atol=1e-2 * np.abs(u3).max())
    assert np.allclose(u1, -flip(u1, 2), atol=1e-2 * np.abs(u1).max())


def test_sources_fp32_and_fp64_oracles_agree(oracle32, oracle64):
    s = sources_small(interseismic=True)
    l32, f32 = oracle32.run(s, 2)
    dts = [l[1] for l in l32[1:]]
    _, f64 = oracle64.run(s, 2, dt_schedule=dts)
    assert rel_l2(f32["u"][..., :-2], f64["u"][..., :-2]) < 1e-5
    assert rel_l2(tensor_array(f32["tau"]), tensor_array(f64["tau"])) < 1e-5
