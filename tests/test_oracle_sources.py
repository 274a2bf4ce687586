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


# --------------------------------------------------------------------------
# eigenstrain sources (--with-eigenstrain, --with-curvilinear)
# --------------------------------------------------------------------------
def _divergence_check(oracle64, body, moment, n, h, net=1e-9):
    """the analytic body force of a source against the reference's
    divergence stencil (equivalentbodyforce) applied to the source's moment
    density: both discretise f = -div m of one eigenstrain"""
    import numpy as np
    from oracle.oracle import TENSOR64_DTYPE
    f = np.zeros((3, n, n, n + 2))
    body(f)
    m = np.zeros((n // 2, n, n), TENSOR64_DTYPE)
    moment(m)
    c = np.zeros((3, n, n, n + 2))
    t = np.zeros((3, n, n + 2))
    oracle64.bodyforce(m, (h, h, h), n, n, n // 2, c, t)
    fa, fd = f[:, : n // 2, :, :n], c[:, : n // 2, :, :n]
    # no net force: the divergence of a compact moment (to the truncation of
    # the tetrahedron's Gaussians at 7 dx1)
    assert np.abs(fa.sum(axis=(1, 2, 3))).max() < net * np.abs(fa).sum()
    errs = []
    for k in range(3):
        a, b = fa[k].ravel(), fd[k].ravel()
        errs.append((rel_l2(a, b), float(np.corrcoef(a, b)[0, 1])))
    return errs


def test_cuboid_body_force_is_the_divergence_of_its_moment(oracle64):
    """cuboidSource (src/elastic3d.f90:1680-1884) and momentDensityCuboid
    (:2927-3029) restated: at half the taper width per grid step the two
    agree to the stencil's error (which halves with the step)."""
    from relax_b200.config import relax_tensor
    e = relax_tensor(1e-2, 4e-3, -3e-3, -5e-3, 2e-3, 6e-3)
    geo = (0.0, 0.0, 12.0, 10.0, 12.0, 6.0, 0.3, 0.5)
    n, h = 128, 0.5
    errs = _divergence_check(
        oracle64,
        lambda f: oracle64.cuboidsource(1.0, 1.0, e, geo, 0.2, (n, n, n), (h, h, h), f),
        lambda m: oracle64.momentdensitycuboid(1.0, 1.0, e, geo, 0.2, n, n, n // 2, (h, h, h), m), n, h)
    for k, (err, corr) in enumerate(errs):
        assert err < 0.25 and corr > 0.99, (k, errs)


def test_tetrahedron_body_force_is_the_divergence_of_its_moment(oracle64):
    """tetrahedronSource (src/elastic3d.f90:1916-2039) and
    momentDensityTetrahedron (:2788-2873) on a tetrahedron whose inradius
    exceeds the 7 dx1 band of the moment's point test."""
    import numpy as np
    from relax_b200.config import relax_tensor
    e = relax_tensor(5e-3, 1e-3, 2e-3, -4e-3, -1e-3, 1e-3)
    V = [np.array(v) for v in ((-15.0, -12.0, 3.0), (22.0, -10.0, 4.0), (0.0, 24.0, 2.0), (2.0, 1.0, 28.0))]
    n, h = 128, 0.5
    errs = _divergence_check(
        oracle64,
        lambda f: oracle64.tetrahedronsource(1.0, 1.0, e, V, (n, n, n), (h, h, h), f),
        lambda m: oracle64.momentdensitytetrahedron(1.0, 1.0, e, V, n, n, n // 2, (h, h, h), m), n, h, net=1e-6)
    for k, (err, corr) in enumerate(errs):
        assert err < 0.25 and corr > 0.99, (k, errs)


def test_eigenstrain_fp32_and_fp64_oracles_agree(oracle32, oracle64):
    from cases import eigenstrain_small
    s = eigenstrain_small()
    l32, f32 = oracle32.run(s, 2)
    dts = [l[1] for l in l32[1:]]
    _, f64 = oracle64.run(s, 2, dt_schedule=dts)
    assert np.abs(f32["u"]).max() > 0
    assert rel_l2(f32["u"][..., :-2], f64["u"][..., :-2]) < 1e-5
    assert rel_l2(tensor_array(f32["tau"]), tensor_array(f64["tau"])) < 1e-5
