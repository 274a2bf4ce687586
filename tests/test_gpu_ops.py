"""Per-operator parity of the CUDA kernels with the CPU oracle (FP32
restatement of the reference), called through the C ABI on device buffers.

Tolerance (floating point): relative L2 <= 1e-5 per operator unless noted;
the minimum-reduction Maxwell times agree to 1e-5 relative.
"""
import ctypes as C

import numpy as np
import pytest

from relax_b200 import _lib
from relax_b200.config import TENSOR_DTYPE, relax_layer, relax_plane, relax_tensor_layer

from cases import rel_l2, tensor_array

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def ptr(t):
    return C.c_void_p(t.data_ptr())


def host(t, like):
    return t.cpu().numpy().view(like.dtype).reshape(like.shape)


def tensors_random(rng, shape, scale=1.0):
    t = np.zeros(shape, TENSOR_DTYPE)
    for n in TENSOR_DTYPE.names:
        t[n] = scale * rng.standard_normal(shape)
    return t


def tensors_smooth(shape, scale=0.1, seed=0):
    rng = np.random.default_rng(seed)
    sz, sy, sx = shape
    z, y, x = np.meshgrid(np.arange(sz), np.arange(sy), np.arange(sx), indexing="ij")
    t = np.zeros(shape, TENSOR_DTYPE)
    for k, n in enumerate(TENSOR_DTYPE.names):
        a, b, c, d = rng.uniform(0.5, 2.0, 4)
        t[n] = scale * (np.sin(2 * np.pi * a * x / sx + d) * np.cos(2 * np.pi * b * y / sy) *
                        np.exp(-c * z / sz) + 0.3 * (k - 2.5))
    return t


GRIDS = [(32, 32, 32), (64, 48, 32), (96, 32, 36)]
# grids of the 7-point FIR differentiator along x2 (5 <= sx2 <= 14: 6, 8, 9,
# 12; sx2 = 6 wraps the 7 taps around the axis), along x1 (sx1 = 8, 12) or
# both, and of shallow boxes (5 <= sx3/2 <= 14, finite differences
# throughout), and sx2 = 4
FIR_GRIDS = [(32, 8, 16), (32, 6, 12), (48, 12, 24), (64, 9, 18), (32, 4, 12), (8, 32, 16), (12, 16, 12),
             (8, 6, 18), (12, 12, 24)]


@pytest.mark.parametrize("sx1,sx2,sx3", GRIDS + [(16, 12, 8), (128, 96, 64)])
def test_fft3_matches_oracle(oracle32, sx1, sx2, sx3):
    lib = _lib.load()
    rng = np.random.default_rng(sx1 + sx2 + sx3)
    dx = (0.5, 0.7, 0.3)
    a = np.zeros((sx3, sx2, sx1 + 2), np.float32)
    a[:, :, :sx1] = rng.standard_normal((sx3, sx2, sx1))
    ref = a.copy()
    oracle32.fft3(ref, sx1, sx2, sx3, *dx, -1)
    d = dev(a)
    _lib.check(lib.relax_op_fft3(ptr(d), sx1, sx2, sx3, *dx, -1, None))
    torch.cuda.synchronize()
    got = d.cpu().numpy()
    assert rel_l2(got, ref) < 2e-6
    _lib.check(lib.relax_op_fft3(ptr(d), sx1, sx2, sx3, *dx, +1, None))
    torch.cuda.synchronize()
    back = d.cpu().numpy()[:, :, :sx1]
    assert rel_l2(back, a[:, :, :sx1]) < 2e-6


@pytest.mark.parametrize("sx1,sx2,sx3", GRIDS + FIR_GRIDS)
def test_stressupdate_matches_oracle(oracle32, sx1, sx2, sx3):
    lib = _lib.load()
    sx3h = sx3 // 2
    rng = np.random.default_rng(7)
    u = np.zeros((3, sx3h, sx2, sx1 + 2), np.float32)
    u[:, :, :, :sx1] = rng.standard_normal((3, sx3h, sx2, sx1))
    sig = tensors_random(rng, (sx3h, sx2, sx1))
    dx = (0.5, 0.4, 0.25)
    ref = sig.copy()
    oracle32.stressupdate(u, 1.3, 0.8, dx, sx1, sx2, sx3h, ref)
    du = [dev(u[k]) for k in range(3)]
    ds = dev(sig.view(np.float32))
    _lib.check(lib.relax_op_stressupdate(ptr(du[0]), ptr(du[1]), ptr(du[2]), 1.3, 0.8, *dx, sx1, sx2,
                                         sx3h, ptr(ds), None))
    torch.cuda.synchronize()
    got = ds.cpu().numpy().view(TENSOR_DTYPE).reshape(sig.shape)
    assert rel_l2(tensor_array(got), tensor_array(ref)) < 1e-6


@pytest.mark.parametrize("sx1,sx2,sx3", GRIDS + FIR_GRIDS)
def test_bodyforce_matches_oracle(oracle32, sx1, sx2, sx3):
    lib = _lib.load()
    sx3h = sx3 // 2
    rng = np.random.default_rng(8)
    sig = tensors_random(rng, (sx3h, sx2, sx1))
    dx = (0.5, 0.4, 0.25)
    c = np.zeros((3, sx3, sx2, sx1 + 2), np.float32)
    t = np.zeros((3, sx2, sx1 + 2), np.float32)
    cr, tr = c.copy(), t.copy()
    oracle32.bodyforce(sig, dx, sx1, sx2, sx3h, cr, tr)
    dc = [dev(c[k]) for k in range(3)]
    dt = [dev(t[k]) for k in range(3)]
    dsig = dev(sig.view(np.float32))   # held: a temporary's block may be reused
    _lib.check(lib.relax_op_bodyforce(ptr(dsig), *dx, sx1, sx2, sx3h,
                                      *[ptr(x) for x in dc], *[ptr(x) for x in dt], None))
    torch.cuda.synchronize()
    gc = np.stack([x.cpu().numpy() for x in dc])
    gt = np.stack([x.cpu().numpy() for x in dt])
    assert rel_l2(gc, cr) < 1e-6
    assert rel_l2(gt, tr) == 0.0


@pytest.mark.parametrize("power", [1.0, 3.0, 3.5])
@pytest.mark.parametrize("prestress", [False, True])
def test_viscous_eigenstress_matches_oracle(oracle32, power, prestress):
    lib = _lib.load()
    sx1, sx2, sx3 = 64, 32, 32
    sx3h = sx3 // 2
    rng = np.random.default_rng(9)
    sig = tensors_random(rng, (sx3h, sx2, sx1), 0.3)
    mom = tensors_random(rng, (sx3h, sx2, sx1), 0.1)
    st = (relax_layer * sx3h)()
    for k in range(sx3h):
        st[k] = relax_layer(z=0, gammadot0=(0.0 if k < 3 else 10 ** rng.uniform(-1, 1)),
                            stressexponent=power, cohesion=(0.05 if k == 5 else 0.0), friction=0, Gk=0)
    pre = None
    if prestress:
        pre = (relax_tensor_layer * sx3h)()
        for k in range(sx3h):
            pre[k].t.s11, pre[k].t.s22, pre[k].t.s33 = 0.02 * k, -0.01 * k, 0.03
            pre[k].t.s12 = 0.01
    gamma = np.zeros((sx3h, sx2, sx1 + 2), np.float32)
    mref, gref = mom.copy(), gamma.copy()
    rc, tref = oracle32.viscouseigenstress(1.0, st, pre, sig, sx1, sx2, sx3h, mref, maxwell=1e7,
                                           gamma=gref)
    assert rc == 0
    dm = dev(mom.view(np.float32))
    dg = dev(gamma)
    dsig = dev(sig.view(np.float32))
    tm = C.c_double(1e7)
    _lib.check(lib.relax_op_viscouseigenstress(
        1.0, C.cast(st, C.c_void_p), None if pre is None else C.cast(pre, C.c_void_p),
        ptr(dsig), sx1, sx2, sx3h, ptr(dm), C.byref(tm), ptr(dg), None, None))
    torch.cuda.synchronize()
    gm = dm.cpu().numpy().view(TENSOR_DTYPE).reshape(mom.shape)
    assert rel_l2(tensor_array(gm), tensor_array(mref)) < 1e-5
    assert rel_l2(dg.cpu().numpy(), gref) < 1e-5
    assert abs(tm.value - tref) <= 1e-5 * tref


def test_friction_eigenstress_matches_oracle(oracle32):
    lib = _lib.load()
    sx1, sx2, sx3 = 64, 64, 32
    sx3h = sx3 // 2
    sig = tensors_smooth((sx3h, sx2, sx1), 0.05, seed=3)
    mom = tensors_smooth((sx3h, sx2, sx1), 0.01, seed=4)
    st = (relax_layer * sx3h)()
    for k in range(sx3h):
        st[k] = relax_layer(z=0, gammadot0=(0.0 if k < 2 else 1.0), stressexponent=0.1, cohesion=0.0,
                            friction=(0.6 if k < 4 else 0.2), Gk=0)
    plane = relax_plane(x=-2.0, y=1.0, z=6.0, width=8.0, length=20.0, strike=0.3, dip=0.8,
                        rake=-2.0, px2=20, px3=8)
    dx = (1.0, 1.0, 1.0)
    mref = mom.copy()
    rc, tref = oracle32.frictioneigenstress(plane, 0.2, sig, 1.0, st, sx1, sx2, sx3h, dx, mref,
                                            maxwell=1e7)
    assert rc == 0
    dm = dev(mom.view(np.float32))
    dsig = dev(sig.view(np.float32))
    tm = C.c_double(1e7)
    _lib.check(lib.relax_op_frictioneigenstress(
        plane.x, plane.y, plane.z, plane.width, plane.length, plane.strike, plane.dip, plane.rake, 0.2,
        ptr(dsig), 1.0, C.cast(st, C.c_void_p), sx1, sx2, sx3h, *dx, ptr(dm),
        C.byref(tm), None))
    torch.cuda.synchronize()
    gm = dm.cpu().numpy().view(TENSOR_DTYPE).reshape(mom.shape)
    d = tensor_array(gm) - tensor_array(mom)
    dref = tensor_array(mref) - tensor_array(mom)
    assert np.abs(dref).max() > 0
    assert rel_l2(d, dref) < 1e-5
    assert abs(tm.value - tref) <= 1e-6 * tref


def test_friction_abort_is_reported(oracle32):
    """tau/((a-b)sigma) > 20 stops the reference (src/friction3d.f90:204-215);
    the library returns RELAX_ERR_FRICTION."""
    lib = _lib.load()
    sx1, sx2, sx3 = 32, 32, 32
    sx3h = sx3 // 2
    sig = tensors_smooth((sx3h, sx2, sx1), 5.0, seed=5)
    st = (relax_layer * sx3h)()
    for k in range(sx3h):
        st[k] = relax_layer(z=0, gammadot0=1.0, stressexponent=1e-3, cohesion=0.0, friction=0.0, Gk=0)
    plane = relax_plane(x=0.0, y=0.0, z=6.0, width=6.0, length=10.0, strike=0.0, dip=0.0, rake=0.0)
    mom = np.zeros((sx3h, sx2, sx1), TENSOR_DTYPE)
    rc, _ = oracle32.frictioneigenstress(plane, 0.2, sig, 1.0, st, sx1, sx2, sx3h, (1, 1, 1), mom.copy())
    assert rc == 6
    dsig = dev(sig.view(np.float32))
    dmom = dev(mom.view(np.float32))
    rc = lib.relax_op_frictioneigenstress(
        plane.x, plane.y, plane.z, plane.width, plane.length, plane.strike, plane.dip, plane.rake, 0.2,
        ptr(dsig), 1.0, C.cast(st, C.c_void_p), sx1, sx2, sx3h, 1.0, 1.0, 1.0, ptr(dmom), None, None)
    assert rc == 6


# x2/x3 lengths 64..512 take the register-resident column kernels, the others
# the shared-memory Stockham kernels
# register-resident lengths: 32 (8 x 4), 64, 96 (24 x 4), 128, 192 (24 x 8), 256, 512
# sx1 = 256 and 512 take the x passes of the benchmarked boxes (M = 128, 256);
# 256 x 256 x 128 is the C2 box itself
GREEN_GRIDS = GRIDS + [(64, 64, 64), (64, 256, 128), (32, 512, 256), (128, 128, 128), (192, 192, 96),
                       (64, 96, 96), (128, 32, 64), (256, 32, 64), (512, 32, 64), (256, 256, 128),
                       (8, 32, 16), (12, 8, 12)]


@pytest.mark.parametrize("sx1,sx2,sx3", GREEN_GRIDS)
@pytest.mark.parametrize("gam", [0.0, 8.3e-4])
def test_green_function_matches_oracle(oracle32, sx1, sx2, sx3, gam):
    lib = _lib.load()
    rng = np.random.default_rng(11)
    dx = (0.5, 0.4, 0.25)
    c = np.zeros((3, sx3, sx2, sx1 + 2), np.float32)
    c[:, : sx3 // 2, :, :sx1] = rng.standard_normal((3, sx3 // 2, sx2, sx1))
    t = np.zeros((3, sx2, sx1 + 2), np.float32)
    t[:, :, :sx1] = 0.1 * rng.standard_normal((3, sx2, sx1))
    cr, tr = c.copy(), t.copy()
    oracle32.green(cr, tr, sx1, sx2, sx3, dx, 1.0, 1.0, gam)
    dc = [dev(c[k]) for k in range(3)]
    dt = [dev(t[k]) for k in range(3)]
    _lib.check(lib.relax_op_green(*[ptr(x) for x in dc], *[ptr(x) for x in dt], sx1, sx2, sx3, *dx,
                                  1.0, 1.0, gam, None))
    torch.cuda.synchronize()
    got = np.stack([x.cpu().numpy() for x in dc])
    assert rel_l2(got[..., :sx1], cr[..., :sx1]) < 1e-5


def test_green_function_is_linear_bitwise():
    """G(2 f) == 2 G(f) exactly (scaling by two commutes with every rounding)."""
    lib = _lib.load()
    sx1, sx2, sx3 = 64, 64, 32
    rng = np.random.default_rng(12)
    c = np.zeros((3, sx3, sx2, sx1 + 2), np.float32)
    c[:, : sx3 // 2, :, :sx1] = rng.standard_normal((3, sx3 // 2, sx2, sx1))
    t = np.zeros((3, sx2, sx1 + 2), np.float32)
    outs = []
    for s in (1.0, 2.0):
        dc = [dev(s * c[k]) for k in range(3)]
        dt = [dev(t[k]) for k in range(3)]
        _lib.check(lib.relax_op_green(*[ptr(x) for x in dc], *[ptr(x) for x in dt], sx1, sx2, sx3,
                                      1.0, 1.0, 1.0, 1.0, 1.0, 8.3e-4, None))
        torch.cuda.synchronize()
        outs.append(np.stack([x.cpu().numpy() for x in dc]))
    assert np.array_equal(outs[1], 2.0 * outs[0])


def test_tensoramplitude_matches_oracle(oracle32):
    lib = _lib.load()
    rng = np.random.default_rng(13)
    t = tensors_random(rng, (16, 32, 64))
    ref = oracle32.tensoramplitude(t, (0.5, 0.5, 0.5))
    amp = C.c_double()
    dt_ = dev(t.view(np.float32))
    _lib.check(lib.relax_op_tensoramplitude(ptr(dt_), 64, 32, 16, 0.5, 0.5, 0.5, C.byref(amp), None))
    assert abs(amp.value - ref) <= 1e-6 * ref


def test_unsupported_grid_is_rejected():
    lib = _lib.load()
    d = dev(np.zeros((20, 10, 18), np.float32))
    rc = lib.relax_op_fft3(ptr(d), 16, 10, 20, 1.0, 1.0, 1.0, -1, None)   # sx2 = 10 = 2 x 5
    assert rc == 4
    u = dev(np.zeros((4, 8, 18), np.float32))
    sig = dev(np.zeros((4, 8, 16, 6), np.float32))
    rc = lib.relax_op_stressupdate(ptr(u), ptr(u), ptr(u), 1.0, 1.0, 1.0, 1.0, 1.0, 16, 8, 4, ptr(sig), None)
    assert rc == 4                                                         # sx3/2 = 4 < 5


@pytest.mark.parametrize("power", [1.0, 3.0])
@pytest.mark.parametrize("inplace", [False, True])
def test_transient_eigenstress_matches_oracle(oracle32, power, inplace):
    """transienteigenstress, separate and aliased epsilonik / epsilonikdot"""
    lib = _lib.load()
    sx1, sx2, sx3 = 64, 32, 32
    sx3h = sx3 // 2
    rng = np.random.default_rng(21)
    sig = tensors_random(rng, (sx3h, sx2, sx1), 0.3)
    eps = tensors_random(rng, (sx3h, sx2, sx1), 0.05)
    mom = tensors_random(rng, (sx3h, sx2, sx1), 0.1)
    epsdot = tensors_random(rng, (sx3h, sx2, sx1), 1.0)
    dg0 = (0.2 * rng.standard_normal((sx3h, sx2, sx1))).astype(np.float32)
    st = (relax_layer * sx3h)()
    for k in range(sx3h):
        st[k] = relax_layer(z=0, gammadot0=(0.0 if k < 3 else 10 ** rng.uniform(-1, 1)),
                            stressexponent=power, cohesion=0.0, friction=0, Gk=0.25 + 0.05 * k)
    mref = mom.copy()
    eref = eps.copy()
    dref = eref if inplace else epsdot.copy()
    rc, tref = oracle32.transienteigenstress(1.0, st, sig, eref, sx1, sx2, sx3h, mref, dref, maxwell=1e7,
                                             dgammadot0=dg0)
    assert rc == 0
    dm = dev(mom.view(np.float32))
    de = dev(eps.view(np.float32))
    dd = de if inplace else dev(epsdot.view(np.float32))
    ddg = dev(dg0)
    tm = C.c_double(1e7)
    _lib.check(lib.relax_op_transienteigenstress(
        1.0, C.cast(st, C.c_void_p), ptr(dev(sig.view(np.float32))), ptr(de), sx1, sx2, sx3h, ptr(dm),
        ptr(dd), C.byref(tm), ptr(ddg), None))
    torch.cuda.synchronize()
    gm = dm.cpu().numpy().view(TENSOR_DTYPE).reshape(mom.shape)
    gd = dd.cpu().numpy().view(TENSOR_DTYPE).reshape(mom.shape)
    assert rel_l2(tensor_array(gm), tensor_array(mref)) < 1e-5
    assert rel_l2(tensor_array(gd), tensor_array(dref)) < 1e-5
    assert abs(tm.value - tref) <= 1e-5 * tref


@pytest.mark.parametrize("beta", [0.0, 0.2])
def test_weak_zones_match_oracle(oracle32, beta):
    """builddgammadot0: a rotated brick, a sphere and two cylinders"""
    from relax_b200.config import relax_weakzone
    lib = _lib.load()
    sx1, sx2, sx3h = 64, 48, 24
    dx = (1.0, 1.0, 0.5)
    zones = (relax_weakzone * 4)()
    zones[0] = relax_weakzone(dgammadot0=2.0, x=-5.0, y=3.0, z=4.0, width=6.0, length=10.0, thickness=3.0,
                              strike=0.4, dip=1.1)
    zones[1] = relax_weakzone(dgammadot0=1.5, x=10.0, y=-8.0, z=6.0, width=-4.0, length=-4.0, thickness=-4.0,
                              strike=0.0, dip=0.0)
    zones[2] = relax_weakzone(dgammadot0=-0.5, x=0.0, y=12.0, z=3.0, width=5.0, length=-3.0, thickness=-3.0,
                              strike=1.0, dip=0.3)
    zones[3] = relax_weakzone(dgammadot0=0.7, x=-15.0, y=-15.0, z=8.0, width=-3.5, length=7.0,
                              thickness=-3.5, strike=-0.6, dip=0.8)
    ref = oracle32.builddgammadot0(zones, sx1, sx2, sx3h, dx, beta)
    out = torch.zeros((sx3h, sx2, sx1), dtype=torch.float32, device="cuda")
    _lib.check(lib.relax_op_dgammadot0(C.cast(zones, C.c_void_p), 4, sx1, sx2, sx3h, *dx, beta, ptr(out), None))
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.abs(ref).max() > 0.5
    # the taper is a step for beta = 0: a rotated coordinate landing on a zone's edge may
    # round to either side; away from the edges the fields agree to rounding
    bad = np.abs(got - ref) > 1e-5 * np.abs(ref).max()
    assert bad.mean() <= (2e-3 if beta == 0.0 else 0.0), bad.mean()
