"""The reference-layer shim (cu*_ symbols) driven as src/curelax.f90 drives
the reference CUDA layer: the coseismic sequence of src/curelax.f90:300-340
(sources, tau upload, Green's function, u = v, sig = -tau + C:E(u)) read back
through cuexportspatial_ / cuexportpoints_ and compared with the context API,
and the weak-zone and transient wrappers against the oracle."""
import ctypes as C

import numpy as np
import pytest

from relax_b200 import _lib
from relax_b200.api import Relax
from relax_b200.config import (TENSOR_DTYPE, relax_layer, relax_source, relax_tensor, relax_weakzone)

from cases import linear_small, rel_l2, tensor_array

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

P, I, D, F = C.c_void_p, C.c_int, C.c_double, C.c_float


def _shim():
    lib = _lib.load()
    sigs = {
        "cuinflags_": [C.POINTER(I)] * 5 + [I] * 4 + [C.POINTER(I)],
        "cuinit_": [I, I, I, D, D, D, C.POINTER(I)],
        "cudeinit_": [],
        "cusource_": [D] * 11 + [I, I, I, D, D, D] + [P] * 6,
        "copytau_": [P, I, I, I, I],
        "calfftnelasic_": [P] * 6 + [I, I, I, D, D, D, D, D, D, P, P, P, C.POINTER(I)],
        "cufieldrep_": [I, I, I],
        "cutensorfieldadd_": [I, I, I, I, F, F],
        "custressupdatewrapper_": [I, D, D, D, D, D, I, I, I, P, P, P, P],
        "cutensoramp_": [I, I, I, I, C.POINTER(D)],
        "cuexportspatial_": [P, P, P, I],
        "cuexportpoints_": [C.POINTER(D)] * 3 + [C.POINTER(relax_tensor), I, I, I],
        "cuviscouseigen_": [P, P, D, I, I, I, D, D, D, I, C.POINTER(D), I],
        "cubuildgammadot_": [I, I, I, D, D, D, I, P, I],
        "cutransienteigenwrapper_": [I, P, D, I, I, I, D, D, D, I, C.POINTER(D), I],
        "cutensormemset_": [I],
    }
    for name, args in sigs.items():
        f = getattr(lib, name)
        f.restype = None
        f.argtypes = args
    return lib


def _init(lib, sx1, sx2, sx3, dx, transient=0):
    z = [I(0) for _ in range(4)]
    rc = I(-1)
    lib.cuinflags_(C.byref(I(transient)), *[C.byref(v) for v in z], 1, 0, transient, 0, C.byref(rc))
    assert rc.value == 0
    lib.cuinit_(sx1, sx2, sx3, *dx, C.byref(rc))
    assert rc.value == 0


def test_coseismic_sequence_matches_context_api():
    sim = linear_small(sx=64, sz=32)
    sx1, sx2, sx3, sx3h = sim.sx1, sim.sx2, sim.sx3, sim.sx3h
    dx = (sim.dx1, sim.dx2, sim.dx3)
    with Relax(sim) as r:
        r.coseismic()
        u_ref, tau_ref, sig_ref = r.field("u"), r.field("tau"), r.field("sig")
        ev = r.cfg.events[0]
        srcs = [ev.s[k] for k in range(ev.ns)]
    lib = _shim()
    _init(lib, sx1, sx2, sx3, dx)
    try:
        for s in srcs:   # the call of src/elastic3d.f90:2085-2089 (L = width, W = length)
            lib.cusource_(sim.mu, s.slip, s.x, s.y, s.z, s.width, s.length, s.strike, s.dip, s.rake, s.beta,
                          sx1, sx2, sx3, *dx, None, None, None, None, None, None)
        tau = np.ascontiguousarray(tau_ref)
        lib.copytau_(tau.ctypes.data_as(P), sx1, sx2, sx3h, 1)
        rc = I(-1)
        lib.calfftnelasic_(None, None, None, None, None, None, sx1, sx2, sx3, *dx, sim.lambda_, sim.mu,
                           sim.gam, None, None, None, C.byref(rc))
        assert rc.value == 0
        lib.cufieldrep_(sx1 + 2, sx2, sx3h)
        lib.cutensorfieldadd_(2, sx1, sx2, sx3h, 0.0, -1.0)
        lib.custressupdatewrapper_(1, sim.lambda_, sim.mu, *dx, sx1, sx2, sx3h, None, None, None, None)
        u = np.zeros_like(u_ref)
        for i3 in range(sx3h):
            planes = [np.zeros((sx2, sx1 + 2), np.float32) for _ in range(3)]
            lib.cuexportspatial_(*[p.ctypes.data_as(P) for p in planes], i3)
            for k in range(3):
                u[k, i3] = planes[k]
        assert rel_l2(u[..., :sx1], u_ref[..., :sx1]) < 1e-6
        rng = np.random.default_rng(3)
        for _ in range(20):
            i1, i2, i3 = int(rng.integers(sx1)), int(rng.integers(sx2)), int(rng.integers(sx3h))
            u1, u2, u3 = D(), D(), D()
            t = relax_tensor()
            lib.cuexportpoints_(C.byref(u1), C.byref(u2), C.byref(u3), C.byref(t), i1, i2, i3)
            # the point read-back is the plane read-back at that point
            assert (u1.value, u2.value, u3.value) == tuple(float(u[k, i3, i2, i1]) for k in range(3))
            ref = sig_ref[i3, i2, i1]
            got = np.array([getattr(t, n) for n in TENSOR_DTYPE.names])
            want = np.array([ref[n] for n in TENSOR_DTYPE.names], np.float64)
            assert np.allclose(got, want, rtol=1e-4, atol=1e-6 * np.abs(tensor_array(sig_ref)).max())
    finally:
        lib.cudeinit_()


def test_weak_zones_and_transient_wrappers(oracle32):
    sx1, sx2, sx3 = 64, 32, 32
    sx3h = sx3 // 2
    dx = (1.0, 1.0, 1.0)
    lib = _shim()
    _init(lib, sx1, sx2, sx3, dx, transient=1)
    try:
        rng = np.random.default_rng(5)
        sig = np.zeros((sx3h, sx2, sx1), TENSOR_DTYPE)
        for n in TENSOR_DTYPE.names:
            sig[n] = 0.3 * rng.standard_normal(sig.shape)
        # sig enters the shim as tau with sig = -tau (E_TENSOR_SIG_TAU, c1 = 0, c2 = -1)
        tau = np.zeros_like(sig)
        for n in TENSOR_DTYPE.names:
            tau[n] = -sig[n]
        lib.copytau_(tau.ctypes.data_as(P), sx1, sx2, sx3h, 1)
        lib.cutensorfieldadd_(2, sx1, sx2, sx3h, 0.0, -1.0)
        zones = (relax_weakzone * 1)()
        zones[0] = relax_weakzone(dgammadot0=2.0, x=0.0, y=0.0, z=8.0, width=10.0, length=12.0,
                                  thickness=6.0, strike=0.3, dip=1.0)
        lib.cubuildgammadot_(sx1, sx2, sx3h, *dx, 1, C.cast(zones, P), 1)
        st = (relax_layer * sx3h)()
        for k in range(sx3h):
            st[k] = relax_layer(z=0, gammadot0=(0.0 if k < 4 else 0.5), stressexponent=1.0, cohesion=0.0,
                                friction=0.0, Gk=0.3)
        # viscous eigenstress with the linear weak-zone field
        lib.cutensormemset_(2)
        tm = D(1e7)
        lib.cuviscouseigen_(C.cast(st, P), None, 1.0, sx1, sx2, sx3h, *dx, 1, C.byref(tm), 1)
        amp = D()
        lib.cutensoramp_(1, sx1, sx2, sx3h, C.byref(amp))
        dg0 = oracle32.builddgammadot0(zones, sx1, sx2, sx3h, dx, 0.0)
        mref = np.zeros_like(sig)
        _, tref = oracle32.viscouseigenstress(1.0, st, None, sig, sx1, sx2, sx3h, mref, maxwell=1e7,
                                              dgammadot0=dg0)
        aref = oracle32.tensoramplitude(mref, (1.0, 1.0, 1.0))
        assert abs(amp.value - aref) <= 1e-5 * aref
        assert abs(tm.value - tref) <= 1e-5 * tref
        # transient eigenstress on epsilonik = 0 (E_TENSOR_IK), then in place on epsilonikdot
        lib.cutensormemset_(2)
        tm = D(1e7)
        lib.cutransienteigenwrapper_(4, C.cast(st, P), 1.0, sx1, sx2, sx3h, *dx, 1, C.byref(tm), 0)
        lib.cutransienteigenwrapper_(5, C.cast(st, P), 1.0, sx1, sx2, sx3h, *dx, 0, None, 0)
        lib.cutensoramp_(1, sx1, sx2, sx3h, C.byref(amp))
        mref = np.zeros_like(sig)
        eps = np.zeros_like(sig)
        epsdot = np.zeros_like(sig)
        _, tref = oracle32.transienteigenstress(1.0, st, sig, eps, sx1, sx2, sx3h, mref, epsdot, maxwell=1e7)
        oracle32.transienteigenstress(1.0, st, sig, epsdot, sx1, sx2, sx3h, mref, epsdot)
        aref = oracle32.tensoramplitude(mref, (1.0, 1.0, 1.0))
        assert abs(amp.value - aref) <= 1e-5 * aref
        assert abs(tm.value - tref) <= 1e-5 * tref
    finally:
        lib.cudeinit_()
