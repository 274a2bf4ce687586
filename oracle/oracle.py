"""ctypes bindings of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``liboracle32.so`` (FP32-storage restatement of the reference CPU path)
or ``liboracle64.so`` (all-FP64) built by ``oracle/Makefile``.  Only the tests,
``__graft_entry__.smoke`` and the ``cpu_baseline`` leg of ``bench.py`` use this
module, and only as the checker / the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import List, Optional, Sequence

import numpy as np

from relax_b200.config import (TENSOR_DTYPE, relax_config, relax_layer, relax_slippatch,
                               relax_step_log, Simulation)

HERE = os.path.dirname(os.path.abspath(__file__))

TENSOR64_DTYPE = np.dtype([(n, np.float64) for n in ("s11", "s12", "s13", "s22", "s23", "s33")])

_LIBS = {}


def build():
    """Compiles both oracle variants with the system gcc (OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load(precision: int = 32) -> C.CDLL:
    if precision in _LIBS:
        return _LIBS[precision]
    path = os.path.join(HERE, f"liboracle{precision}.so")
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    P, I, D, S = C.c_void_p, C.c_int, C.c_double, C.c_size_t
    sig = {
        "orc_viscoelastic_structure": (I, [P, I, D, I, P]),
        "orc_stressupdate": (I, [P, P, P, D, D, D, D, D, I, I, I, P]),
        "orc_equivalentbodyforce": (I, [P, D, D, D, I, I, I, P, P, P, P, P, P]),
        "orc_viscouseigenstress": (I, [D, P, P, P, I, I, I, P, P, P, P]),
        "orc_transienteigenstress": (I, [D, P, P, P, I, I, I, P, P, P, P]),
        "orc_builddgammadot0": (None, [I, I, I, D, D, D, D, I, P, P]),
        "orc_frictioneigenstress": (I, [D, D, D, D, D, D, D, D, D, P, D, P, I, I, I, D, D, D, P, P]),
        "orc_fft3": (None, [P, I, I, I, D, D, D, I]),
        "orc_fft2": (None, [P, I, I, D, D, I]),
        "orc_fft_c": (None, [P, I, I]),
        "orc_greenfunctioncowling": (I, [P, P, P, P, P, P, I, I, I, D, D, D, D, D, D]),
        "orc_tensoramplitude": (D, [P, S, D, D, D]),
        "orc_elasticresponse": (None, [D, D, P, P, P, I, I, I, D, D, D]),
        "orc_surfacetractioncowling": (None, [D, D, D, P, P, P, I, I, I, D, D, D, P, P, P]),
        "orc_cerrutimodified": (None, [P, P, P, D, D, D, P, P, P, I, I, I, D, D, D]),
        "orc_source": (None, [D, D, D, D, D, D, D, D, D, D, D, I, I, I, D, D, D, P, P, P, P, P, P]),
        "orc_momentdensityshear": (None, [D, D, D, D, D, D, D, D, D, D, D, I, I, I, D, D, D, P]),
        "orc_okada": (None, [D] * 15 + [C.POINTER(D)]),
        "orc_okada_dc3d": (None, [D] * 15 + [C.POINTER(D)]),
        "orc_cuboidsource": (None, [D, D, P] + [D] * 9 + [I, I, I, D, D, D, P, P, P]),
        "orc_momentdensitycuboid": (None, [D, D, P] + [D] * 9 + [I, I, I, D, D, D, P]),
        "orc_tetrahedronsource": (None, [D, D, P, P, P, P, P, I, I, I, D, D, D, P, P, P]),
        "orc_momentdensitytetrahedron": (None, [D, D, P, P, P, P, P, I, I, I, D, D, D, P]),
        "orc_monitor_plane": (None, [P, I, I, I, I, D, D, D, D, D, D, D, D, D, D, D, C.POINTER(I), C.POINTER(I),
                                     P]),
        "orc_state_create": (P, [P]),
        "orc_state_free": (None, [P]),
        "orc_coseismic": (I, [P, P]),
        "orc_step": (I, [P, P, P]),
        "orc_get_field": (I, [P, I, P]),
        "orc_set_field": (I, [P, I, P]),
        "orc_get_patches": (I, [P, I, P]),
        "orc_time": (D, [P]),
        "orc_real_size": (I, []),
        "orc_num_threads": (I, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _LIBS[precision] = lib
    return lib


def ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    """One precision variant of the CPU restatement."""

    def __init__(self, precision: int = 32):
        self.precision = precision
        self.lib = load(precision)
        self.real = np.float32 if precision == 32 else np.float64
        self.tensor = TENSOR_DTYPE if precision == 32 else TENSOR64_DTYPE

    # -- structures ----------------------------------------------------
    def structure_fn(self, layers: Sequence[relax_layer], dx3: float, nz: int):
        arr_in = (relax_layer * len(layers))(*layers)
        out = (relax_layer * nz)()
        rc = self.lib.orc_viscoelastic_structure(C.cast(arr_in, C.c_void_p), len(layers), dx3, nz,
                                                 C.cast(out, C.c_void_p))
        if rc:
            raise ValueError(f"invalid structure ({rc})")
        return out

    def threads(self) -> int:
        return self.lib.orc_num_threads()

    # -- operators on numpy arrays (reference layout) --------------------
    def fft3(self, data: np.ndarray, sx1, sx2, sx3, dx1, dx2, dx3, direction):
        assert data.dtype == self.real and data.flags.c_contiguous
        self.lib.orc_fft3(ptr(data), sx1, sx2, sx3, dx1, dx2, dx3, direction)

    def fft2(self, data, sx1, sx2, dx1, dx2, direction):
        self.lib.orc_fft2(ptr(data), sx1, sx2, dx1, dx2, direction)

    def fft_c(self, x: np.ndarray, sign: int) -> np.ndarray:
        a = np.ascontiguousarray(x, dtype=np.complex128).copy()
        self.lib.orc_fft_c(ptr(a), a.size, sign)
        return a

    def stressupdate(self, u, lam, mu, dx, sx1, sx2, sx3h, sig):
        rc = self.lib.orc_stressupdate(ptr(u[0]), ptr(u[1]), ptr(u[2]), lam, mu, *dx, sx1, sx2,
                                       sx3h, ptr(sig))
        assert rc == 0

    def bodyforce(self, sig, dx, sx1, sx2, sx3h, c, t):
        rc = self.lib.orc_equivalentbodyforce(ptr(sig), *dx, sx1, sx2, sx3h, ptr(c[0]), ptr(c[1]),
                                              ptr(c[2]), ptr(t[0]), ptr(t[1]), ptr(t[2]))
        assert rc == 0

    def viscouseigenstress(self, mu, structure, prestress, sig, sx1, sx2, sx3h, moment,
                           maxwell: Optional[float] = None, gamma=None, dgammadot0=None):
        tm = C.c_double(maxwell) if maxwell is not None else None
        rc = self.lib.orc_viscouseigenstress(
            mu, C.cast(structure, C.c_void_p), None if prestress is None else C.cast(prestress, C.c_void_p),
            ptr(sig), sx1, sx2, sx3h, ptr(moment), None if tm is None else C.byref(tm), ptr(gamma),
            ptr(dgammadot0))
        return rc, (tm.value if tm is not None else None)

    def transienteigenstress(self, mu, structure, sig, eps, sx1, sx2, sx3h, moment, epsdot,
                             maxwell: Optional[float] = None, dgammadot0=None):
        """eps and epsdot may be the same array"""
        tm = C.c_double(maxwell) if maxwell is not None else None
        rc = self.lib.orc_transienteigenstress(
            mu, C.cast(structure, C.c_void_p), ptr(sig), ptr(eps), sx1, sx2, sx3h, ptr(moment), ptr(epsdot),
            None if tm is None else C.byref(tm), ptr(dgammadot0))
        return rc, (tm.value if tm is not None else None)

    def builddgammadot0(self, zones, sx1, sx2, sx3h, dx, beta):
        out = np.zeros((sx3h, sx2, sx1), self.real)
        arr = C.cast(zones, C.c_void_p) if len(zones) else None
        self.lib.orc_builddgammadot0(sx1, sx2, sx3h, *dx, beta, len(zones), arr, ptr(out))
        return out

    def frictioneigenstress(self, plane, beta, sig, mu, structure, sx1, sx2, sx3h, dx, moment,
                            maxwell: Optional[float] = None):
        tm = C.c_double(maxwell) if maxwell is not None else None
        rc = self.lib.orc_frictioneigenstress(
            plane.x, plane.y, plane.z, plane.width, plane.length, plane.strike, plane.dip,
            plane.rake, beta, ptr(sig), mu, C.cast(structure, C.c_void_p), sx1, sx2, sx3h, *dx,
            ptr(moment), None if tm is None else C.byref(tm))
        return rc, (tm.value if tm is not None else None)

    # eigenstrain sources: e a relax_tensor, geometry in the internal convention
    def cuboidsource(self, lam, mu, e, geo, beta, sx, dx, f):
        """geo = (x, y, z, L, W, T, strike, dip) as dislocations passes them"""
        self.lib.orc_cuboidsource(lam, mu, C.byref(e), *geo, beta, *sx, *dx, ptr(f[0]), ptr(f[1]), ptr(f[2]))

    def momentdensitycuboid(self, mu, lam, e, geo, beta, sx1, sx2, sx3h, dx, sig):
        self.lib.orc_momentdensitycuboid(mu, lam, C.byref(e), *geo, beta, sx1, sx2, sx3h, *dx, ptr(sig))

    def tetrahedronsource(self, lam, mu, e, verts, sx, dx, f):
        v = [np.ascontiguousarray(x, np.float64) for x in verts]
        self.lib.orc_tetrahedronsource(lam, mu, C.byref(e), *[ptr(x) for x in v], *sx, *dx, ptr(f[0]), ptr(f[1]),
                                       ptr(f[2]))

    def momentdensitytetrahedron(self, mu, lam, e, verts, sx1, sx2, sx3h, dx, sig):
        v = [np.ascontiguousarray(x, np.float64) for x in verts]
        self.lib.orc_momentdensitytetrahedron(mu, lam, C.byref(e), *[ptr(x) for x in v], sx1, sx2, sx3h, *dx,
                                              ptr(sig))

    def green(self, c, t, sx1, sx2, sx3, dx, lam, mu, gam):
        rc = self.lib.orc_greenfunctioncowling(ptr(c[0]), ptr(c[1]), ptr(c[2]), ptr(t[0]),
                                               ptr(t[1]), ptr(t[2]), sx1, sx2, sx3, *dx, lam, mu,
                                               gam)
        assert rc == 0

    def tensoramplitude(self, t, dx):
        return self.lib.orc_tensoramplitude(ptr(t), t.size, *dx)

    # -- the time loop ------------------------------------------------------
    def run(self, sim: Simulation, nsteps: int, dt_schedule: Optional[Sequence[float]] = None,
            fields: bool = True, config=None):
        """Coseismic solve + nsteps RK2 steps.  Returns (logs, fields dict).
        config: a relax_config to run instead of sim.to_c (e.g. one read
        from an input file; sim then only gives the array shapes)."""
        cfg, keep = (config, None) if config is not None else sim.to_c(self.structure_fn)
        st = self.lib.orc_state_create(C.byref(cfg))
        if not st:
            raise MemoryError("oracle state allocation failed")
        try:
            logs: List[tuple] = []
            lg = relax_step_log()
            rc = self.lib.orc_coseismic(st, C.byref(lg))
            if rc:
                raise RuntimeError(f"orc_coseismic failed ({rc})")
            logs.append(lg.as_tuple())
            tmt = [(lg.tm_tl, lg.tm_tnl)]
            for k in range(nsteps):
                dtp = C.byref(C.c_double(dt_schedule[k])) if dt_schedule is not None else None
                rc = self.lib.orc_step(st, dtp, C.byref(lg))
                if rc:
                    raise RuntimeError(f"orc_step failed ({rc}) at step {k + 1}")
                if lg.i == 0:
                    break
                logs.append(lg.as_tuple())
                tmt.append((lg.tm_tl, lg.tm_tnl))
            out = {"tm_transient": tmt}
            if fields:
                out.update(self.get_fields(st, sim))
                out["patches"] = [self.get_patches(st, k, cfg.planes[k].px2 * cfg.planes[k].px3)
                                  for k in range(cfg.np)]
            return logs, out
        finally:
            self.lib.orc_state_free(st)

    def get_fields(self, st, sim: Simulation):
        out = {}
        u = np.zeros(sim.vec_shape(), self.real)
        self.lib.orc_get_field(st, 1, ptr(u))
        out["u"] = u
        for name, which in (("sig", 2), ("tau", 3), ("moment", 4)):
            a = np.zeros(sim.tensor_shape(), self.tensor)
            self.lib.orc_get_field(st, which, ptr(a))
            out[name] = a
        g = np.zeros(sim.vec_shape()[1:], self.real)
        self.lib.orc_get_field(st, 5, ptr(g))
        out["gamma"] = g
        return out

    def get_patches(self, st, k, n):
        arr = (relax_slippatch * n)()
        self.lib.orc_get_patches(st, k, C.cast(arr, C.c_void_p))
        return arr
