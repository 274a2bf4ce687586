"""Python mirror of the context API: one RELAX instance on one GPU.

    sim = relax_b200.config.powerlaw_thrust()
    with Relax(sim) as r:
        log0 = r.coseismic()
        for _ in range(10):
            log = r.step()
        u = r.field("u")

Every call goes through ``librelax_b200.so``; host arrays use RELAX's layout
(padded vectors (3, sx3/2, sx2, sx1+2), TENSOR structs (sx3/2, sx2, sx1)).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from .config import (TENSOR_DTYPE, Simulation, relax_config, relax_input_info, relax_obsplane, relax_segment,
                     relax_slippatch, relax_step_log, relax_tensor, relax_weakzone)

FIELDS = {"u": 1, "sig": 2, "tau": 3, "moment": 4, "gamma": 5, "eps": 6, "v": 7, "ur": 8}
NCOMP = {"u": 3, "gamma": 1, "sig": 6, "tau": 6, "moment": 6, "eps": 6, "v": 3, "ur": 3}


def _path(p) -> bytes:
    return os.fsencode(p)


def format_log(log: relax_step_log, interval: float, transient: bool = False) -> str:
    """The step log line of RELAX (formats 1100-1103, src/relax.f90:1102-1105)."""
    buf = C.create_string_buffer(256)
    _lib.check(_lib.load().relax_format_log(C.byref(log), interval, 1 if transient else 0, buf, 256))
    return buf.value.decode()


def log_header(transient: bool = False) -> str:
    """The column header printed before the log (formats 0990/0991)."""
    return _lib.load().relax_log_header(1 if transient else 0).decode()


def es_format(v: float, w: int, d: int, e: int) -> str:
    """Fortran ESw.dEe of one value."""
    buf = C.create_string_buffer(128)
    _lib.check(_lib.load().relax_es_format(v, w, d, e, buf, 128))
    return buf.value.decode()


SEGMENT_EXPORTS = {"gmt": 1, "traction": 2, "vtp": 3}


def write_segments(kind: str, segments: Sequence[relax_segment], filename, sig=None, sig0=None):
    """exportgmt_rfaults_stress ("gmt"), exportgmt_rfaults_traction
    ("traction") or exportvtk_rfaults_stress ("vtp") of the segments, from
    the stress at their centres (None: zero) less sig0 when given."""
    n = len(segments)
    sop = (relax_segment * n)(*segments)
    s = (relax_tensor * n)(*sig) if sig is not None else None
    s0 = (relax_tensor * n)(*sig0) if sig0 is not None else None
    _lib.check(_lib.load().relax_write_segments(SEGMENT_EXPORTS[kind], n, sop, s, s0, _path(filename)))


def write_coulomb(segments: Sequence[relax_segment], sig, time: float, wdir, isnew: bool):
    """exportcoulombstress: a line per segment in wdir/cfaults-sigma-KKKK.txt."""
    n = len(segments)
    sop = (relax_segment * n)(*segments)
    s = (relax_tensor * n)(*sig)
    _lib.check(_lib.load().relax_write_coulomb(n, sop, s, time, _path(wdir), 1 if isnew else 0))


def write_grd(z: np.ndarray, x0: float, y0: float, dx: float, dy: float, title: str, filename):
    """A GMT netCDF grid of z (ny, nx), x_i = x0 + i dx, y_j = y0 + j dy."""
    z = np.ascontiguousarray(z, np.float32)
    ny, nx = z.shape
    _lib.check(_lib.load().relax_write_grd(z.ctypes.data_as(C.POINTER(C.c_float)), nx, ny, x0, y0, dx, dy,
                                           title.encode(), _path(filename)))


def write_grd3(planes, dx1: float, dx2: float, origx: float, origy: float, wdir, index: int, convention: int):
    """exportgrd of three (sx2, sx1) planes (x1 fastest) into wdir."""
    ps = [np.ascontiguousarray(p, np.float32) for p in planes]
    sx2, sx1 = ps[0].shape
    fp = C.POINTER(C.c_float)
    _lib.check(_lib.load().relax_write_grd3(*[p.ctypes.data_as(fp) for p in ps], sx1, sx2, dx1, dx2, origx, origy,
                                            _path(wdir), index, convention))


def write_vtk(comps, dx: Sequence[float], strides: Sequence[int], filename, title: str = "", name: str = "field"):
    """VTK legacy binary file of 3 vector or 6 tensor components, each (sx3, sx2, sx1)."""
    cs = [np.ascontiguousarray(c, np.float32) for c in comps]
    sx3, sx2, sx1 = cs[0].shape
    fp = C.POINTER(C.c_float)
    arr = (fp * len(cs))(*[c.ctypes.data_as(fp) for c in cs])
    _lib.check(_lib.load().relax_write_vtk(arr, len(cs), sx1, sx2, sx3, *dx, *strides, _path(filename),
                                           title.encode(), name.encode()))


def shifted_index(x, sx, dx):
    """shiftedindex (src/elastic3d.f90:4063-4101): 0-based (i1, i2, i3) of a
    point; sx[2] is the number of x3-planes held."""
    i = [C.c_int() for _ in range(3)]
    _lib.check(_lib.load().relax_shifted_index(*x, *sx, *dx, *[C.byref(v) for v in i]))
    return tuple(v.value for v in i)


class Input:
    """A RELAX input file read by the library (src/input.f90:43-1767).

        inp = Input.parse(open("relax.inp").read(), transient=True)
        with Relax.from_input(inp) as r:
            ...
    """

    def __init__(self, handle):
        self.lib = _lib.load()
        self.h = handle

    @classmethod
    def parse(cls, text: str, transient: bool = False, eigenstrain: bool = False, curvilinear: bool = False,
              echo: bool = False) -> "Input":
        lib = _lib.load()
        flags = (1 if transient else 0) | (2 if eigenstrain else 0) | (4 if curvilinear else 0) | \
            (8 if echo else 0)
        h = C.c_void_p()
        _lib.check(lib.relax_input_parse(text.encode(), flags, C.byref(h)))
        return cls(h)

    def close(self):
        if getattr(self, "h", None):
            self.lib.relax_input_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def config(self) -> relax_config:
        """The relax_config (owned by the input)."""
        return self.lib.relax_input_config(self.h).contents

    @property
    def info(self) -> relax_input_info:
        i = relax_input_info()
        _lib.check(self.lib.relax_input_get_info(self.h, C.byref(i)))
        return i

    def weakzones(self, mechanism: int):
        z = C.POINTER(relax_weakzone)()
        n = C.c_int()
        _lib.check(self.lib.relax_input_weakzones(self.h, mechanism, C.byref(z), C.byref(n)))
        return [z[k] for k in range(n.value)]

    def export_geometry(self, vtk: bool = True):
        """The geometry files that the reference's input reader writes into
        the output directory (grid, interfaces, weak zones, planes, faults)."""
        _lib.check(self.lib.relax_input_export_geometry(self.h, 1 if vtk else 0))

    def obsplanes(self):
        """Observation planes (internal convention, radians)."""
        z = C.POINTER(relax_obsplane)()
        n = C.c_int()
        _lib.check(self.lib.relax_input_obsplanes(self.h, C.byref(z), C.byref(n)))
        return [z[k] for k in range(n.value)]

    def segments(self):
        """Stress observation segments (internal convention, radians)."""
        z = C.POINTER(relax_segment)()
        n = C.c_int()
        _lib.check(self.lib.relax_input_segments(self.h, C.byref(z), C.byref(n)))
        return [z[k] for k in range(n.value)]

    def build_weakzones(self, device: int = 0):
        _lib.check(self.lib.relax_input_build_weakzones(self.h, device))

    def simulation(self) -> Simulation:
        """The grid and scalar parameters as a Simulation (array shapes)."""
        c = self.config
        return Simulation(sx1=c.sx1, sx2=c.sx2, sx3=c.sx3, dx1=c.dx1, dx2=c.dx2, dx3=c.dx3, beta=c.beta,
                          nyquist=c.nyquist, lambda_=c.lambda_, mu=c.mu, gam=c.gam, interval=c.interval,
                          odt=c.odt, tscale=c.tscale)


def release_cached_memory(device: int = 0):
    """Returns the device memory that the library keeps pooled after
    destroyed contexts, batches and operators (relax_release_cached_memory)."""
    _lib.check(_lib.load().relax_release_cached_memory(device))


class Relax:
    def __init__(self, sim: Simulation, device: int = 0, config: Optional[relax_config] = None, keep=None):
        self.lib = _lib.load()
        self.sim = sim
        if config is None:
            self.cfg, self._keep = sim.to_c(_lib.structure_fn)
        else:
            self.cfg, self._keep = config, keep
        h = C.c_void_p()
        _lib.check(self.lib.relax_create(C.byref(self.cfg), device, C.byref(h)))
        self.h = h

    @classmethod
    def from_input(cls, inp: Input, device: int = 0) -> "Relax":
        """A context for an input file (weak-zone fields built on `device`)."""
        if any(inp.info.nwz):
            inp.build_weakzones(device)
        return cls(inp.simulation(), device, config=inp.config, keep=inp)

    def close(self):
        if getattr(self, "h", None):
            self.lib.relax_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- time loop ---------------------------------------------------------
    def coseismic(self, e: int = 0) -> tuple:
        lg = relax_step_log()
        _lib.check(self.lib.relax_coseismic(self.h, e, C.byref(lg)))
        self.last_log = lg
        return lg.as_tuple()

    def step(self, dt: Optional[float] = None) -> tuple:
        lg = relax_step_log()
        dtp = C.byref(C.c_double(dt)) if dt is not None else None
        _lib.check(self.lib.relax_step(self.h, dtp, C.byref(lg)))
        self.last_log = lg        # the full record (transient Maxwell times included)
        return lg.as_tuple()

    def run(self, nsteps: int, dt_schedule: Optional[Sequence[float]] = None) -> List[tuple]:
        logs = (relax_step_log * (nsteps + 1))()
        n = C.c_int(0)
        sched = None
        if dt_schedule is not None:
            arr = (C.c_double * nsteps)(*dt_schedule[:nsteps])
            sched = C.cast(arr, C.POINTER(C.c_double))
        _lib.check(self.lib.relax_run(self.h, nsteps, sched, logs, C.byref(n)))
        return [logs[k].as_tuple() for k in range(n.value + 1)]

    def set_precision(self, mode: str):
        """"fp32" (default) or "mixed": the x3 transform's length-64 DFTs on
        the tensor cores (split BF16, FP32 accumulation), 128-deep boxes."""
        _lib.check(self.lib.relax_set_precision(self.h, {"fp32": 0, "mixed": 1}[mode]))

    def synchronize(self):
        _lib.check(self.lib.relax_synchronize(self.h))

    # -- profiling -----------------------------------------------------------
    def profile(self, enable: bool):
        _lib.check(self.lib.relax_profile(self.h, 1 if enable else 0))

    def profile_read(self):
        """{kernel name: (total ms, launches)} of the recorded stages."""
        out = {}
        for s in range(self.lib.relax_profile_stages()):
            ms = C.c_double()
            n = C.c_int()
            name = C.c_char_p()
            _lib.check(self.lib.relax_profile_read(self.h, s, C.byref(ms), C.byref(n), C.byref(name)))
            if n.value:
                out[name.value.decode()] = (ms.value, n.value)
        return out

    def launch_count(self) -> int:
        n = C.c_longlong()
        _lib.check(self.lib.relax_launch_count(self.h, C.byref(n)))
        return n.value

    # -- fields --------------------------------------------------------------
    def field_shape(self, name: str):
        """(shape, dtype) of a field in the reference layout."""
        s = self.sim
        if name == "u":
            return s.vec_shape(), np.dtype(np.float32)
        if name == "gamma":
            return s.vec_shape()[1:], np.dtype(np.float32)
        return s.tensor_shape(), TENSOR_DTYPE

    def field(self, name: str) -> np.ndarray:
        shape, dt = self.field_shape(name)
        return self.field_into(name, np.zeros(shape, dt))

    def field_into(self, name: str, out) -> np.ndarray:
        """Reads a field into a caller's buffer (a numpy array, or any object
        with the array interface and the field's size, page-locked or not)."""
        a = np.asarray(out)
        shape, dt = self.field_shape(name)
        if a.nbytes != int(np.prod(shape)) * dt.itemsize or not a.flags.c_contiguous:
            raise ValueError(f"field {name}: need a contiguous buffer of {int(np.prod(shape)) * dt.itemsize} bytes")
        _lib.check(self.lib.relax_get_field(self.h, FIELDS[name], a.ctypes.data_as(C.c_void_p), a.nbytes))
        return out

    def set_field(self, name: str, a: np.ndarray):
        a = np.ascontiguousarray(a)
        _lib.check(self.lib.relax_set_field(self.h, FIELDS[name], a.ctypes.data_as(C.c_void_p),
                                            a.nbytes))

    def save(self, path):
        """Checkpoint of the state between steps (relax_checkpoint_save)."""
        _lib.check(self.lib.relax_checkpoint_save(self.h, _path(path)))

    def load(self, path):
        """Restores a checkpoint written by a context of the same configuration."""
        _lib.check(self.lib.relax_checkpoint_load(self.h, _path(path)))

    def track_relaxation(self, vel_planes: int = 0, ur_planes: int = 0, inter_i3: int = -1):
        """Keep the corrector's velocity and the postseismic displacement (see the header)."""
        _lib.check(self.lib.relax_track_relaxation(self.h, vel_planes, ur_planes, inter_i3))

    def plane(self, name: str, i3: int) -> np.ndarray:
        """Plane i3 of a field as (ncomp, sx2, sx1), unpadded."""
        s = self.sim
        a = np.zeros((NCOMP[name], s.sx2, s.sx1), np.float32)
        _lib.check(self.lib.relax_get_plane(self.h, FIELDS[name], i3, a.ctypes.data_as(C.c_void_p), a.nbytes))
        return a

    def points(self, index) -> tuple:
        """Displacement (n, 3) and stress (n,) TENSOR_DTYPE at 0-based (i1, i2, i3) points."""
        idx = np.ascontiguousarray(index, np.int32).reshape(-1, 3)
        n = idx.shape[0]
        u = np.zeros((n, 3), np.float64)
        sig = (relax_tensor * max(n, 1))()
        _lib.check(self.lib.relax_get_points(self.h, n, idx.ctypes.data_as(C.POINTER(C.c_int)),
                                             u.ctypes.data_as(C.POINTER(C.c_double)), sig))
        out = np.zeros(n, TENSOR_DTYPE)
        for k in range(n):
            out[k] = tuple(getattr(sig[k], f) for f in TENSOR_DTYPE.names)
        return u, out

    def export_grd(self, name: str, wdir, index: int, oz: float = 0.0, origx: float = 0.0, origy: float = 0.0):
        """exportgrd (u) / exportstressgrd (sig, eps) of the current state into wdir."""
        _lib.check(self.lib.relax_export_grd(self.h, FIELDS[name], oz, origx, origy, _path(wdir), index))

    def export_vtk(self, name: str, filename, sx3: int, strides=(4, 4, 8), title: str = "", vname: str = "field"):
        _lib.check(self.lib.relax_export_vtk(self.h, FIELDS[name], sx3, *strides, _path(filename), title.encode(),
                                             vname.encode()))

    def export_creep(self, wdir, index: int, txt: bool = True, grd: bool = True, vtk: bool = False):
        """exportcreep_asc / exportcreep_grd / exportcreep_vtk: the afterslip
        planes' patches as NNN.sKKKKK.creep.dat, NNN.sKKKKK.{slip,vel}*.grd and
        creep-KKKKKs-NNN.vtk files in wdir."""
        formats = (1 if txt else 0) | (2 if grd else 0) | (4 if vtk else 0)
        _lib.check(self.lib.relax_export_creep(self.h, _path(wdir), index, formats))

    def monitor_plane(self, op, name: str = "sig", beta: float = 0.0):
        """monitorstressfield / monitorfield: the stress (patch.sig) or gamma
        (patch.slip) sampled on an observation plane; an array of
        (px3+1, px2+1) patches."""
        px2, px3 = C.c_int(), C.c_int()
        _lib.check(self.lib.relax_monitor_plane(self.h, FIELDS[name], C.byref(op), beta, None, 0, C.byref(px2),
                                                C.byref(px3)))
        n = (px2.value + 1) * (px3.value + 1)
        arr = (relax_slippatch * n)()
        _lib.check(self.lib.relax_monitor_plane(self.h, FIELDS[name], C.byref(op), beta, arr, n, C.byref(px2),
                                                C.byref(px3)))
        return np.ctypeslib.as_array(arr).copy().reshape(px3.value + 1, px2.value + 1)

    def segment_stress(self, segments: Sequence[relax_segment]):
        """The stress at the segment centres (nearest grid node)."""
        n = len(segments)
        sop = (relax_segment * n)(*segments)
        sig = (relax_tensor * n)()
        _lib.check(self.lib.relax_segment_stress(self.h, n, sop, sig))
        return sig

    def export_plane_stress(self, planes: Sequence[relax_obsplane], wdir, index: int, origx: float = 0.0,
                            origy: float = 0.0, name: str = "sig"):
        """exportplanestress (name "sig") / exporteigenstrain (name "gamma")."""
        n = len(planes)
        op = (relax_obsplane * n)(*planes)
        _lib.check(self.lib.relax_export_plane_stress(self.h, FIELDS[name], n, op, origx, origy, _path(wdir), index))

    def export_points(self, xyz, names: Sequence[str], time: float, wdir, isnew: bool, rot: float = 0.0):
        """exportpoints: one .ned line per observation point (x1, x2, x3 in the computational frame)."""
        x = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        nm = (C.c_char_p * len(names))(*[n.encode() for n in names])
        _lib.check(self.lib.relax_export_points(self.h, x.shape[0], x.ctypes.data_as(C.POINTER(C.c_double)), nm,
                                                time, rot, _path(wdir), 1 if isnew else 0))

    def patches(self, k: int):
        p = self.cfg.planes[k]
        n = p.px2 * p.px3
        arr = (relax_slippatch * n)()
        _lib.check(self.lib.relax_get_patches(self.h, k, arr, n))
        return arr

    def time(self):
        t = C.c_double()
        i = C.c_int()
        e = C.c_int()
        _lib.check(self.lib.relax_get_time(self.h, C.byref(t), C.byref(i), C.byref(e)))
        return t.value, i.value, e.value


class _Member(Relax):
    """A batch member: field, patch and time access through the member's
    context, which the batch owns."""

    def __init__(self, lib, sim: Simulation, cfg, handle):
        self.lib = lib
        self.sim = sim
        self.cfg = cfg
        self.h = handle

    def close(self):
        self.h = None


_MODES = {0: "measuring", 1: "batched", 2: "in turn"}


class Batch:
    """Members sharing grid and elastic constants, stepped together.

        with Batch([sim_a, sim_b, ...]) as b:
            b.coseismic()
            for _ in range(100):
                logs = b.step()          # one log tuple per member
            u0 = b.member(0).field("u")
    """

    def __init__(self, sims: Sequence[Simulation], device: int = 0):
        self.lib = _lib.load()
        self.sims = list(sims)
        cfgs, self._keep = [], []
        for s in self.sims:
            cfg, keep = s.to_c(_lib.structure_fn)
            cfgs.append(cfg)
            self._keep.append(keep)
        self._cfgs = (type(cfgs[0]) * len(cfgs))(*cfgs)
        h = C.c_void_p()
        _lib.check(self.lib.relax_batch_create(self._cfgs, len(cfgs), device, C.byref(h)))
        self.h = h
        self.n = len(cfgs)

    def close(self):
        if getattr(self, "h", None):
            self.lib.relax_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def coseismic(self) -> List[tuple]:
        logs = (relax_step_log * self.n)()
        _lib.check(self.lib.relax_batch_coseismic(self.h, logs))
        return [logs[k].as_tuple() for k in range(self.n)]

    def step(self) -> List[tuple]:
        logs = (relax_step_log * self.n)()
        _lib.check(self.lib.relax_batch_step(self.h, logs))
        return [logs[k].as_tuple() for k in range(self.n)]

    def member(self, k: int) -> Relax:
        h = C.c_void_p()
        _lib.check(self.lib.relax_batch_member(self.h, k, C.byref(h)))
        return _Member(self.lib, self.sims[k], self._cfgs[k], h)

    def launch_count(self) -> int:
        n = C.c_longlong()
        _lib.check(self.lib.relax_batch_launch_count(self.h, C.byref(n)))
        return n.value

    def stream(self) -> int:
        s = C.c_void_p()
        _lib.check(self.lib.relax_batch_get_stream(self.h, C.byref(s)))
        return s.value

    def tuning(self) -> dict:
        """The batch's choice between one launch per stage for all members
        and the members stepped in turn, from its first six steps:
        {"mode": "measuring" | "batched" | "in turn", "batched_ms", "in_turn_ms"}
        (step times, -1 until measured)."""
        m, tb, tt = C.c_int(), C.c_double(), C.c_double()
        _lib.check(self.lib.relax_batch_tuning(self.h, C.byref(m), C.byref(tb), C.byref(tt)))
        return {"mode": _MODES[m.value], "batched_ms": tb.value, "in_turn_ms": tt.value}


class Ensemble(Batch):
    """Members with uneven grids, grouped by shape into batches stepped one
    after the other (each tuned on its own); one host synchronisation per
    ensemble step.

        with Ensemble(ensemble_uneven(seed=4)) as e:
            e.coseismic()
            for _ in range(100):
                logs = e.step()
    """

    def __init__(self, sims: Sequence[Simulation], device: int = 0):
        self.lib = _lib.load()
        self.sims = list(sims)
        cfgs, self._keep = [], []
        for s in self.sims:
            cfg, keep = s.to_c(_lib.structure_fn)
            cfgs.append(cfg)
            self._keep.append(keep)
        self._cfgs = (type(cfgs[0]) * len(cfgs))(*cfgs)
        h = C.c_void_p()
        _lib.check(self.lib.relax_ensemble_create(self._cfgs, len(cfgs), device, C.byref(h)))
        self.h = h
        self.n = len(cfgs)

    def close(self):
        if getattr(self, "h", None):
            self.lib.relax_ensemble_destroy(self.h)
            self.h = None

    def groups(self) -> int:
        g = C.c_int()
        _lib.check(self.lib.relax_ensemble_size(self.h, None, C.byref(g)))
        return g.value

    def coseismic(self) -> List[tuple]:
        logs = (relax_step_log * self.n)()
        _lib.check(self.lib.relax_ensemble_coseismic(self.h, logs))
        return [logs[k].as_tuple() for k in range(self.n)]

    def step(self) -> List[tuple]:
        logs = (relax_step_log * self.n)()
        _lib.check(self.lib.relax_ensemble_step(self.h, logs))
        return [logs[k].as_tuple() for k in range(self.n)]

    def member(self, k: int) -> Relax:
        h = C.c_void_p()
        _lib.check(self.lib.relax_ensemble_member(self.h, k, C.byref(h)))
        return _Member(self.lib, self.sims[k], self._cfgs[k], h)

    def launch_count(self) -> int:
        n = C.c_longlong()
        _lib.check(self.lib.relax_ensemble_launch_count(self.h, C.byref(n)))
        return n.value

    def stream(self) -> int:
        raise NotImplementedError("an ensemble runs one stream per shape group")

    def tuning(self) -> List[dict]:
        """Per shape group: {"grid": (sx1, sx2, sx3), "members", "mode",
        "batched_ms", "in_turn_ms"} as Batch.tuning reports them."""
        out = []
        for q in range(self.groups()):
            sx = (C.c_int * 3)()
            nm, m, tb, tt = C.c_int(), C.c_int(), C.c_double(), C.c_double()
            _lib.check(self.lib.relax_ensemble_tuning(self.h, q, sx, C.byref(nm), C.byref(m), C.byref(tb),
                                                      C.byref(tt)))
            out.append({"grid": (sx[0], sx[1], sx[2]), "members": nm.value, "mode": _MODES[m.value],
                        "batched_ms": tb.value, "in_turn_ms": tt.value})
        return out
