"""Host-side description of one RELAX simulation and its C-ABI mirror.

The ctypes structures below mirror ``include/relax_b200.h`` field for field
(and therefore RELAX's own types, src/types.f90:26-266).  ``Simulation``
holds an input deck in RELAX's *input-file* convention (geologic fault
geometry in degrees, interface lists) and ``Simulation.to_c`` turns it into
a ``relax_config`` in the internal convention the time loop reads:

* faults and afterslip planes go through ``wang_convention``
  (src/input.f90:1780-1800) and the afterslip rake flip
  (src/input.f90:1079-1083);
* interface lists are expanded to one entry per physical layer by a
  caller-supplied ``structure_fn`` (the library's
  ``relax_viscoelastic_structure`` or the oracle's restatement).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

DEG2RAD = 0.01745329251994329547437168059786927


class relax_tensor(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("s11", "s12", "s13", "s22", "s23", "s33")]


class relax_tensor_layer(C.Structure):
    _fields_ = [("z", C.c_float), ("dum", C.c_float), ("t", relax_tensor)]


class relax_layer(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("z", "gammadot0", "stressexponent", "cohesion", "friction", "Gk")]


class relax_source(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("slip", "x", "y", "z", "width", "length", "strike", "dip", "rake",
                 "period", "phase", "beta", "opening")]


class relax_plane(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("x", "y", "z", "width", "length", "strike", "dip", "rake")] + \
               [("px2", C.c_int), ("px3", C.c_int)]


class relax_slippatch(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("x1", "x2", "x3", "lx", "lz", "slip", "ss", "ds", "v", "vss", "vds",
                 "taus")] + [("sig", relax_tensor)]


class relax_obsplane(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("x", "y", "z", "length", "width", "strike", "dip")]


class relax_segment(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("x", "y", "z", "length", "width", "strike", "dip", "friction")]


class relax_weakzone(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("dgammadot0", "x", "y", "z", "width", "length", "thickness", "strike", "dip")] + \
               [("e", relax_tensor)]


class relax_tetrahedron(C.Structure):
    _fields_ = [("e", relax_tensor), ("i1", C.c_int), ("i2", C.c_int), ("i3", C.c_int), ("i4", C.c_int)]


class relax_event(C.Structure):
    _fields_ = [("time", C.c_double), ("ns", C.c_int), ("nt", C.c_int), ("nm", C.c_int),
                ("nl", C.c_int), ("s", C.POINTER(relax_source)),
                ("ts", C.POINTER(relax_source)), ("m", C.POINTER(relax_source)),
                ("l", C.POINTER(relax_source)),
                ("nc", C.c_int), ("ntet", C.c_int), ("nvert", C.c_int),
                ("c", C.POINTER(relax_weakzone)), ("tet", C.POINTER(relax_tetrahedron)),
                ("vert", C.POINTER(C.c_double))]


class relax_config(C.Structure):
    _fields_ = [("sx1", C.c_int), ("sx2", C.c_int), ("sx3", C.c_int),
                ("dx1", C.c_double), ("dx2", C.c_double), ("dx3", C.c_double),
                ("beta", C.c_double), ("nyquist", C.c_double),
                ("lambda_", C.c_double), ("mu", C.c_double), ("gam", C.c_double),
                ("interval", C.c_double), ("odt", C.c_double), ("tscale", C.c_double),
                ("skip", C.c_int),
                ("stressstruc", C.POINTER(relax_tensor_layer)),
                ("linearstruc", C.POINTER(relax_layer)),
                ("nonlinearstruc", C.POINTER(relax_layer)),
                ("faultcreepstruc", C.POINTER(relax_layer)),
                ("lineardgammadot0", C.POINTER(C.c_float)),
                ("nonlineardgammadot0", C.POINTER(C.c_float)),
                ("np", C.c_int), ("planes", C.POINTER(relax_plane)),
                ("ne", C.c_int), ("events", C.POINTER(relax_event)),
                ("inter", relax_event),
                ("ltransientstruc", C.POINTER(relax_layer)),
                ("nltransientstruc", C.POINTER(relax_layer)),
                ("ltransientdgammadot0", C.POINTER(C.c_float)),
                ("nltransientdgammadot0", C.POINTER(C.c_float)),
                ("x0", C.c_double), ("y0", C.c_double), ("rot", C.c_double)]


class relax_input_info(C.Structure):
    _fields_ = [("wdir", C.c_char_p)] + [(n, C.c_double) for n in ("x0", "y0", "rot", "oz", "ozs")] + \
               [("npts", C.c_int), ("pts", C.POINTER(C.c_double)), ("ptsname", C.POINTER(C.c_char_p)),
                ("nop", C.c_int), ("nsop", C.c_int), ("nwz", C.c_int * 4),
                ("minlength", C.c_double), ("minwidth", C.c_double)]


class relax_step_log(C.Structure):
    _fields_ = [("i", C.c_int), ("event", C.c_int)] + \
               [(n, C.c_double) for n in ("dt", "tm_ve", "tm_pl", "tm_as", "t", "power", "cei",
                                          "tm_tl", "tm_tnl")] + \
               [("output", C.c_int)]

    def as_tuple(self):
        return (self.i, self.dt, self.tm_ve, self.tm_pl, self.tm_as, self.t, self.power,
                self.cei)


TENSOR_DTYPE = np.dtype([(n, np.float32) for n in ("s11", "s12", "s13", "s22", "s23", "s33")])


def wang_convention(slip, x, y, z, length, width, strike, dip, rake, x0=0.0, y0=0.0, rot=0.0):
    """wangconvention + rotation, src/input.f90:1780-1815.

    Geologic description (upper end of the top edge, strike/dip/rake in
    degrees) -> internal convention (centre, radians, slip sign flipped).
    """
    slip = -slip
    strike = -90.0 - strike
    dip = 90.0 - dip
    strike = strike * DEG2RAD
    dip = dip * DEG2RAD
    rake = rake * DEG2RAD
    x = x - x0 - length / 2.0 * math.sin(strike) + width / 2.0 * math.sin(dip) * math.cos(strike)
    y = y - y0 - length / 2.0 * math.cos(strike) - width / 2.0 * math.sin(dip) * math.sin(strike)
    z = z + width / 2.0 * math.cos(dip)
    alpha = rot * DEG2RAD
    xx, yy = x, y
    x = +xx * math.cos(alpha) + yy * math.sin(alpha)
    y = -xx * math.sin(alpha) + yy * math.cos(alpha)
    strike = strike + rot * DEG2RAD
    return slip, x, y, z, strike, dip, rake


def antialiasing_filter(slip, length, width, dx1, dx2, dx3, nyquist):
    """antialiasingfilter, src/input.f90:1836-1856: segments smaller than
    nyquist * min(dx) are widened with their slip scaled down."""
    dx = min(dx1, dx2, dx3) * nyquist
    if length < dx:
        slip = slip * length / dx
        length = dx
    if width < dx:
        slip = slip * width / dx
        width = dx
    return slip, length, width


def fix(number: float) -> int:
    """fix, src/elastic3d.f90:69-80 (round half down)."""
    f, c = math.floor(number), math.ceil(number)
    return int(c if (number - f) > 0.5 else f)


@dataclass
class Fault:
    """One shear dislocation in input-file convention (src/input.f90:1299-1303)."""
    slip: float
    x: float
    y: float
    z: float
    length: float
    width: float
    strike: float
    dip: float
    rake: float
    beta: Optional[float] = None


@dataclass
class Plane:
    """One afterslip plane in input-file convention (src/input.f90:1059-1062)."""
    x: float
    y: float
    z: float
    length: float
    width: float
    strike: float
    dip: float
    rake: float


@dataclass
class Tensile:
    """An opening crack in input-file convention (src/input.f90:1389-1440)."""
    opening: float
    x: float
    y: float
    z: float
    length: float
    width: float
    strike: float
    dip: float


@dataclass
class Point:
    """A dilatation (Mogi) point source (src/input.f90:1460-1484)."""
    amplitude: float
    x: float
    y: float
    z: float


@dataclass
class Load:
    """A surface load (src/input.f90:1676-1735): traction t3 (force per
    surface, positive down) on a tapered L x W rectangle centred at (x, y);
    period T > 0 gives t3 sin(2 pi t / T + phase), T = 0 a step t3 H(t)
    (src/elastic3d.f90:2517-2590).  beta None takes the deck's smoothing."""
    x: float
    y: float
    length: float
    width: float
    t3: float
    period: float = 0.0
    phase: float = 0.0
    beta: Optional[float] = None


@dataclass
class Cuboid:
    """A cuboid of eigenstrain (--with-eigenstrain, src/input.f90:1496-1560):
    strain (e11, e12, e13, e22, e23, e33) in the source's (strike, normal,
    dip) frame, centre geometry as a fault's, thickness across it."""
    e: Tuple[float, float, float, float, float, float]
    x: float
    y: float
    z: float
    length: float
    width: float
    thickness: float
    strike: float
    dip: float


@dataclass
class Tetrahedron:
    """A tetrahedron of eigenstrain (--with-curvilinear, src/input.f90:
    1588-1660): strain in the grid frame and four 1-based vertex numbers."""
    e: Tuple[float, float, float, float, float, float]
    vertices: Tuple[int, int, int, int]


@dataclass
class Event:
    time: float
    faults: List[Fault] = field(default_factory=list)
    tensile: List[Tensile] = field(default_factory=list)
    points: List[Point] = field(default_factory=list)
    loads: List[Load] = field(default_factory=list)
    cuboids: List[Cuboid] = field(default_factory=list)
    tetrahedra: List[Tetrahedron] = field(default_factory=list)
    vertices: List[Tuple[float, float, float]] = field(default_factory=list)


@dataclass
class Simulation:
    """An input deck restricted to what the relaxation loop reads."""
    sx1: int
    sx2: int
    sx3: int
    dx1: float
    dx2: float
    dx3: float
    beta: float = 0.2
    nyquist: float = 2.0
    lambda_: float = 1.0
    mu: float = 1.0
    gam: float = 0.0
    interval: float = 1.0
    odt: float = -1.0          # 2nd entry of the time line; <0 selects skip mode
    tscale: float = 1.0
    x0: float = 0.0
    y0: float = 0.0
    rot: float = 0.0
    # interface lists: (depth, gammadot0, power, cohesion) for viscous layers,
    # (depth, V0, (a-b)sigma, friction, cohesion) for fault creep
    linear: List[Tuple[float, ...]] = field(default_factory=list)
    nonlinear: List[Tuple[float, ...]] = field(default_factory=list)
    faultcreep: List[Tuple[float, ...]] = field(default_factory=list)
    # transient (Burgers) interfaces, src/input.f90:738-900:
    # linear (depth, gammadot0, Gk), nonlinear (depth, gammadot0, power, Gk)
    ltransient: List[Tuple[float, ...]] = field(default_factory=list)
    nltransient: List[Tuple[float, ...]] = field(default_factory=list)
    planes: List[Plane] = field(default_factory=list)
    events: List[Event] = field(default_factory=list)
    # interseismic loading rates (src/input.f90:1107-1240): shear (faults)
    # and tensile segments; the time is not used
    inter: Optional[Event] = None
    name: str = "relax"

    @property
    def sx3h(self) -> int:
        return self.sx3 // 2

    @property
    def skip(self) -> int:
        # src/input.f90:308-316: "T, -n, t_s" -> skip = ceiling(n), odt < 0
        return int(math.ceil(-self.odt)) if self.odt < 0 else 0

    def has_eigenstrain(self) -> bool:
        return any(ev.cuboids or ev.tetrahedra for ev in self.events)

    @property
    def npoints(self) -> int:
        return self.sx1 * self.sx2 * self.sx3

    # -------------------------------------------------------------- #
    def layer_lists(self):
        lin = [relax_layer(z=d, gammadot0=g, stressexponent=1.0,
                           cohesion=(c[0] if c else 0.0), friction=0.0, Gk=0.0)
               for (d, g, *c) in self.linear]
        non = [relax_layer(z=d, gammadot0=g, stressexponent=n, cohesion=c, friction=0.0, Gk=0.0)
               for (d, g, n, c) in self.nonlinear]
        fc = [relax_layer(z=d, gammadot0=v0, stressexponent=ab, friction=f, cohesion=c, Gk=0.0)
              for (d, v0, ab, f, c) in self.faultcreep]
        return lin, non, fc

    def transient_lists(self):
        # the linear transient exponent is 1 (src/input.f90:760)
        lt = [relax_layer(z=d, gammadot0=g, stressexponent=1.0, cohesion=0.0, friction=0.0, Gk=gk)
              for (d, g, gk) in self.ltransient]
        nlt = [relax_layer(z=d, gammadot0=g, stressexponent=n, cohesion=0.0, friction=0.0, Gk=gk)
               for (d, g, n, gk) in self.nltransient]
        return lt, nlt

    def to_c(self, structure_fn: Callable[[Sequence[relax_layer], float, int], C.Array]):
        """Returns (relax_config, keepalive) for this deck."""
        keep = []
        nz = self.sx3h
        cfg = relax_config()
        cfg.sx1, cfg.sx2, cfg.sx3 = self.sx1, self.sx2, self.sx3
        cfg.dx1, cfg.dx2, cfg.dx3 = self.dx1, self.dx2, self.dx3
        cfg.beta, cfg.nyquist = self.beta, self.nyquist
        cfg.lambda_, cfg.mu, cfg.gam = self.lambda_, self.mu, self.gam
        cfg.interval, cfg.tscale = self.interval, self.tscale
        cfg.odt = self.odt
        cfg.skip = self.skip
        cfg.x0, cfg.y0, cfg.rot = self.x0, self.y0, self.rot
        lin, non, fc = self.layer_lists()
        lt, nlt = self.transient_lists()
        for name, lst in (("linearstruc", lin), ("nonlinearstruc", non),
                          ("faultcreepstruc", fc), ("ltransientstruc", lt), ("nltransientstruc", nlt)):
            if lst:
                arr = structure_fn(lst, self.dx3, nz)
                keep.append(arr)
                setattr(cfg, name, C.cast(arr, C.POINTER(relax_layer)))
        # afterslip planes (src/input.f90:1059-1101)
        if self.planes:
            parr = (relax_plane * len(self.planes))()
            for k, p in enumerate(self.planes):
                rake = p.rake - 180.0 if p.rake >= 0.0 else p.rake + 180.0
                _, x, y, z, strike, dip, rake = wang_convention(
                    0.0, p.x, p.y, p.z, p.length, p.width, p.strike, p.dip, rake,
                    self.x0, self.y0, self.rot)
                parr[k] = relax_plane(x=x, y=y, z=z, width=p.width, length=p.length,
                                      strike=strike, dip=dip, rake=rake,
                                      px2=fix(p.length / self.dx2), px3=fix(p.width / self.dx3))
            keep.append(parr)
            cfg.np = len(self.planes)
            cfg.planes = C.cast(parr, C.POINTER(relax_plane))
        # events
        earr = (relax_event * max(1, len(self.events)))()
        for e, ev in enumerate(self.events):
            earr[e].time = ev.time
            if ev.faults:
                sarr = (relax_source * len(ev.faults))()
                for k, f in enumerate(ev.faults):
                    slip, x, y, z, strike, dip, rake = wang_convention(
                        f.slip, f.x, f.y, f.z, f.length, f.width, f.strike, f.dip, f.rake,
                        self.x0, self.y0, self.rot)
                    sarr[k] = relax_source(slip=slip, x=x, y=y, z=z, width=f.width,
                                           length=f.length, strike=strike, dip=dip, rake=rake,
                                           period=0.0, phase=0.0,
                                           beta=self.beta if f.beta is None else f.beta,
                                           opening=0.0)
                keep.append(sarr)
                earr[e].ns = len(ev.faults)
                earr[e].s = C.cast(sarr, C.POINTER(relax_source))
            if ev.tensile:
                tarr = (relax_source * len(ev.tensile))()
                for k, t in enumerate(ev.tensile):
                    # slip = opening goes through wangconvention; the opening stays
                    slip, x, y, z, strike, dip, _ = wang_convention(
                        t.opening, t.x, t.y, t.z, t.length, t.width, t.strike, t.dip, 0.0,
                        self.x0, self.y0, self.rot)
                    tarr[k] = relax_source(slip=slip, x=x, y=y, z=z, width=t.width, length=t.length,
                                           strike=strike, dip=dip, rake=0.0, period=0.0, phase=0.0,
                                           beta=self.beta, opening=t.opening)
                keep.append(tarr)
                earr[e].nt = len(ev.tensile)
                earr[e].ts = C.cast(tarr, C.POINTER(relax_source))
            if ev.points:
                marr = (relax_source * len(ev.points))()
                for k, m in enumerate(ev.points):
                    # rotation only (src/input.f90:1481)
                    a = self.rot * DEG2RAD
                    x = m.x * math.cos(a) + m.y * math.sin(a)
                    y = -m.x * math.sin(a) + m.y * math.cos(a)
                    marr[k] = relax_source(slip=m.amplitude, x=x, y=y, z=m.z, beta=self.beta)
                keep.append(marr)
                earr[e].nm = len(ev.points)
                earr[e].m = C.cast(marr, C.POINTER(relax_source))
            if ev.loads:
                larr = (relax_source * len(ev.loads))()
                for k, ld in enumerate(ev.loads):
                    # rotation only (src/input.f90:1733)
                    a = self.rot * DEG2RAD
                    x = ld.x * math.cos(a) + ld.y * math.sin(a)
                    y = -ld.x * math.sin(a) + ld.y * math.cos(a)
                    larr[k] = relax_source(slip=ld.t3, x=x, y=y, length=ld.length, width=ld.width,
                                           period=ld.period, phase=ld.phase,
                                           beta=self.beta if ld.beta is None else ld.beta)
                keep.append(larr)
                earr[e].nl = len(ev.loads)
                earr[e].l = C.cast(larr, C.POINTER(relax_source))
            if ev.cuboids:
                carr = (relax_weakzone * len(ev.cuboids))()
                for k, q in enumerate(ev.cuboids):
                    # wangconvention on the weak-zone geometry (src/input.f90:1548-1558)
                    _, x, y, z, strike, dip, _ = wang_convention(
                        0.0, q.x, q.y, q.z, q.length, q.width, q.strike, q.dip, 0.0, self.x0, self.y0, self.rot)
                    carr[k] = relax_weakzone(dgammadot0=0.0, x=x, y=y, z=z, width=q.width, length=q.length,
                                             thickness=q.thickness, strike=strike, dip=dip, e=relax_tensor(*q.e))
                keep.append(carr)
                earr[e].nc = len(ev.cuboids)
                earr[e].c = C.cast(carr, C.POINTER(relax_weakzone))
            if ev.tetrahedra:
                tarr = (relax_tetrahedron * len(ev.tetrahedra))()
                for k, q in enumerate(ev.tetrahedra):
                    tarr[k] = relax_tetrahedron(relax_tensor(*q.e), *q.vertices)
                varr = (C.c_double * (3 * len(ev.vertices)))(*[c for v in ev.vertices for c in v])
                keep += [tarr, varr]
                earr[e].ntet = len(ev.tetrahedra)
                earr[e].tet = C.cast(tarr, C.POINTER(relax_tetrahedron))
                earr[e].nvert = len(ev.vertices)
                earr[e].vert = C.cast(varr, C.POINTER(C.c_double))
        keep.append(earr)
        cfg.ne = len(self.events)
        cfg.events = C.cast(earr, C.POINTER(relax_event))
        if self.inter is not None:
            d = (self.dx1, self.dx2, self.dx3, self.nyquist)
            if self.inter.faults:
                sarr = (relax_source * len(self.inter.faults))()
                for k, f in enumerate(self.inter.faults):
                    slip, length, width = antialiasing_filter(f.slip, f.length, f.width, *d)
                    slip, x, y, z, strike, dip, rake = wang_convention(
                        slip, f.x, f.y, f.z, length, width, f.strike, f.dip, f.rake, self.x0, self.y0, self.rot)
                    sarr[k] = relax_source(slip=slip, x=x, y=y, z=z, width=width, length=length, strike=strike,
                                           dip=dip, rake=rake, beta=self.beta if f.beta is None else f.beta)
                keep.append(sarr)
                cfg.inter.ns = len(self.inter.faults)
                cfg.inter.s = C.cast(sarr, C.POINTER(relax_source))
            if self.inter.tensile:
                tarr = (relax_source * len(self.inter.tensile))()
                for k, t in enumerate(self.inter.tensile):
                    # the filter acts on slip = 0 (src/input.f90:1205, :1233-1235): only the
                    # dimensions change; the opening rate stays
                    _, length, width = antialiasing_filter(0.0, t.length, t.width, *d)
                    slip, x, y, z, strike, dip, _ = wang_convention(
                        0.0, t.x, t.y, t.z, length, width, t.strike, t.dip, 0.0, self.x0, self.y0, self.rot)
                    tarr[k] = relax_source(slip=slip, x=x, y=y, z=z, width=width, length=length,
                                           strike=strike, dip=dip, beta=self.beta, opening=t.opening)
                keep.append(tarr)
                cfg.inter.nt = len(self.inter.tensile)
                cfg.inter.ts = C.cast(tarr, C.POINTER(relax_source))
        return cfg, keep

    def to_input(self, wdir: str = "output", oz: float = 0.0, ozs: float = 0.0,
                 points: Sequence[Tuple[str, float, float, float]] = (),
                 obsplanes: Sequence[Tuple[float, ...]] = (), segments: Sequence[Tuple[float, ...]] = ()) -> str:
        """This deck as a RELAX input file (the order of src/input.f90:43-1767,
        written with --with-transient sections when the deck has transient
        interfaces).  Numbers are written with repr, so reading them back
        gives the same doubles.  obsplanes: (x1, x2, x3, length, width,
        strike, dip) and segments: (x1, x2, x3, length, width, strike, dip,
        friction), in the input file's convention (degrees).  Decks with
        eigenstrain sources are written with the --with-eigenstrain sections
        (and --with-curvilinear ones when a tetrahedron is present): read
        them with those flags."""
        r = repr
        eigen = self.has_eigenstrain()
        curvilinear = any(ev.tetrahedra for ev in self.events)
        out = ["# grid dimension (sx1,sx2,sx3)", f"{self.sx1} {self.sx2} {self.sx3}",
               "# sampling (dx1,dx2,dx3), smoothing (beta, nyquist)",
               f"{r(self.dx1)} {r(self.dx2)} {r(self.dx3)} {r(self.beta)} {r(self.nyquist)}",
               "# origin position and rotation", f"{r(self.x0)} {r(self.y0)} {r(self.rot)}",
               "# observation depth (displacement and stress)", f"{r(oz)} {r(ozs)}",
               "# output directory", wdir,
               "# elastic parameters and gamma", f"{r(self.lambda_)} {r(self.mu)} {r(self.gam)}",
               "# integration time, time step or (negative skip, scaling)",
               f"{r(self.interval)} {r(self.odt)}" + (f" {r(self.tscale)}" if self.odt < 0 else ""),
               "# number of observation planes", str(len(obsplanes))]
        out += [f"{k + 1} " + " ".join(r(float(v)) for v in p) for k, p in enumerate(obsplanes)]
        out += ["# number of observation points", str(len(points))]
        out += [f"{k + 1} {n} {r(x)} {r(y)} {r(z)}" for k, (n, x, y, z) in enumerate(points)]
        out += ["# number of stress observation segments", str(len(segments))]
        out += [f"{k + 1} " + " ".join(r(float(v)) for v in g) for k, g in enumerate(segments)]
        out += ["# number of prestress interfaces", "0",
                "# number of linear viscous interfaces", str(len(self.linear))]
        out += [f"{k + 1} {r(d)} {r(g)} {r(c[0] if c else 0.0)}" for k, (d, g, *c) in enumerate(self.linear)]
        if self.linear:
            out += ["# number of linear weak zones", "0"]
        out += ["# number of nonlinear viscous interfaces", str(len(self.nonlinear))]
        out += [f"{k + 1} {r(d)} {r(g)} {r(n)} {r(c)}" for k, (d, g, n, c) in enumerate(self.nonlinear)]
        if self.nonlinear:
            out += ["# number of nonlinear weak zones", "0"]
        if self.ltransient or self.nltransient:
            out += ["# number of linear transient interfaces", str(len(self.ltransient))]
            out += [f"{k + 1} {r(d)} {r(g)} {r(gk)}" for k, (d, g, gk) in enumerate(self.ltransient)]
            if self.ltransient:
                out += ["# number of transient weak zones", "0"]
            out += ["# number of nonlinear transient interfaces", str(len(self.nltransient))]
            out += [f"{k + 1} {r(d)} {r(g)} {r(n)} {r(gk)}" for k, (d, g, n, gk) in enumerate(self.nltransient)]
            if self.nltransient:
                out += ["# number of transient weak zones", "0"]
        out += ["# number of fault creep interfaces", str(len(self.faultcreep))]
        out += [f"{k + 1} {r(d)} {r(v)} {r(ab)} {r(f)} {r(c)}" for k, (d, v, ab, f, c) in enumerate(self.faultcreep)]
        if self.faultcreep:
            out += ["# number of afterslip planes", str(len(self.planes))]
            out += [f"{k + 1} {r(p.x)} {r(p.y)} {r(p.z)} {r(p.length)} {r(p.width)} {r(p.strike)} {r(p.dip)} "
                    f"{r(p.rake)}" for k, p in enumerate(self.planes)]
        inter = self.inter or Event(0.0)
        out += ["# number of interseismic strike-slip segments", str(len(inter.faults))]
        out += [f"{k + 1} {r(f.slip)} {r(f.x)} {r(f.y)} {r(f.z)} {r(f.length)} {r(f.width)} {r(f.strike)} "
                f"{r(f.dip)} {r(f.rake)}" for k, f in enumerate(inter.faults)]
        out += ["# number of interseismic tensile segments", str(len(inter.tensile))]
        out += [f"{k + 1} {r(t.opening)} {r(t.x)} {r(t.y)} {r(t.z)} {r(t.length)} {r(t.width)} {r(t.strike)} "
                f"{r(t.dip)}" for k, t in enumerate(inter.tensile)]
        out += ["# number of coseismic events", str(len(self.events))]
        for e, ev in enumerate(self.events):
            if e > 0:
                out += ["# time of next event", r(ev.time)]
            out += ["# number of shear dislocations", str(len(ev.faults))]
            out += [f"{k + 1} {r(f.slip)} {r(f.x)} {r(f.y)} {r(f.z)} {r(f.length)} {r(f.width)} {r(f.strike)} "
                    f"{r(f.dip)} {r(f.rake)}" + ("" if f.beta is None else f" {r(f.beta)}")
                    for k, f in enumerate(ev.faults)]
            out += ["# number of tensile cracks", str(len(ev.tensile))]
            out += [f"{k + 1} {r(t.opening)} {r(t.x)} {r(t.y)} {r(t.z)} {r(t.length)} {r(t.width)} "
                    f"{r(t.strike)} {r(t.dip)}" for k, t in enumerate(ev.tensile)]
            out += ["# number of dilatation sources", str(len(ev.points))]
            out += [f"{k + 1} {r(m.amplitude)} {r(m.x)} {r(m.y)} {r(m.z)}" for k, m in enumerate(ev.points)]
            if eigen:
                out += ["# number of cuboid eigenstrain sources", str(len(ev.cuboids))]
                out += [f"{k + 1} " + " ".join(r(float(v)) for v in q.e) +
                        f" {r(q.x)} {r(q.y)} {r(q.z)} {r(q.length)} {r(q.width)} {r(q.thickness)} {r(q.strike)} "
                        f"{r(q.dip)}" for k, q in enumerate(ev.cuboids)]
                if curvilinear:
                    out += ["# number of tetrahedra", str(len(ev.tetrahedra))]
                    out += [f"{k + 1} " + " ".join(r(float(v)) for v in q.e) + " " +
                            " ".join(str(i) for i in q.vertices) for k, q in enumerate(ev.tetrahedra)]
                    if ev.tetrahedra:
                        out += ["# number of vertices", str(len(ev.vertices))]
                        out += [f"{k + 1} {r(v[0])} {r(v[1])} {r(v[2])}" for k, v in enumerate(ev.vertices)]
            out += ["# number of surface loads", str(len(ev.loads))]
            out += [f"{k + 1} {r(ld.x)} {r(ld.y)} {r(ld.length)} {r(ld.width)} {r(ld.t3)} {r(ld.period)} "
                    f"{r(ld.phase)}" + ("" if ld.beta is None else f" {r(ld.beta)}")
                    for k, ld in enumerate(ev.loads)]
        return "\n".join(out) + "\n"

    # field sizes in the reference layout
    def vec_shape(self, full: bool = False):
        return (3, self.sx3 if full else self.sx3h, self.sx2, self.sx1 + 2)

    def tensor_shape(self):
        return (self.sx3h, self.sx2, self.sx1)


# ---------------------------------------------------------------------- #
# synthetic workloads (seeded; shapes and distributions of the named
# benchmark configurations)
# ---------------------------------------------------------------------- #

def linear_maxwell(sx: int = 128, sz: int = 128, dx: float = 0.8, steps: int = 20) -> Simulation:
    """Plain FP32 linear Maxwell (n=1): vertical strike-slip fault L=40 W=15
    centred, slip 1, uniform gammadot0 = 1 below 30 km, Dt = 0.5 exactly
    (tm = 1/gammadot0, Dt = tm/10 * tscale with tscale = 5).  The FFT box is
    sx*sx*sz; its physical half-space holds sz/2 layers."""
    return Simulation(
        sx1=sx, sx2=sx, sx3=sz, dx1=dx, dx2=dx, dx3=dx, beta=0.2, nyquist=2.0,
        lambda_=1.0, mu=1.0, gam=0.0, interval=0.5 * steps, odt=-1, tscale=5.0,
        linear=[(30.0, 1.0)],
        events=[Event(0.0, [Fault(1.0, -20.0, 0.0, 0.0, 40.0, 15.0, 0.0, 90.0, 0.0)])],
        name=f"linear-maxwell-{sx}x{sx}x{sz}")


def powerlaw_thrust(sx: int = 256, sz: int = 128, dx: float = 0.5, steps: int = 200,
                    afterslip: bool = True) -> Simulation:
    """Power-law n=3 under a 20-degree thrust: eta(z) = 10^(1.5 - z/20) below
    20 km entered as one nonlinear interface per dx3 layer, thrust L=80 W=40
    slip 2 (normalised units), one rate-strengthening afterslip plane
    down-dip of it (50 km x 20 km, i.e. 40 patches of 5 km when binned),
    a-b = 1e-3 at a normalised effective normal stress of 100, i.e.
    (a-b)sigma = 0.1.  Adaptive dt (skip mode, tscale 1)."""
    depth = dx * sz / 2
    nl = []
    z = 20.0
    while z < depth + 1e-9:
        nl.append((z, 10.0 ** (z / 20.0 - 1.5), 3.0, 0.0))
        z += dx
    top = 1.0
    bottom = top + 40.0 * math.sin(math.radians(20.0))
    planes = []
    fc = []
    if afterslip:
        planes = [Plane(x=-25.0, y=40.0 * math.cos(math.radians(20.0)), z=bottom, length=50.0,
                        width=20.0, strike=0.0, dip=20.0, rake=90.0)]
        fc = [(0.0, 1.0, 0.1, 0.0, 0.0)]
    return Simulation(
        sx1=sx, sx2=sx, sx3=sz, dx1=dx, dx2=dx, dx3=dx, beta=0.2, nyquist=2.0,
        lambda_=1.0, mu=1.0, gam=0.0, interval=1.0e6, odt=-1, tscale=1.0,
        nonlinear=nl, faultcreep=fc, planes=planes,
        events=[Event(0.0, [Fault(2.0, -40.0, 0.0, top, 80.0, 40.0, 0.0, 20.0, 90.0)])],
        name=f"powerlaw-thrust-{sx}x{sx}x{sz}")


def random_faults(seed: int, sx: int = 512, sz: int = 256, dx: float = 0.4, nfaults: int = 3,
                  lid: float = 25.0, n: float = 3.5, gam: float = 8.3e-4, sx2: Optional[int] = None,
                  lmax: float = 100.0) -> Simulation:
    """Large instance with gravity: faults drawn from `seed` (lengths
    U[20, lmax] km, dip U[30,90], slip lognormal median 1 sigma 0.5, width
    L/2, centres inside the middle 60 % of the box), power-law n below an
    elastic lid.  sx2 (default sx) narrows the box along x2 for reduced
    parity cases."""
    rng = np.random.default_rng(seed)
    sx2 = sx if sx2 is None else sx2
    half1 = 0.3 * sx * dx
    half2 = 0.3 * sx2 * dx
    faults = []
    for _ in range(nfaults):
        L = float(rng.uniform(20, lmax))
        dip = float(rng.uniform(30, 90))
        slip = float(np.exp(rng.normal(0.0, 0.5)))
        faults.append(Fault(slip, float(rng.uniform(-half1, half1 - L)),
                            float(rng.uniform(-half2, half2)), float(rng.uniform(0, 5)), L, L / 2,
                            float(rng.uniform(0, 360)), dip, float(rng.uniform(-180, 180))))
    return Simulation(
        sx1=sx, sx2=sx2, sx3=sz, dx1=dx, dx2=dx, dx3=dx, beta=0.2, nyquist=2.0, lambda_=1.0,
        mu=1.0, gam=gam, interval=1.0e6, odt=-1, tscale=1.0,
        nonlinear=[(lid, 1.0, n, 0.0)], events=[Event(0.0, faults)],
        name=f"random-faults-{sx}x{sx2}x{sz}-seed{seed}")


ENSEMBLE_SHAPES = ((64, 64, 64), (128, 128, 64), (128, 128, 128), (192, 192, 96))


def ensemble_uneven(seed: int = 4, n: int = 64) -> List[Simulation]:
    """Batched ensemble of `n` members with uneven grids drawn from
    {64^3, 128^2 x 64, 128^3, 192^2 x 96}.  Per member: stress exponent
    U[1, 3.5], log10 of the fluidity prefactor U[-1, 1], elastic lid depth
    U[15, 40] km, one strike-slip (dip 90, rake 0) or thrust (dip 25, rake 90)
    fault with slip lognormal of median 1 (sigma 0.5), length U[10, 30] km,
    width L/2.  The grid spacing makes every box 64 km deep (128 km / sx3),
    so the lid lies inside the physical half-space.  Skip mode, Dt = tm/10."""
    rng = np.random.default_rng(seed)
    sims = []
    for k in range(n):
        sx1, sx2, sx3 = ENSEMBLE_SHAPES[int(rng.integers(len(ENSEMBLE_SHAPES)))]
        dx = 128.0 / sx3
        nexp = float(rng.uniform(1.0, 3.5))
        g0 = float(10.0 ** rng.uniform(-1.0, 1.0))
        lid = float(rng.uniform(15.0, 40.0))
        L = float(rng.uniform(10.0, 30.0))
        slip = float(np.exp(rng.normal(0.0, 0.5)))
        if rng.integers(2):
            f = Fault(slip, -L / 2, 0.0, 0.0, L, L / 2, 0.0, 90.0, 0.0)
        else:
            f = Fault(slip, -L / 2, 0.0, 1.0, L, L / 2, 0.0, 25.0, 90.0)
        sims.append(Simulation(
            sx1=sx1, sx2=sx2, sx3=sx3, dx1=dx, dx2=dx, dx3=dx, beta=0.2, nyquist=2.0, lambda_=1.0,
            mu=1.0, gam=0.0, interval=1.0e6, odt=-1, tscale=1.0,
            nonlinear=[(lid, g0, nexp, 0.0)], events=[Event(0.0, [f])],
            name=f"ensemble-{k}-{sx1}x{sx2}x{sx3}"))
    return sims


def ensemble_thrust_afterslip(seed: int = 5, n: int = 16, sx: int = 256, sz: int = 128,
                              dx: float = 0.5) -> List[Simulation]:
    """Ensemble of `n` thrust instances on one 256^2 x 128 box (dx = 0.5 km,
    gravity 8.3e-4): a 20-degree thrust 80 km x 40 km made of 5 km patches
    (16 x 8) with slip 2 (1 + N(0, 0.2)) each, two rate-strengthening
    afterslip planes (one down-dip of the rupture, one shallow in front of
    it), power law n = 3
    below 35 km with a fluidity prefactor drawn per member (10^U[-0.5, 0.5]).
    Skip mode, Dt = tm/10."""
    rng = np.random.default_rng(seed)
    sd, cd = math.sin(math.radians(20.0)), math.cos(math.radians(20.0))
    top, width, length, patch = 1.0, 40.0, 80.0, 5.0
    sims = []
    for k in range(n):
        faults = []
        for i in range(int(length / patch)):
            for j in range(int(width / patch)):
                slip = float(2.0 * (1.0 + rng.normal(0.0, 0.2)))
                faults.append(Fault(slip, -length / 2 + i * patch, j * patch * cd, top + j * patch * sd, patch,
                                    patch, 0.0, 20.0, 90.0))
        bottom = top + width * sd
        planes = [Plane(x=-25.0, y=width * cd, z=bottom, length=50.0, width=20.0, strike=0.0, dip=20.0,
                        rake=90.0),
                  Plane(x=-25.0, y=-12.0 * cd, z=top + 0.5, length=50.0, width=10.0, strike=0.0, dip=20.0,
                        rake=90.0)]
        g0 = float(10.0 ** rng.uniform(-0.5, 0.5))
        sims.append(Simulation(
            sx1=sx, sx2=sx, sx3=sz, dx1=dx, dx2=dx, dx3=dx, beta=0.2, nyquist=2.0, lambda_=1.0, mu=1.0,
            gam=8.3e-4, interval=1.0e6, odt=-1, tscale=1.0, nonlinear=[(35.0, g0, 3.0, 0.0)],
            faultcreep=[(0.0, 1.0, 0.1, 0.0, 0.0)], planes=planes, events=[Event(0.0, faults)],
            name=f"thrust-afterslip-{k}"))
    return sims


def reference_output2() -> Simulation:
    """The input echoed in examples/tutorials/output2.param:8-62 (power-law
    n=3 relaxation after a strike-slip fault, 256^3)."""
    return Simulation(
        sx1=256, sx2=256, sx3=256, dx1=0.05, dx2=0.05, dx3=0.05, beta=0.2, nyquist=2.0,
        lambda_=1.0, mu=1.0, gam=8.33e-4, interval=100.0, odt=-1, tscale=0.5,
        nonlinear=[(2.0, 5e3, 3.0, 0.0), (8.0, 5e3, 3.0, 0.0)],
        events=[Event(0.0, [Fault(1.0, -1.0, 0.0, 0.0, 2.0, 1.0, 0.0, 90.0, 0.0)])],
        name="reference-output2")


def reference_output3() -> Simulation:
    """The input echoed in examples/tutorials/output3.param:8-69 (afterslip
    on a vertical plane below a strike-slip fault, 256^3)."""
    return Simulation(
        sx1=256, sx2=256, sx3=256, dx1=0.05, dx2=0.05, dx3=0.05, beta=0.2, nyquist=1.0,
        lambda_=1.0, mu=1.0, gam=8.33e-4, interval=0.5, odt=-1, tscale=1e-2,
        faultcreep=[(1.0, 1e3, 1e3, 0.0, 0.0)],
        planes=[Plane(-2.0, 0.0, 1.0, 4.0, 2.0, 0.0, 90.0, 0.0)],
        events=[Event(0.0, [Fault(1.0, -0.5, 0.0, 0.0, 1.0, 1.0, 0.0, 90.0, 0.0)])],
        name="reference-output3")


WORKLOADS = {
    "linear-maxwell": linear_maxwell,
    "powerlaw-thrust": powerlaw_thrust,
    "random-faults": random_faults,
}
