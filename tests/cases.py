"""Small seeded decks for the parity tests (shapes of the benchmark
workloads, sizes the CPU oracle finishes in seconds)."""
import math

import numpy as np

from relax_b200.config import Event, Fault, Plane, Simulation


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def tensor_array(t):
    """structured TENSOR array -> (..., 6) float64"""
    return np.stack([t[n].astype(np.float64) for n in t.dtype.names], axis=-1)


def linear_small(sx=64, sz=32, dx=1.0, steps=5):
    """Linear Maxwell (n=1) below 6 km, vertical strike-slip fault, Dt = 0.5."""
    return Simulation(
        sx1=sx, sx2=sx, sx3=sz, dx1=dx, dx2=dx, dx3=dx, beta=0.2, nyquist=2.0, lambda_=1.0, mu=1.0,
        gam=0.0, interval=0.5 * steps, odt=-1, tscale=5.0, linear=[(6.0, 1.0)],
        events=[Event(0.0, [Fault(1.0, -10.0, 0.0, 0.0, 20.0, 6.0, 0.0, 90.0, 0.0)])],
        name="linear-small")


def powerlaw_small(sx=64, sz=32, dx=1.0, gam=8.3e-4, afterslip=True):
    """Power-law n=3 with depth-dependent prefactor, 20-degree thrust, one
    afterslip plane down-dip, gravity."""
    depth = dx * sz / 2
    nl = []
    z = 8.0
    while z < depth + 1e-9:
        nl.append((z, 10.0 ** (z / 8.0 - 1.0), 3.0, 0.0))
        z += dx
    top = 1.0
    bottom = top + 16.0 * math.sin(math.radians(20.0))
    planes, fc = [], []
    if afterslip:
        planes = [Plane(x=-10.0, y=16.0 * math.cos(math.radians(20.0)), z=bottom, length=20.0,
                        width=8.0, strike=0.0, dip=20.0, rake=90.0)]
        fc = [(0.0, 1.0, 0.1, 0.0, 0.0)]
    return Simulation(
        sx1=sx, sx2=sx, sx3=sz, dx1=dx, dx2=dx, dx3=dx, beta=0.2, nyquist=2.0, lambda_=1.0,
        mu=1.0, gam=gam, interval=1.0e6, odt=-1, tscale=1.0, nonlinear=nl, faultcreep=fc,
        planes=planes,
        events=[Event(0.0, [Fault(2.0, -16.0, 0.0, top, 32.0, 16.0, 0.0, 20.0, 90.0)])],
        name="powerlaw-small")


def two_events(sx=64, sz=32, dx=1.0):
    """Linear Maxwell with a second coseismic event at t = 1.0 (the step
    before it is shortened to land on the event time)."""
    s = linear_small(sx, sz, dx, steps=8)
    s.tscale = 3.0   # Dt = 0.3 -> steps land on 0.3, 0.6, 0.9, then 1.0
    s.events.append(Event(1.0, [Fault(0.5, -5.0, 8.0, 0.0, 10.0, 5.0, 30.0, 60.0, 45.0)]))
    s.name = "two-events"
    return s


def transient_small(linear=True, nonlinear=False, viscous=False, sx=64, sz=32):
    """Transient (Burgers) rheology below 6 km: linear (gammadot0 1, Gk 0.5)
    and/or nonlinear (gammadot0 2, n 3, Gk 1) transient layers, optionally a
    linear Maxwell layer as well; the vertical strike-slip fault of
    linear_small."""
    s = linear_small(sx, sz, steps=4)
    s.name = "transient-small"
    s.interval = 1.0e6       # the nonlinear transient's first steps are long
    if not viscous:
        s.linear = []
    if linear:
        s.ltransient = [(6.0, 1.0, 0.5)]
    if nonlinear:
        s.nltransient = [(6.0, 2.0, 3.0, 1.0)]
    return s


def sources_small(sx=64, sz=32, interseismic=False):
    """Linear Maxwell below 6 km with a coseismic tensile crack and a
    dilatation point source (their images lie in the lower half of the box),
    optionally interseismic shear and tensile loading."""
    from relax_b200.config import Point, Tensile
    s = linear_small(sx, sz, steps=4)
    s.name = "sources-small"
    s.events[0].tensile = [Tensile(0.5, 6.0, -4.0, 2.0, 12.0, 6.0, 20.0, 60.0)]
    s.events[0].points = [Point(0.8, -8.0, 6.0, 5.0)]
    if interseismic:
        s.inter = Event(0.0, [Fault(0.1, -15.0, 10.0, 8.0, 10.0, 4.0, 0.0, 30.0, 90.0)],
                        tensile=[Tensile(0.05, 10.0, 10.0, 6.0, 1.0, 5.0, 0.0, 90.0)])
    return s


def oracle_monitor_plane(lib, field, sx, dx, op, beta=0.0):
    """The oracle's monitorstressfield / monitorfield on field (6 or 1
    components of sx3h x sx2 x sx1 floats); returns an array of
    (px3 + 1, px2 + 1, 5 + nc) doubles: x1, x2, x3, yr, zr and the values."""
    import ctypes as C
    f = np.ascontiguousarray(field, np.float32)
    nc = 1 if f.ndim == 3 else f.shape[0]
    px2, px3 = C.c_int(), C.c_int()
    args = [nc, sx[0], sx[1], sx[2], dx[0], dx[1], dx[2], op.x, op.y, op.z, op.width, op.length, op.strike, op.dip,
            beta, C.byref(px2), C.byref(px3)]
    lib.orc_monitor_plane(f.ctypes.data, *args, None)
    out = np.zeros((px3.value + 1, px2.value + 1, 5 + nc))
    lib.orc_monitor_plane(f.ctypes.data, *args, out.ctypes.data)
    return out


def loads_small(periodic=True, second_event=True, sx=64, sz=32):
    """Linear Maxwell below 6 km with surface loads (src/elastic3d.f90:2517-2590):
    a step load t3 H(t) with the coseismic fault, optionally a periodic load
    t3 sin(2 pi t / T + phase) whose rate enters every step (the predictor's
    rate with the reference's Dt/2e8, src/relax.f90:685, the corrector's
    with Dt, :806), and a second event at t = 1.0 carrying its own loads."""
    from relax_b200.config import Load
    s = linear_small(sx, sz, steps=8)
    s.name = "loads-small"
    s.tscale = 3.0           # Dt = 0.3: steps land on 0.3, 0.6, 0.9, then 1.0
    s.events[0].loads = [Load(4.0, -3.0, 12.0, 8.0, 0.3)]
    if periodic:
        s.events[0].loads.append(Load(-6.0, 5.0, 10.0, 10.0, 0.2, period=2.0, phase=0.3, beta=0.3))
    if second_event:
        s.events.append(Event(1.0, [Fault(0.5, -5.0, 8.0, 0.0, 10.0, 5.0, 30.0, 60.0, 45.0)],
                              loads=[Load(2.0, 2.0, 8.0, 6.0, -0.25, period=1.5, phase=-0.4)]))
    return s


def eigenstrain_small(sx=64, sz=32, tetra=True):
    """Linear Maxwell below 6 km with coseismic eigenstrain sources
    (--with-eigenstrain): a dipping cuboid with a full strain tensor, a
    vertical one (the method of images, src/elastic3d.f90:1810-1826) and,
    with --with-curvilinear, a tetrahedron of 4 listed vertices."""
    from relax_b200.config import Cuboid, Tetrahedron
    s = linear_small(sx, sz, steps=4)
    s.name = "eigenstrain-small"
    ev = s.events[0]
    ev.faults = []
    ev.cuboids = [Cuboid((1e-2, 4e-3, -3e-3, -5e-3, 2e-3, 6e-3), -6.0, 4.0, 3.0, 12.0, 6.0, 4.0, 30.0, 60.0),
                  Cuboid((0.0, 8e-3, 0.0, 0.0, 0.0, 0.0), 6.0, -6.0, 0.0, 10.0, 5.0, 3.0, 0.0, 90.0)]
    if tetra:
        ev.vertices = [(8.0, 8.0, 2.0), (14.0, 8.0, 3.0), (9.0, 15.0, 2.5), (10.0, 10.0, 9.0)]
        ev.tetrahedra = [Tetrahedron((5e-3, 0.0, 2e-3, -4e-3, 0.0, 1e-3), (1, 2, 3, 4))]
    return s
