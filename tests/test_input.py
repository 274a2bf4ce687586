"""The input file reader (subroutine init, src/input.f90:43-1767): a deck
written from a Simulation reads back into the same relax_config that
Simulation.to_c builds (wangconvention, the afterslip rake flip, the
antialiasing filter, rotations, expanded depth structures), plus the
reader's syntax (comments, list-directed records) and its errors.  Host
code only: runs on the CPU."""
import ctypes as C
import math

import pytest

from relax_b200 import _lib
from relax_b200.api import Input
from relax_b200.config import Event, Fault, Plane, Point, Tensile, relax_layer, relax_source

from cases import eigenstrain_small, linear_small, loads_small, powerlaw_small, sources_small, transient_small, two_events


def _src_eq(a, b, what):
    for f, _ in relax_source._fields_:
        assert getattr(a, f) == getattr(b, f), (what, f, getattr(a, f), getattr(b, f))


def _layers_eq(a, b, nz, what):
    assert bool(a) == bool(b), what
    if not a:
        return
    for k in range(nz):
        for f, _ in relax_layer._fields_:
            assert getattr(a[k], f) == getattr(b[k], f), (what, k, f)


def compare(got, want, nz):
    for f in ("sx1", "sx2", "sx3", "dx1", "dx2", "dx3", "beta", "nyquist", "lambda_", "mu", "gam", "interval",
              "odt", "skip", "np", "ne", "x0", "y0", "rot"):
        assert getattr(got, f) == getattr(want, f), f
    if want.skip:
        assert got.tscale == want.tscale
    for f in ("linearstruc", "nonlinearstruc", "faultcreepstruc", "ltransientstruc", "nltransientstruc"):
        _layers_eq(getattr(got, f), getattr(want, f), nz, f)
    assert not got.stressstruc and not got.lineardgammadot0 and not got.nonlineardgammadot0
    for k in range(want.np):
        for f, _ in got.planes[k]._fields_:
            assert getattr(got.planes[k], f) == getattr(want.planes[k], f), ("plane", k, f)
    for e in range(want.ne):
        ge, we = got.events[e], want.events[e]
        assert ge.time == we.time
        for kind in ("s", "ts", "m", "l"):
            n = getattr(we, "n" + kind if kind != "s" else "ns") if kind != "ts" else we.nt
            gn = getattr(ge, "n" + kind if kind != "s" else "ns") if kind != "ts" else ge.nt
            assert gn == n, (e, kind)
            for k in range(n):
                _src_eq(getattr(ge, kind)[k], getattr(we, kind)[k], (e, kind, k))
        # eigenstrain sources: cuboids (weak-zone geometry), tetrahedra, vertices
        assert (ge.nc, ge.ntet, ge.nvert) == (we.nc, we.ntet, we.nvert), e
        for k in range(we.nc):
            for f, _ in ge.c[k]._fields_:
                if f == "e":
                    assert tuple(getattr(ge.c[k].e, n) for n, _ in ge.c[k].e._fields_) == \
                        tuple(getattr(we.c[k].e, n) for n, _ in we.c[k].e._fields_), (e, k)
                else:
                    assert getattr(ge.c[k], f) == getattr(we.c[k], f), (e, k, f)
        for k in range(we.ntet):
            assert (ge.tet[k].i1, ge.tet[k].i2, ge.tet[k].i3, ge.tet[k].i4) == \
                (we.tet[k].i1, we.tet[k].i2, we.tet[k].i3, we.tet[k].i4)
            assert ge.tet[k].e.s13 == we.tet[k].e.s13
        for k in range(3 * we.nvert):
            assert ge.vert[k] == we.vert[k]
    for kind, n in (("s", want.inter.ns), ("ts", want.inter.nt)):
        assert (got.inter.ns if kind == "s" else got.inter.nt) == n
        for k in range(n):
            _src_eq(getattr(got.inter, kind)[k], getattr(want.inter, kind)[k], ("inter", kind, k))


def _rotated(sim):
    s = two_events()
    s.x0, s.y0, s.rot = 3.5, -2.25, 17.0
    s.events[0].faults[0].beta = 0.3
    s.events[0].points = [Point(0.2, 4.0, -3.0, 6.0)]
    return s


def _eigen_rotated():
    s = eigenstrain_small(tetra=False)
    s.x0, s.y0, s.rot = 2.0, -1.0, 35.0
    return s


def _loads_rotated():
    s = loads_small()
    s.x0, s.y0, s.rot = -1.5, 2.0, 23.0
    return s


CASES = {
    "linear": lambda: linear_small(),
    "powerlaw-afterslip": lambda: powerlaw_small(),
    "two-events": lambda: two_events(),
    "transient": lambda: transient_small(linear=True, nonlinear=True, viscous=True),
    "sources-interseismic": lambda: sources_small(interseismic=True),
    "rotated-origin": lambda: _rotated(None),
    "surface-loads": lambda: loads_small(),
    "surface-loads-rotated": lambda: _loads_rotated(),
    "eigenstrain": lambda: eigenstrain_small(),
    "eigenstrain-rotated": lambda: _eigen_rotated(),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_deck_reads_back_to_the_same_config(name):
    sim = CASES[name]()
    transient = bool(sim.ltransient or sim.nltransient)
    inp = Input.parse(sim.to_input(), transient=transient, eigenstrain=sim.has_eigenstrain(),
                      curvilinear=any(ev.tetrahedra for ev in sim.events))
    want, _keep = sim.to_c(_lib.structure_fn)
    compare(inp.config, want, sim.sx3h)


def test_info_and_points():
    sim = linear_small()
    sim.x0, sim.y0, sim.rot = 10.0, 20.0, 30.0
    text = sim.to_input(wdir="out/dir", oz=1.5, ozs=2.5, points=[("GPS1", 12.0, 21.0, 0.0), ("AB", 5.0, 25.0, 3.0)])
    inp = Input.parse(text)          # the info points into the input
    i = inp.info
    assert i.wdir == b"out/dir"
    assert (i.x0, i.y0, i.rot, i.oz, i.ozs) == (10.0, 20.0, 30.0, 1.5, 2.5)
    assert i.npts == 2
    # names are CHARACTER(LEN=4): blank-padded
    assert [i.ptsname[k] for k in range(2)] == [b"GPS1", b"AB  "]
    a = math.radians(30.0)
    for k, (x, y, z) in enumerate([(12.0, 21.0, 0.0), (5.0, 25.0, 3.0)]):
        x1, x2 = x - 10.0, y - 20.0
        want = (x1 * math.cos(a) + x2 * math.sin(a), -x1 * math.sin(a) + x2 * math.cos(a), z)
        assert tuple(i.pts[3 * k + j] for j in range(3)) == want
    assert i.minlength == 20.0 and i.minwidth == 6.0


def _deck(lines):
    return "\n".join(lines) + "\n"


BASE = ["64 64 32", "1 1 1 0.2 2", "0 0 0", "0 0", "out", "1 1 0", "10 -1 5",
        "0", "0", "0", "0",            # planes, points, segments, prestress
        "1", "1 6 1 0", "0",           # one linear interface, no weak zones
        "0", "0",                      # nonlinear, fault creep
        "0", "0",                      # interseismic
        "1", "1", "1 1 -10 0 0 20 6 0 90 0", "0", "0", "0"]


def test_syntax_comments_commas_repeat_and_d_exponents():
    lines = list(BASE)
    lines[1] = "  1,1,1, 0.2d0 2.0D0   extra values are ignored"
    lines[2] = "3*0"
    lines[6] = "10 -1 5 / comment after the slash"
    lines.insert(3, "   # a comment line")
    lines.insert(4, "")
    inp = Input.parse(_deck(lines))
    c = inp.config
    assert (c.dx1, c.dx2, c.dx3, c.beta, c.nyquist) == (1.0, 1.0, 1.0, 0.2, 2.0)
    assert (c.interval, c.odt, c.tscale, c.skip) == (10.0, -1.0, 5.0, 1)
    assert c.events[0].s[0].beta == 0.2        # the default smoothing


def test_optional_beta_and_event_time_rounding():
    lines = list(BASE)
    lines[6] = "10 0.5"                       # odt > 0: event times on multiples of odt
    lines[-4] = "1 1 -10 0 0 20 6 0 90 0 0.35"
    lines[-5:-5] = []
    lines += ["# next event", "2.3", "1", "1 0.5 0 0 0 10 5 0 90 0", "0", "0", "0"]
    lines[lines.index("1", 18)] = "2"        # two events
    inp = Input.parse(_deck(lines))
    c = inp.config
    assert c.skip == 0 and c.ne == 2
    assert c.events[0].s[0].beta == 0.35
    assert c.events[1].time == 2.5           # NINT(2.3 / 0.5) * 0.5


@pytest.mark.parametrize("mutate,msg", [
    (lambda l: l.__setitem__(12, "2 6 1 0"), "index misfit"),
    (lambda l: l.__setitem__(12, "1 6 -1 0"), "strain rates must be positive"),
    (lambda l: l.__setitem__(12, "1 6 1"), "cohesion missing"),
    (lambda l: l.__setitem__(0, "64 x 32"), "not an integer"),
    (lambda l: l.__setitem__(1, "1 1 1 0.2 two"), "not a number"),
    (lambda l: l.__setitem__(-4, "1 1 -10 0 0 0 0 0 90 0"), "lengths must be positive"),
    (lambda l: l.__setitem__(-4, "1 1 -10 0 0 20 6 0 90 0 1e9"), "smoothing"),
    (lambda l: l.__delitem__(slice(-3, None)), "input ends before"),
])
def test_errors(mutate, msg):
    lines = list(BASE)
    mutate(lines)
    with pytest.raises(_lib.RelaxError) as e:
        Input.parse(_deck(lines))
    assert e.value.code == 1
    assert msg in str(e.value)


def test_event_times_must_increase():
    lines = list(BASE)
    lines[18] = "2"
    lines += ["-1.0", "0", "0", "0", "0"]
    with pytest.raises(_lib.RelaxError, match="must increase"):
        Input.parse(_deck(lines))


def test_cuboid_records_and_tetrahedron_vertex_checks():
    """A cuboid record (src/input.f90:1510-1558): the strain as REAL*4, the
    geometry through wangconvention; a tetrahedron naming a vertex beyond
    the list is an input error."""
    lines = list(BASE)
    lines.insert(-1, "1")
    lines.insert(-1, "1 1e-3 0 0 0 0 0 0 0 2 5 5 5 0 90")
    inp = Input.parse(_deck(lines), eigenstrain=True)
    ev = inp.config.events[0]
    assert ev.nc == 1 and ev.c[0].e.s11 == pytest.approx(1e-3) and ev.c[0].thickness == 5.0
    assert ev.c[0].dip == 0.0                      # 90 - 90 after the convention
    bad = list(BASE)
    bad.insert(-1, "0")                            # no cuboids
    bad.insert(-1, "1")                            # one tetrahedron
    bad.insert(-1, "1 1e-3 0 0 0 0 0 1 2 3 5")
    bad.insert(-1, "4")
    for k in range(4):
        bad.insert(-1, f"{k + 1} {k} 0 1")
    with pytest.raises(_lib.RelaxError) as e:
        Input.parse(_deck(bad), eigenstrain=True, curvilinear=True)
    assert e.value.code == 1


def test_weak_zones_in_internal_convention():
    lines = list(BASE)
    lines[13] = "2"
    lines.insert(14, "1 2.0 0 0 8 10 12 6 0.3 90")
    lines.insert(15, "2 1.0 5 -5 4 -3 -3 -3 0 90")
    inp = Input.parse(_deck(lines))
    assert list(inp.info.nwz) == [2, 0, 0, 0]
    z = inp.weakzones(0)
    from relax_b200.config import wang_convention
    _, x, y, zz, strike, dip, _ = wang_convention(0.0, 0, 0, 8, 10, 12, 0.3, 90, 0.0)
    assert (z[0].dgammadot0, z[0].x, z[0].y, z[0].z, z[0].strike, z[0].dip) == (2.0, x, y, zz, strike, dip)
    assert (z[0].length, z[0].width, z[0].thickness) == (10.0, 12.0, 6.0)


def test_echo_formats(capfd):
    Input.parse(_deck(BASE), echo=True)
    out = capfd.readouterr().out.splitlines()
    assert out[:4] == ["# grid dimension (sx1,sx2,sx3)", "   64   64   32",
                       "# sampling (dx1,dx2,dx3), smoothing (beta, nyquist)",
                       "  1.00E+0  1.00E+0  1.00E+0  2.00E-1  2.00E+0"]
    assert "# output every 001 steps, dt scaled by 5.00E+0" in out
    assert "001  6.00E+00  1.00E+00  0.00E+00" in out
    assert "0001  1.00E+0 -1.00E+1  0.00E+0  0.00E+0 2.00E+1 6.00E+0    0.0  90.0    0.0" in out


def test_observation_planes_and_segments_in_internal_convention():
    from relax_b200.config import wang_convention
    sim = linear_small(sx=32, sz=16)
    sim.x0, sim.y0, sim.rot = 2.0, -1.0, 15.0
    planes = [(1.0, 2.0, 0.5, 8.0, 6.0, 30.0, 60.0), (-3.0, 4.0, 1.0, 5.0, 5.0, -20.0, 90.0)]
    segs = [(0.5, -1.5, 2.0, 4.0, 3.0, 10.0, 45.0, 0.6)]
    inp = Input.parse(sim.to_input(obsplanes=planes, segments=segs))
    assert (inp.info.nop, inp.info.nsop) == (2, 1)
    for got, (x, y, z, L, W, s, d) in zip(inp.obsplanes(), planes):
        _, wx, wy, wz, ws, wd, _ = wang_convention(0.0, x, y, z, L, W, s, d, 0.0, 2.0, -1.0, 15.0)
        assert (got.x, got.y, got.z, got.length, got.width, got.strike, got.dip) == (wx, wy, wz, L, W, ws, wd)
    (g,) = inp.segments()
    x, y, z, L, W, s, d, fr = segs[0]
    _, wx, wy, wz, ws, wd, _ = wang_convention(0.0, x, y, z, L, W, s, d, 0.0, 2.0, -1.0, 15.0)
    assert (g.x, g.y, g.z, g.length, g.width, g.strike, g.dip, g.friction) == (wx, wy, wz, L, W, ws, wd, fr)
