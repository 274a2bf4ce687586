"""Output files written from a context's device fields: plane and point
read-backs against the full-field copy, the GRD grids of exportgrd /
exportstressgrd (src/export.f90:860-1057), the VTK legacy files
(src/writevtk.c), the .ned series of exportpoints (src/util.f90:59-170) and
the isoutput flag of the log (src/relax.f90:907, :1364-1376)."""
import math

import numpy as np
import pytest
from scipy.io import netcdf_file

from relax_b200 import api
from relax_b200.api import Relax

from cases import linear_small, powerlaw_small, transient_small

pytestmark = pytest.mark.gpu


def _grd(path):
    with netcdf_file(path, "r", mmap=False) as f:
        return f.variables["z"][:].copy()


def _fix(x):
    f, c = math.floor(x), math.ceil(x)
    return c if x - f > 0.5 else f


@pytest.fixture(scope="module")
def stepped():
    sim = linear_small(sx=64, sz=32)
    r = Relax(sim)
    r.coseismic()
    for _ in range(2):
        r.step()
    yield sim, r
    r.close()


def test_plane_and_points_match_fields(stepped):
    sim, r = stepped
    u = r.field("u")[..., :sim.sx1]
    sig = r.field("sig")
    for i3 in (0, 5, sim.sx3h - 1):
        np.testing.assert_array_equal(r.plane("u", i3), u[:, i3])
        p = r.plane("sig", i3)
        for k, n in enumerate(sig.dtype.names):
            np.testing.assert_array_equal(p[k], sig[n][i3])
    rng = np.random.default_rng(1)
    idx = np.stack([rng.integers(0, s, 40) for s in (sim.sx1, sim.sx2, sim.sx3h)], axis=1)
    pu, ps = r.points(idx)
    for k, (i1, i2, i3) in enumerate(idx):
        assert tuple(pu[k]) == tuple(float(u[c, i3, i2, i1]) for c in range(3))
        assert ps[k] == sig[i3, i2, i1]


def test_grd_exports(stepped, tmp_path):
    sim, r = stepped
    oz = 2.6 * sim.dx3
    r.export_grd("u", tmp_path, 3, oz=oz, origx=10.0, origy=-4.0)
    u = r.field("u")[..., :sim.sx1]
    k3 = int(oz / sim.dx3)
    for c, n in enumerate(("north", "east", "up")):
        want = np.fft.fftshift(u[c, k3].T) * (-1 if c == 2 else 1)
        np.testing.assert_array_equal(_grd(tmp_path / f"003-{n}.grd"), want)
    r.export_grd("sig", tmp_path, 3, oz=oz)
    sig = r.field("sig")
    k3 = _fix(oz / sim.dx3)
    for n in sig.dtype.names:
        np.testing.assert_array_equal(_grd(tmp_path / f"003-{n}.grd"), np.fft.fftshift(sig[n][k3].T))


def test_vtk_export(stepped, tmp_path):
    sim, r = stepped
    depth, j = sim.sx3 // 4, (4, 4, 2)
    path = tmp_path / "disp-001.vtk"
    r.export_vtk("u", path, depth, j, title="cumulative displacement vector field", vname="displacement")
    raw = path.read_bytes()
    head = raw.split(b"\n", 9)
    assert head[8] == b"VECTORS displacement float"
    data = np.frombuffer(head[9], ">f4").reshape(-1, 3)
    u = r.field("u")[..., :sim.sx1]
    i1 = [(sim.sx1 + k) % sim.sx1 for k in range(-sim.sx1 // 2, sim.sx1 // 2, j[0])]
    i2 = [(sim.sx2 + k) % sim.sx2 for k in range(-sim.sx2 // 2, sim.sx2 // 2, j[1])]
    i3 = list(range(0, depth, j[2]))
    want = np.stack([u[c][np.ix_(i3, i2, i1)].ravel() for c in range(3)], axis=1)
    np.testing.assert_array_equal(data, want)
    # the tensor form through the host writer gives the same bytes
    sig = r.field("sig")
    path2 = tmp_path / "sig-a.vtk"
    r.export_vtk("sig", path2, depth, j, title="stress", vname="stress")
    path3 = tmp_path / "sig-b.vtk"
    api.write_vtk([sig[n] for n in sig.dtype.names], (sim.dx1, sim.dx2, sim.dx3), j, path3,
                  title="stress", name="stress")
    # the host writer covers every plane it is given; cut it at `depth`
    a = path2.read_bytes()
    b = path3.read_bytes()
    ha, hb = a.split(b"\n", 9), b.split(b"\n", 9)
    n = len(ha[9])
    assert ha[0:4] == hb[0:4] and ha[5:7] == hb[5:7] and ha[8] == hb[8]
    assert ha[9] == hb[9][:n]


def test_points_ned(stepped, tmp_path):
    sim, r = stepped
    xyz = np.array([[0.0, 0.0, 0.0], [-5.0, 3.0, 2.0], [7.4, -12.6, 4.5]])
    names = ["GPS1", "GPS2", "BH03"]
    rot = 30.0
    r.export_points(xyz, names, 0.0, tmp_path, isnew=True, rot=rot)
    r.export_points(xyz, names, 1.0, tmp_path, isnew=False, rot=rot)
    u = r.field("u")[..., :sim.sx1]
    sig = r.field("sig")
    a = math.radians(-rot)
    for k, name in enumerate(names):
        lines = (tmp_path / f"{name}.ned").read_text().splitlines()
        assert lines[0] == api._lib.load().relax_ned_header().decode()
        assert len(lines) == 3
        i1, i2, i3 = api.shifted_index(xyz[k], (sim.sx1, sim.sx2, sim.sx3h), (sim.dx1, sim.dx2, sim.dx3))
        uv = [float(u[c, i3, i2, i1]) for c in range(3)]
        v1 = uv[0] * math.cos(a) + uv[1] * math.sin(a)
        v2 = -uv[0] * math.sin(a) + uv[1] * math.cos(a)
        for t, line in zip((0.0, 1.0), lines[1:]):
            vals = [float(line[16 * j:16 * j + 16]) for j in range(10)]
            assert vals[0] == t
            np.testing.assert_allclose(vals[1:4], [v1, v2, uv[2]], rtol=1e-7, atol=1e-12)
            np.testing.assert_allclose(vals[4:], [float(sig[n][i3, i2, i1]) for n in sig.dtype.names],
                                       rtol=1e-7, atol=1e-12)
        ct = (tmp_path / f"{name}.c.txt").read_text().splitlines()
        assert len(ct) == 3 and ct[0].split() == ["#", "t", "u1", "u2", "u3"]


def test_output_flag_follows_isoutput():
    sim = linear_small(sx=64, sz=32, steps=6)
    sim.odt = 1.0          # output every unit of time: Dt = tm/10, cut to land on them
    with Relax(sim) as r:
        r.coseismic()
        oi, flags = 1, []
        while True:
            lg = r.step()
            if lg[0] == 0:
                break
            want = abs(lg[5] - oi * sim.odt) < 1e-6 * sim.odt
            if want:
                oi += 1
            flags.append(r.last_log.output)
            assert r.last_log.output == int(want), (lg, oi)
        assert sum(flags) >= 2 and 0 in flags
        line = api.format_log(r.last_log, sim.interval)
        assert line[3] in "* " and "/" in line


def test_transient_strain_grids(tmp_path):
    sim = transient_small(linear=True)
    with Relax(sim) as r:
        r.coseismic()
        r.step()
        r.step()
        eps = r.field("eps")
        assert any(np.abs(eps[n]).max() > 0 for n in eps.dtype.names)
        r.export_grd("eps", tmp_path, 1, oz=0.0)
        for n in eps.dtype.names:
            e = "e" + n[1:]
            np.testing.assert_array_equal(_grd(tmp_path / f"001-{e}.grd"), np.fft.fftshift(eps[n][0].T))


def test_creep_exports(tmp_path):
    """exportcreep_asc / exportcreep_grd (src/export.f90:563-767) of an
    afterslip plane: every third patch per line in ES11.3E2, and the
    strike-reversed grids of slip and slip rate (the reference's vel-strike
    grid holds the dip-slip rate, vel-dip the strike-slip rate)."""
    sim = powerlaw_small(sx=64, sz=32)
    with Relax(sim) as r:
        r.coseismic()
        for _ in range(3):
            r.step()
        r.export_creep(tmp_path, 4, vtk=True)
        p = np.ctypeslib.as_array(r.patches(0)).copy()
        n1, n2 = r.cfg.planes[0].px2, r.cfg.planes[0].px3
    assert n1 >= 6 and n2 >= 4 and np.abs(p["v"]).max() > 0
    p = p.reshape(n2, n1)
    names = ("x1", "x2", "x3", "lx", "lz", "slip", "ss", "ds", "v", "vss", "vds", "taus")
    lines = (tmp_path / "004.s00001.creep.dat").read_text().splitlines()
    assert lines[0].split() == ["#", "x1", "x2", "x3", "yr", "yz", "slip", "strike-slip", "dip-slip", "velocity",
                                "ss", "vel", "ds", "vel", "taus", "sig11", "sig12", "sig13", "sig22", "sig23",
                                "sig33"]
    want = []
    for i2 in range(0, n2, 3):
        for i1 in range(0, n1, 3):
            q = p[i2, i1]
            vals = [q[n] for n in names] + [q["sig"][n] for n in ("s11", "s12", "s13", "s22", "s23", "s33")]
            want.append("".join(api.es_format(float(v), 11, 3, 2) for v in vals))
    assert lines[1:] == want
    for f, name in (("ds", "slip-dip"), ("ss", "slip-strike"), ("slip", "slip"), ("vds", "vel-strike"),
                    ("vss", "vel-dip"), ("v", "vel")):
        with netcdf_file(tmp_path / f"004.s00001.{name}.grd", "r", mmap=False) as g:
            z = g.variables["z"][:].copy()
            x = g.variables["x"][:].copy()
            y = g.variables["y"][:].copy()
        np.testing.assert_array_equal(z, p[f][:, ::-1].astype(np.float32))
        assert x[0] == p["lx"].min() and y[0] == -p["lz"].max()
        np.testing.assert_allclose(np.diff(x), sim.dx2)
        np.testing.assert_allclose(np.diff(y), sim.dx3)
    # exportcreep_vtk: points, two triangles per cell, seven scalar fields
    flat = p.reshape(-1)
    text = (tmp_path / "creep-00001s-004.vtk").read_text().splitlines()
    assert text[:5] == ["# vtk DataFile Version 3.0", "afterslip", "ASCII", "DATASET POLYDATA",
                        f"POINTS {n1 * n2} float"]
    pts = text[5:5 + n1 * n2]
    assert pts == ["".join(api.es_format(float(q[f]), 11, 3, 2) for f in ("x1", "x2", "x3")) for q in flat]
    k = 5 + n1 * n2
    ncell = (n1 - 1) * (n2 - 1)
    assert text[k] == "" and text[k + 1] == f"POLYGONS {2 * ncell} {8 * ncell}"
    tri = [list(map(int, l.split()))[1:] for l in text[k + 2:k + 2 + 2 * ncell]]
    assert tri[0] == [0, 1, n1 + 1] and tri[1] == [0, n1, n1 + 1]
    a0 = (n2 - 2) * n1 + n1 - 2
    assert tri[-2] == [a0, a0 + 1, (n2 - 1) * n1 + n1 - 1]
    assert tri[-1] == [a0, (n2 - 1) * n1 + n1 - 2, (n2 - 1) * n1 + n1 - 1]
    k += 2 + 2 * ncell
    assert text[k] == "" and text[k + 1] == f"POINT_DATA {n1 * n2}"
    k += 2
    for name, f in (("afterslip", "slip"), ("strike_slip", "ss"), ("dip-slip", "ds"), ("velocity", "v"),
                    ("velocity_strike_slip", "vss"), ("velocity_dip_slip", "vds"), ("shear_stress", "taus")):
        assert text[k:k + 2] == [f"SCALARS {name} float", "LOOKUP_TABLE default"]
        vals = np.array([float(v) for v in text[k + 2:k + 2 + n1 * n2]])
        np.testing.assert_array_equal(vals, flat[f])
        k += 2 + n1 * n2
    assert k == len(text)
