"""The output files of RELAX written by the library's host code: GMT netCDF
grids (src/exportnetcdf.f90, exportgrd of src/export.f90:917-1057), VTK
legacy files (src/writevtk.c), the .ned rows and the log line (Fortran
ES edit descriptors of src/relax.f90:1102-1105 and src/util.f90:120) and
shiftedindex (src/elastic3d.f90:4063-4101).  No device work: these run on
the CPU."""
import os

import numpy as np
import pytest
from scipy.io import netcdf_file

from relax_b200 import _lib, api
from relax_b200.config import relax_step_log, relax_tensor


@pytest.fixture(scope="module", autouse=True)
def lib():
    return _lib.load()


def _read_grd(path):
    with netcdf_file(path, "r", mmap=False) as f:
        x = f.variables["x"][:].copy()
        y = f.variables["y"][:].copy()
        z = f.variables["z"][:].copy()
        out = dict(x=x, y=y, z=z, zdims=f.variables["z"].dimensions,
                   ztype=f.variables["z"].typecode(), xtype=f.variables["x"].typecode(),
                   xrange=f.variables["x"].actual_range.copy(), yrange=f.variables["y"].actual_range.copy(),
                   zrange=f.variables["z"].actual_range.copy(), zrangetype=f.variables["z"].actual_range.dtype,
                   title=f.title, history=f.history, conventions=f.Conventions, node_offset=f.node_offset,
                   long_names=[f.variables[v].long_name for v in ("x", "y", "z")])
    return out


def test_grd_layout(tmp_path):
    rng = np.random.default_rng(0)
    z = rng.standard_normal((6, 10)).astype(np.float32)        # ny = 6, nx = 10
    path = tmp_path / "t.grd"
    api.write_grd(z, x0=-5.0, y0=2.0, dx=0.5, dy=0.25, title="007-north", filename=path)
    g = _read_grd(path)
    assert g["zdims"] == ("y", "x")
    assert g["ztype"] == "f" and g["xtype"] == "d"
    np.testing.assert_array_equal(g["x"], -5.0 + 0.5 * np.arange(10))
    np.testing.assert_array_equal(g["y"], 2.0 + 0.25 * np.arange(6))
    np.testing.assert_array_equal(g["z"], z)
    # pixel registration: the range extends half a cell beyond the nodes
    np.testing.assert_array_equal(g["xrange"], [-5.25, -5.0 + 0.5 * 9 + 0.25])
    np.testing.assert_array_equal(g["yrange"], [2.0 - 0.125, 2.0 + 0.25 * 5 + 0.125])
    assert g["zrangetype"].kind == "f" and g["zrangetype"].itemsize == 4
    np.testing.assert_array_equal(g["zrange"], [z.min(), z.max()])
    assert g["node_offset"] == 1
    assert g["title"] == b"007-north"
    assert g["history"] == b"Relax output"
    assert g["conventions"] == b"COARDS/CF-1.0"
    assert g["long_names"] == [b"x", b"y", b"z"]
    # the header is padded to 4 bytes and the data follow it
    raw = path.read_bytes()
    assert raw[:4] == b"CDF\x01"
    assert len(raw) % 4 == 0
    assert raw.endswith(z.astype(">f4").tobytes())


def _exportspatial(plane):
    """exportspatial with doflip (src/elastic3d.f90:4166-4207): (sx2, sx1)
    x1-fastest plane -> (sx1, sx2) x2-fastest, the origin in the middle."""
    return np.fft.fftshift(plane.T)


@pytest.mark.parametrize("convention", [1, 2, 3, 4, 5, 6, 7])
def test_exportgrd_files(tmp_path, convention):
    sx1, sx2 = 16, 8
    dx1, dx2, origx, origy = 0.5, 2.0, 100.0, -30.0
    rng = np.random.default_rng(convention)
    planes = [rng.standard_normal((sx2, sx1)).astype(np.float32) for _ in range(3)]
    api.write_grd3(planes, dx1, dx2, origx, origy, tmp_path, 12, convention)
    names = {1: ("north", "east", "up"), 2: ("relax-north", "relax-east", "relax-up"),
             3: ("eqbf-north", "eqbf-east", "eqbf-up"), 4: ("s11", "s12", "s13"), 5: ("s22", "s23", "s33"),
             6: ("e11", "e12", "e13"), 7: ("e22", "e23", "e33")}[convention]
    assert sorted(os.listdir(tmp_path)) == sorted(f"012-{n}.grd" for n in names)
    for k, n in enumerate(names):
        g = _read_grd(tmp_path / f"012-{n}.grd")
        want = _exportspatial(planes[k])
        if k == 2 and convention <= 3:
            want = -want                     # positive up
        np.testing.assert_array_equal(g["z"], want)
        # x east from origy, y north from origx
        np.testing.assert_array_equal(g["x"], origy - sx2 // 2 * dx2 + dx2 * np.arange(sx2))
        np.testing.assert_array_equal(g["y"], origx - sx1 // 2 * dx1 + dx1 * np.arange(sx1))
        assert g["title"] == f"012-{n}".encode()


def test_exportgrd_rejects_bad_convention(tmp_path):
    p = [np.zeros((4, 4), np.float32)] * 3
    with pytest.raises(_lib.RelaxError):
        api.write_grd3(p, 1.0, 1.0, 0.0, 0.0, tmp_path, 0, 8)
    with pytest.raises(_lib.RelaxError):
        api.write_grd3(p, 1.0, 1.0, 0.0, 0.0, tmp_path / "missing-dir", 0, 1)


def _read_vtk(path):
    raw = path.read_bytes()
    lines, pos = [], 0
    while len(lines) < 9:
        e = raw.index(b"\n", pos)
        lines.append(raw[pos:e].decode())
        pos = e + 1
    return lines, np.frombuffer(raw[pos:], ">f4")


def _vtk_order(field, j):
    """The point order of src/writevtk.c:114-136: k3 from 0, k2 and k1 from
    -sx/2, every j-th point; field (sx3, sx2, sx1)."""
    sx3, sx2, sx1 = field.shape
    i1 = [(sx1 + k) % sx1 for k in range(-sx1 // 2, sx1 // 2, j[0])]
    i2 = [(sx2 + k) % sx2 for k in range(-sx2 // 2, sx2 // 2, j[1])]
    i3 = list(range(0, sx3, j[2]))
    return field[np.ix_(i3, i2, i1)]


@pytest.mark.parametrize("ncomp,strides", [(3, (1, 1, 1)), (3, (4, 2, 2)), (6, (2, 2, 1))])
def test_vtk_legacy(tmp_path, ncomp, strides):
    sx1, sx2, sx3 = 16, 8, 6
    dx = (0.5, 0.25, 2.0)
    rng = np.random.default_rng(ncomp)
    comps = [rng.standard_normal((sx3, sx2, sx1)).astype(np.float32) for _ in range(ncomp)]
    path = tmp_path / "f.vtk"
    api.write_vtk(comps, dx, strides, path, title="cumulative displacement vector field", name="displacement")
    lines, data = _read_vtk(path)
    n1, n2, n3 = sx1 // strides[0], sx2 // strides[1], sx3 // strides[2]
    assert lines == ["# vtk DataFile Version 3.0", "cumulative displacement vector field", "BINARY",
                     "DATASET STRUCTURED_POINTS", f"DIMENSIONS {n1} {n2} {n3}",
                     "ORIGIN %f %f %f" % (-dx[0] * (sx1 // 2), -dx[1] * (sx2 // 2), 0.0),
                     "SPACING %f %f %f" % (dx[0] * strides[0], dx[1] * strides[1], dx[2] * strides[2]),
                     f"POINT_DATA {n1 * n2 * n3}",
                     ("VECTORS" if ncomp == 3 else "TENSORS") + " displacement float"]
    sel = [_vtk_order(c, strides).ravel() for c in comps]
    if ncomp == 3:
        want = np.stack(sel, axis=1)
    else:
        s11, s12, s13, s22, s23, s33 = sel
        want = np.stack([s11, s12, s13, s12, s22, s23, s13, s23, s33], axis=1)
    np.testing.assert_array_equal(data, want.ravel())


@pytest.mark.parametrize("v,w,d,e,want", [
    (1234.5, 9, 2, 2, " 1.23E+03"),
    (-0.000123, 9, 2, 2, "-1.23E-04"),
    (0.0, 9, 2, 2, " 0.00E+00"),
    (1234.5, 11, 2, 0, "   1.23E+03"),
    (-4.5e-7, 11, 2, 0, "  -4.50E-07"),
    (1.0e150, 11, 2, 0, "   1.00+150"),
    (-2.5e-120, 11, 2, 0, "  -2.50-120"),
    (1.0e300, 11, 2, 0, "   1.00+300"),
    (-1.0e300, 8, 2, 0, "********"),
    (9.996, 9, 2, 2, " 1.00E+01"),
    (1e100, 9, 2, 2, "*********"),
    (100.0, 7, 2, 1, "1.00E+2"),
    (1e10, 7, 2, 1, "*******"),
    (-100.0, 7, 2, 1, "*******"),
    (3.14159265358979, 16, 8, 2, "  3.14159265E+00"),
    (-2.5e-7, 16, 8, 2, " -2.50000000E-07"),
    (12.0, 11, 3, 2, "  1.200E+01"),
])
def test_es_edit_descriptor(v, w, d, e, want):
    assert api.es_format(v, w, d, e) == want


def test_log_line():
    lg = relax_step_log(i=5, event=0, dt=0.5, tm_ve=1e3, tm_pl=0.0, tm_as=0.0, t=2.5, power=1.5e-3, cei=2.0,
                        tm_tl=7.0, tm_tnl=8.0, output=1)
    assert api.format_log(lg, 10.0) == \
        "005* 5.00E-01 1.00E+03 0.00E+00 0.00E+00 2.50E+00/1.00E+1 1.50E-03 2.00E+00"
    lg.output = 0
    assert api.format_log(lg, 10.0, transient=True) == \
        "005  5.00E-01 1.00E+03 0.00E+00 0.00E+00 7.00E+00 8.00E+00 2.50E+00/1.00E+1 1.50E-03 2.00E+00"
    lg.i = 1234                         # I3.3 overflows
    assert api.format_log(lg, 10.0).startswith("*** ")
    assert api.log_header() == " I  |   Dt   | tm(ve) | tm(pl) | tm(as) |     t/tmax     | power  |  C:E^i | "
    assert "tm(kl) | tm(kn)" in api.log_header(True)


def test_ned_row(lib):
    import ctypes as C
    u = (C.c_double * 3)(1.0, -2.0, 3.5e-3)
    s = relax_tensor(s11=1, s12=2, s13=3, s22=4, s23=5, s33=-6)
    buf = C.create_string_buffer(400)
    _lib.check(lib.relax_format_ned(0.25, u, C.byref(s), buf, 400))
    row = buf.value.decode()
    assert len(row) == 10 * 16
    vals = [float(row[16 * k:16 * k + 16]) for k in range(10)]
    assert vals == [0.25, 1.0, -2.0, 3.5e-3, 1, 2, 3, 4, 5, -6]
    assert lib.relax_ned_header().decode().split() == \
        ["#", "t", "u1", "u2", "u3", "s11", "s12", "s13", "s22", "s23", "s33"]


def _fix(x):
    """fix, src/elastic3d.f90:70-83: halves round down."""
    f, c = np.floor(x), np.ceil(x)
    return int(c) if x - f > 0.5 else int(f)


def test_shifted_index():
    sx, dx = (16, 8, 8), (2.0, 3.0, 1.5)
    rng = np.random.default_rng(3)
    cases = [(0.0, 0.0, 0.0), (-16.0, -12.0, 0.0), (14.0, 9.0, 10.5), (1.0, 1.5, 0.75), (-1.0, -1.5, 2.25),
             (-3.0, 4.5, 3.0)]
    cases += [(rng.uniform(-16, 14), rng.uniform(-12, 9), rng.uniform(0, 10.5)) for _ in range(50)]
    for x in cases:
        want = ((sx[0] + _fix(x[0] / dx[0])) % sx[0], (sx[1] + _fix(x[1] / dx[1])) % sx[1], _fix(x[2] / dx[2]))
        assert api.shifted_index(x, sx, dx) == want, x
    for bad in [(14.5, 0, 0), (-16.5, 0, 0), (0, 9.5, 0), (0, -12.5, 0), (0, 0, 11.0), (0, 0, -0.1)]:
        with pytest.raises(_lib.RelaxError):
            api.shifted_index(bad, sx, dx)
