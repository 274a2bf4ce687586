"""The geometry files of the input reader (src/export.f90:1068-1206,
1216-1354, 2014-2153, 2295-2599, written by init, src/input.f90:296-1452):
names and contents against a restatement of the reference's corner formulas
and edit descriptors; host code only."""
import math
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from relax_b200 import api
from relax_b200.api import Input


def _es(v, w=11, d=2, e=0):
    return api.es_format(float(v), w, d, e)


def _frame(strike, dip):
    cs, ss, cd, sd = math.cos(strike), math.sin(strike), math.cos(dip), math.sin(dip)
    return (ss, cs, 0.0), (cs * sd, -ss * sd, cd), (cd * cs, -cd * ss, -sd)


def _corner(x, L, W, T, frame, sd, ss, sn):
    s, d, n = frame
    out = []
    for k in range(3):
        v = x[k] + sd * d[k] * W / 2 + ss * s[k] * L / 2
        if sn:
            v = v + sn * n[k] * T / 2.0
        out.append(v)
    return out


RECT = [(-1, -1), (-1, 1), (1, 1), (1, -1)]


def _deck(wdir):
    return "\n".join([
        "64 64 32", "1 1 1 0.2 2", "2 -1 10", "0 0", str(wdir), "1 1 0", "10 -1 5",
        "0", "0", "0", "0",
        "1", "1 6 1 0",
        "2", "1 2.0 0 0 8 10 12 6 0.3 90", "2 1.0 5 -5 4 3 4 2 30 60",
        "0", "0", "0", "0",
        "1", "1", "1 1 -10 0 0 20 6 0 90 0", "1", "1 0.5 3 4 1 5 2 20 80", "0", "0"]) + "\n"


@pytest.fixture(scope="module")
def exported(tmp_path_factory):
    d = tmp_path_factory.mktemp("geometry")
    inp = Input.parse(_deck(d))
    inp.export_geometry(vtk=True)
    return d, inp


def _body(el):
    return el.text.split("\n")[1:-1]


def test_files_written(exported):
    d, _ = exported
    names = sorted(p.name for p in d.iterdir())
    assert names == ["cgrid.vtp", "linearlayer-001.vtp", "rdykes-001.vtp", "rdykes-001.xy", "rfaults-001.vtp",
                     "rfaults-001.xy", "weakzone-001.xy", "weakzone-002.xy", "weakzones-linear.vtp"]


def test_grid_box(exported):
    d, _ = exported
    a, b, c = 64 * 1.0 / 2, 64 * 1.0 / 2, 32 * 1.0 / 2
    vals = [-a, -b, c, a, -b, c, a, b, c, -a, b, c, -a, -b, 0.0, a, -b, 0.0, a, b, 0.0, -a, b, 0.0]
    root = ET.fromstring((d / "cgrid.vtp").read_text().split("\n", 1)[1])
    piece = root.find("PolyData").find("Piece")
    assert piece.attrib == {"NumberOfPoints": "8", "NumberOfPolys": "6"}
    assert _body(piece.find("Points").find("DataArray")) == ["".join(_es(v, 9, 2, 1) for v in vals)]
    polys = {a.attrib["Name"]: a.text.strip() for a in piece.find("Polys").findall("DataArray")}
    assert polys == {"connectivity": "0 1 2 3 4 5 6 7 2 3 7 6 0 3 7 4 0 1 5 4 1 2 6 5",
                     "offsets": "4 8 12 16 20 24"}


def test_layer_rectangle(exported):
    d, _ = exported
    fr = _frame(0.0, 1.5708)
    want = "".join(_es(v) for sd, ss in RECT for v in _corner((0.0, 0.0, 6.0), 64.0, 64.0, 0.0, fr, sd, ss, 0))
    root = ET.fromstring((d / "linearlayer-001.vtp").read_text().split("\n", 1)[1])
    assert _body(root.find("PolyData").find("Piece").find("Points").find("DataArray")) == [want]


def test_weak_zones(exported):
    d, inp = exported
    zones = inp.weakzones(0)
    assert len(zones) == 2
    pieces = ET.fromstring((d / "weakzones-linear.vtp").read_text().split("\n", 1)[1]).find("PolyData").findall(
        "Piece")
    assert len(pieces) == 4
    order = [(-1, -1, -1), (-1, 1, -1), (1, 1, -1), (1, -1, -1), (1, -1, 1), (-1, -1, 1), (-1, 1, 1), (1, 1, 1)]
    for k, z in enumerate(zones):
        fr = _frame(z.strike, z.dip)
        x = (z.x, z.y, z.z)
        # GMT: the faces below and above the mid-plane, (east, north, depth)
        lines = (d / f"weakzone-{k + 1:03d}.xy").read_text().splitlines()
        want = []
        for sd in (-1, 1):
            want.append(">")
            for ss, sn in [(-1, -1), (1, -1), (1, 1), (-1, 1), (-1, -1)]:
                c = _corner(x, z.length, z.width, z.thickness, fr, sd, ss, sn)
                want.append(_es(c[1]) + _es(c[0]) + _es(c[2]))
        assert lines == want
        pts = "".join(_es(v) for o in order for v in _corner(x, z.length, z.width, z.thickness, fr, *o))
        for piece, conn in zip(pieces[2 * k:2 * k + 2], ("7 4 5 6 7 4 3 2 7 2 1 6", "0 1 2 3 0 5 4 3 0 1 6 5")):
            assert _body(piece.find("Points").find("DataArray")) == [pts]
            polys = {a.attrib["Name"]: a.text.strip() for a in piece.find("Polys").findall("DataArray")}
            assert polys == {"connectivity": conn, "offsets": "12"}
            cells = {a.attrib["Name"]: _body(a) for a in piece.find("CellData").findall("DataArray")}
            assert list(cells) == ["isotropic strain", "deviatoric strain", "e11", "e12", "e13", "e22", "e23",
                                   "e33"]
            assert all(v == [_es(0.0)] for v in cells.values())


def test_event_faults(exported):
    d, inp = exported
    ev = inp.config.events[0]
    assert ev.ns == 1 and ev.nt == 1
    s = ev.s[0]
    fr = _frame(s.strike, s.dip)
    # GMT polygons carry the origin (x0, y0) = (2, -1)
    for stem in ("rfaults", "rdykes"):      # the dykes file holds the event's shear faults, as in the reference
        lines = (d / f"{stem}-001.xy").read_text().splitlines()
        x = (s.x + 2.0, s.y - 1.0, s.z)
        want = ["> # east, north", "> -Z" + _es(abs(s.slip))]
        for sd, ss in RECT:
            c = _corner(x, s.length, s.width, 0.0, fr, sd, ss, 0)
            want.append(_es(c[1]) + _es(c[0]))
        assert lines == want
        piece = ET.fromstring((d / f"{stem}-001.vtp").read_text().split("\n", 1)[1]).find("PolyData").find("Piece")
        pts = "".join(_es(v) for sd, ss in RECT for v in _corner((s.x, s.y, s.z), s.length, s.width, 0.0, fr, sd,
                                                                 ss, 0))
        assert _body(piece.find("Points").find("DataArray")) == [pts]
        cells = {a.attrib["Name"]: _body(a) for a in piece.find("CellData").findall("DataArray")}
        sv, dv, nv = fr
        slip = [(sv[k] * math.cos(s.rake) + dv[k] * math.sin(s.rake)) * s.slip for k in range(3)]
        assert cells["slip"] == ["".join(_es(v) for v in slip)]
        assert cells["opening"] == ["".join(_es(nv[k] * s.opening) for k in range(3))]


def test_without_vtk_only_gmt(tmp_path):
    inp = Input.parse(_deck(tmp_path))
    inp.export_geometry(vtk=False)
    assert sorted(p.name for p in tmp_path.iterdir()) == ["rdykes-001.xy", "rfaults-001.xy", "weakzone-001.xy",
                                                         "weakzone-002.xy"]
