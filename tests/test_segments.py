"""Stress observation segments (src/export.f90:1403-2005): the GMT polygons
of exportgmt_rfaults_stress, the traction rows of
exportgmt_rfaults_traction, the VTK PolyData of exportvtk_rfaults_stress and
the time series of exportcoulombstress, checked line by line against a
restatement of the reference's resolution of the stress on each segment
(single-precision tensor, double-precision vectors, ES edit descriptors)."""
import math
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from relax_b200 import api
from relax_b200.config import relax_segment, relax_tensor

NAMES = ("s11", "s12", "s13", "s22", "s23", "s33")


def _segments(n=4, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        out.append(relax_segment(x=rng.uniform(-20, 20), y=rng.uniform(-20, 20), z=rng.uniform(0, 15),
                                 length=rng.uniform(1, 30), width=rng.uniform(1, 10),
                                 strike=rng.uniform(-math.pi, math.pi), dip=rng.uniform(0, math.pi / 2),
                                 friction=rng.uniform(0, 0.8)))
    return out


def _tensors(n, seed, scale=1e-3):
    rng = np.random.default_rng(seed)
    return [relax_tensor(*[float(np.float32(v)) for v in rng.normal(0, scale, 6)]) for _ in range(n)]


def _resolve(g, sig, sig0=None):
    """The normal, shear and Coulomb stress of src/export.f90:1580-1622."""
    t32 = np.array([getattr(sig, n) for n in NAMES], np.float32) if sig is not None else np.zeros(6, np.float32)
    if sig is not None and sig0 is not None:
        t32 = t32 - np.array([getattr(sig0, n) for n in NAMES], np.float32)
    s11, s12, s13, s22, s23, s33 = (float(v) for v in t32)
    cs, ss, cd, sd = math.cos(g.strike), math.sin(g.strike), math.cos(g.dip), math.sin(g.dip)
    n = (cd * cs, -cd * ss, -sd)
    s = (ss, cs, 0.0)
    d = (-cs * sd, ss * sd, -cd)
    t = (s11 * n[0] + s12 * n[1] + s13 * n[2], s12 * n[0] + s22 * n[1] + s23 * n[2],
         s13 * n[0] + s23 * n[1] + s33 * n[2])
    taun = t[0] * n[0] + t[1] * n[1] + t[2] * n[2]
    ts = tuple(t[k] - taun * n[k] for k in range(3))
    taus = math.sqrt(ts[0] * ts[0] + ts[1] * ts[1] + ts[2] * ts[2])
    tstrike = ts[0] * s[0] + ts[1] * s[1] + ts[2] * s[2]
    tdip = ts[0] * d[0] + ts[1] * d[1] + ts[2] * d[2]
    return dict(sig=(s11, s12, s13, s22, s23, s33), n=n, s=s, d=d, t=t, ts=ts, taun=taun, taus=taus,
                tstrike=tstrike, tdip=tdip, coulomb=taus + g.friction * taun)


def _row(vals, w=11, d=2, e=0):
    return "".join(api.es_format(float(v), w, d, e) for v in vals)


def _body(element):
    """The lines of a DataArray between its tags."""
    return element.text.split("\n")[1:-1]


def _corners(g, r):
    x1, x2, x3, W, L = g.x, g.y, g.z, g.width, g.length
    s, d = r["s"], r["d"]
    return [(x1 - d[0] * W / 2 - s[0] * L / 2, x2 - d[1] * W / 2 - s[1] * L / 2, x3 - d[2] * W / 2 - s[2] * L / 2),
            (x1 - d[0] * W / 2 + s[0] * L / 2, x2 - d[1] * W / 2 + s[1] * L / 2, x3 - d[2] * W / 2 + s[2] * L / 2),
            (x1 + d[0] * W / 2 + s[0] * L / 2, x2 + d[1] * W / 2 + s[1] * L / 2, x3 + d[2] * W / 2 + s[2] * L / 2),
            (x1 + d[0] * W / 2 - s[0] * L / 2, x2 + d[1] * W / 2 - s[1] * L / 2, x3 + d[2] * W / 2 - s[2] * L / 2)]


@pytest.mark.parametrize("with_sig,with_sig0", [(True, False), (True, True), (False, False)])
def test_gmt_polygons(tmp_path, with_sig, with_sig0):
    segs = _segments()
    sig = _tensors(len(segs), 1) if with_sig else None
    sig0 = _tensors(len(segs), 2) if with_sig0 else None
    f = tmp_path / "rfaults-sigma-0001.xy"
    api.write_segments("gmt", segs, f, sig, sig0)
    want = []
    for k, g in enumerate(segs):
        r = _resolve(g, sig[k] if sig else None, sig0[k] if sig0 else None)
        want.append("> -Z" + _row([r["taus"], r["taun"], r["coulomb"], r["tstrike"], r["tdip"]]))
        # GMT order: east (x2), north (x1)
        want += [_row([c[1], c[0]]) for c in _corners(g, r)]
    assert f.read_text().splitlines() == want


def test_traction_rows(tmp_path):
    segs = _segments(5, seed=7)
    sig = _tensors(len(segs), 4)
    f = tmp_path / "rfaults-traction-0000.dat"
    api.write_segments("traction", segs, f, sig)
    lines = f.read_text().splitlines()
    assert lines[0] == "# position east, north, up, traction e, n, u, normal vector e, n, u"
    for k, g in enumerate(segs):
        r = _resolve(g, sig[k])
        assert lines[1 + k] == _row([g.y, g.x, -g.z, r["ts"][1], r["ts"][0], -r["ts"][2], r["n"][1], r["n"][0],
                                     -r["n"][2]])
        # the shear traction lies in the plane
        assert abs(sum(r["ts"][m] * r["n"][m] for m in range(3))) < 1e-12


def test_vtp_polydata(tmp_path):
    segs = _segments(3, seed=9)
    sig = _tensors(len(segs), 5)
    sig0 = _tensors(len(segs), 6)
    f = tmp_path / "rfaults-dsigma-0002.vtp"
    api.write_segments("vtp", segs, f, sig, sig0)
    text = f.read_text()
    assert text.startswith('<?xml version="1.0"?>\n<VTKFile type="PolyData" version="0.1">\n  <PolyData>\n')
    root = ET.fromstring(text.split("\n", 1)[1])
    pieces = root.find("PolyData").findall("Piece")
    assert len(pieces) == len(segs)
    for k, (g, piece) in enumerate(zip(segs, pieces)):
        r = _resolve(g, sig[k], sig0[k])
        assert piece.attrib == {"NumberOfPoints": "4", "NumberOfPolys": "1"}
        pts = piece.find("Points").find("DataArray")
        assert _body(pts) == [_row([v for c in _corners(g, r) for v in c])]
        arrays = {a.attrib["Name"]: a for a in piece.find("CellData").findall("DataArray")}
        assert _body(arrays["stress tensor"]) == [_row(r["sig"])]
        assert _body(arrays["traction vector"]) == [_row(r["t"])]
        assert _body(arrays["shear traction vector"]) == [_row([v]) for v in r["ts"]]
        for name, key in (("shear stress", "taus"), ("normal stress", "taun"), ("Coulomb stress", "coulomb"),
                          ("stress in strike direction", "tstrike"), ("stress in dip direction", "tdip")):
            assert _body(arrays[name]) == [_row([r[key]])]
        polys = {a.attrib["Name"]: a.text.strip() for a in piece.find("Polys").findall("DataArray")}
        assert polys == {"connectivity": "0 1 2 3", "offsets": "4"}


def test_coulomb_series(tmp_path):
    segs = _segments(3, seed=11)
    series = [(0.0, _tensors(3, 20)), (0.5, _tensors(3, 21)), (1.25, _tensors(3, 22))]
    for i, (t, sig) in enumerate(series):
        api.write_coulomb(segs, sig, t, tmp_path, isnew=(i == 0))
    for k, g in enumerate(segs):
        lines = (tmp_path / f"cfaults-sigma-{k + 1:04d}.txt").read_text().splitlines()
        assert lines[0] == "# center position (north, east, down): " + _row([g.x, g.y, g.z], 9, 2, 0)
        assert lines[1].split() == ["#", "t", "s11", "s12", "s13", "s22", "s23", "s33", "taus", "taud", "tau",
                                    "taun", "Coulomb"]
        assert len(lines) == 2 + len(series)
        for j, (t, sig) in enumerate(series):
            r = _resolve(g, sig[k])
            assert lines[2 + j] == _row([t, *r["sig"], r["tstrike"], r["tdip"], r["taus"], r["taun"],
                                         r["coulomb"]], 11, 3, 2)


def test_no_segments_writes_nothing(tmp_path):
    api.write_segments("gmt", [], tmp_path / "none.xy")
    assert not (tmp_path / "none.xy").exists()
