"""Observation planes and stress observation segments on the device: the
sinc-window sampler of monitorstressfield / monitorfield
(src/elastic3d.f90:3404-3762) against the oracle's restatement on the same
stress and gamma fields, the grids of exportplanestress
(src/export.f90:308-397), the segments' nearest-node stress
(src/export.f90:1364-1394) and the program's segment and plane files."""
import os
import subprocess

import numpy as np
import pytest
from scipy.io import netcdf_file

from relax_b200 import _lib, api
from relax_b200.api import Input, Relax
from relax_b200.config import relax_obsplane, relax_segment

from cases import linear_small, oracle_monitor_plane, powerlaw_small

pytestmark = pytest.mark.gpu

CLI = os.path.join(os.path.dirname(_lib.LIBPATH), "relax")
NAMES = ("s11", "s12", "s13", "s22", "s23", "s33")

PLANES = [
    relax_obsplane(x=3.0, y=-2.0, z=6.0, length=8.0, width=6.0, strike=0.0, dip=0.0),      # on the nodes
    relax_obsplane(x=0.3, y=1.7, z=5.2, length=12.3, width=9.1, strike=0.4, dip=0.7),
    relax_obsplane(x=-4.0, y=2.5, z=1.0, length=20.0, width=14.0, strike=-1.1, dip=1.2),   # partly above ground
    relax_obsplane(x=25.0, y=0.0, z=8.0, length=30.0, width=4.0, strike=1.4, dip=0.2),     # partly outside the box
]


@pytest.fixture(scope="module")
def stepped():
    sim = powerlaw_small(sx=64, sz=32)
    r = Relax(sim)
    r.coseismic()
    for _ in range(3):
        r.step()
    sig = r.field("sig")
    soa = np.stack([sig[n] for n in NAMES])
    gamma = np.ascontiguousarray(r.field("gamma")[..., :sim.sx1])
    yield sim, r, soa, gamma
    r.close()


def _check(got, want, nc):
    """Positions to rounding, samples within the single-precision rounding
    of the window sum (the device's and the host's sin may differ by an ulp
    in the weights)."""
    assert got.shape == want.shape[:2]
    np.testing.assert_allclose(got["x1"], want[..., 0], rtol=0, atol=1e-12)
    np.testing.assert_allclose(got["x2"], want[..., 1], rtol=0, atol=1e-12)
    np.testing.assert_allclose(got["x3"], want[..., 2], rtol=0, atol=1e-12)
    np.testing.assert_array_equal(got["lx"], want[..., 3])
    np.testing.assert_array_equal(got["lz"], want[..., 4])
    if nc == 1:
        vals = got["slip"][..., None]
    else:
        vals = np.stack([got["sig"][n] for n in NAMES], axis=-1).astype(np.float64)
    scale = max(np.abs(want[..., 5:]).max(), 1e-30)
    assert np.abs(vals - want[..., 5:]).max() <= 1e-6 * scale


@pytest.mark.parametrize("k", range(len(PLANES)))
def test_stress_sampler_matches_oracle(stepped, oracle32, k):
    sim, r, soa, _ = stepped
    assert np.abs(soa).max() > 0
    got = r.monitor_plane(PLANES[k], "sig")
    want = oracle_monitor_plane(oracle32.lib, soa, (sim.sx1, sim.sx2, sim.sx3h), (sim.dx1, sim.dx2, sim.dx3),
                                PLANES[k])
    _check(got, want, 6)


@pytest.mark.parametrize("k", [1, 2])
def test_gamma_sampler_matches_oracle(stepped, oracle32, k):
    sim, r, _, gamma = stepped
    got = r.monitor_plane(PLANES[k], "gamma", beta=0.1)
    want = oracle_monitor_plane(oracle32.lib, gamma, (sim.sx1, sim.sx2, sim.sx3h), (sim.dx1, sim.dx2, sim.dx3),
                                PLANES[k], beta=0.1)
    _check(got, want, 1)


def test_plane_stress_grids(stepped, tmp_path):
    sim, r, _, _ = stepped
    r.export_plane_stress(PLANES[:2], tmp_path, 7, origx=10.0, origy=-5.0)
    for k, op in enumerate(PLANES[:2]):
        p = r.monitor_plane(op, "sig")
        for n in NAMES:
            with netcdf_file(tmp_path / f"007.op{k + 1:03d}-{n}.grd", "r", mmap=False) as g:
                z = g.variables["z"][:].copy()
                x = g.variables["x"][:].copy()
                y = g.variables["y"][:].copy()
                title = g.title
            np.testing.assert_array_equal(z, p["sig"][n][:, ::-1])
            assert x[0] == p["lx"].min() and y[0] == -p["lz"].max()
            np.testing.assert_allclose(np.diff(x), sim.dx2)
            np.testing.assert_allclose(np.diff(y), sim.dx3)
            assert title == b"monitor tensor field"
    r.export_plane_stress(PLANES[1:2], tmp_path, 8, name="gamma")
    with netcdf_file(tmp_path / "008.s00001.estrain.grd", "r", mmap=False) as g:
        z = g.variables["z"][:].copy()
    np.testing.assert_array_equal(z, r.monitor_plane(PLANES[1], "gamma")["slip"][:, ::-1].astype(np.float32))


def test_segment_stress_reads_the_nearest_node(stepped):
    sim, r, soa, _ = stepped
    segs = [relax_segment(x=1.4, y=-2.6, z=3.5, length=4.0, width=2.0, strike=0.3, dip=0.5, friction=0.6),
            relax_segment(x=-20.0, y=11.0, z=0.2, length=4.0, width=2.0, strike=0.3, dip=0.5, friction=0.6)]
    sig = r.segment_stress(segs)
    for g, s in zip(segs, sig):
        i1, i2, i3 = api.shifted_index((g.x, g.y, g.z), (sim.sx1, sim.sx2, sim.sx3), (sim.dx1, sim.dx2, sim.dx3))
        assert tuple(getattr(s, n) for n in NAMES) == tuple(float(soa[m, i3, i2, i1]) for m in range(6))
    deep = relax_segment(x=0.0, y=0.0, z=sim.sx3h * sim.dx3 + 1.0, length=1.0, width=1.0, strike=0.0, dip=0.0,
                         friction=0.0)
    with pytest.raises(_lib.RelaxError, match="below the stored half"):
        r.segment_stress([deep])


def test_program_writes_plane_and_segment_files(tmp_path):
    sim = linear_small(sx=64, sz=32)
    sim.interval, sim.odt = 0.6, 0.3
    planes = [(2.0, -3.0, 0.0, 10.0, 8.0, 20.0, 70.0)]
    segs = [(1.0, 4.0, 2.0, 6.0, 3.0, 45.0, 60.0, 0.4), (-5.0, 0.0, 1.0, 4.0, 2.0, 0.0, 90.0, 0.6)]
    deck = sim.to_input(wdir=str(tmp_path), obsplanes=planes, segments=segs)
    r = subprocess.run([CLI], input=deck, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    inp = Input.parse(deck)
    op, sop = inp.obsplanes(), inp.segments()
    with Relax.from_input(inp) as rr:
        rr.coseismic()
        sig0 = rr.segment_stress(sop)
        p0 = rr.monitor_plane(op[0], "sig")
        outputs = []
        while True:
            rr.step()
            lg = rr.last_log
            if lg.i == 0:
                break
            if lg.output:
                outputs.append((lg.t, rr.segment_stress(sop), rr.monitor_plane(op[0], "sig")))
    assert len(outputs) >= 2
    with netcdf_file(tmp_path / "000.op001-s12.grd", "r", mmap=False) as g:
        np.testing.assert_array_equal(g.variables["z"][:], p0["sig"]["s12"][:, ::-1])
    oi = len(outputs)
    with netcdf_file(tmp_path / f"{oi:03d}.op001-s33.grd", "r", mmap=False) as g:
        np.testing.assert_array_equal(g.variables["z"][:], outputs[-1][2]["sig"]["s33"][:, ::-1])
    api.write_segments("gmt", sop, tmp_path / "want-dsigma.xy", outputs[-1][1], sig0)
    assert (tmp_path / f"rfaults-dsigma-{oi:04d}.xy").read_text() == (tmp_path / "want-dsigma.xy").read_text()
    api.write_segments("traction", sop, tmp_path / "want-traction.dat", sig0)
    assert (tmp_path / "rfaults-traction-0000.dat").read_text() == (tmp_path / "want-traction.dat").read_text()
    api.write_segments("vtp", sop, tmp_path / "want.vtp", outputs[0][1])
    assert (tmp_path / "rfaults-sigma-0001.vtp").read_text() == (tmp_path / "want.vtp").read_text()
    for k in range(len(sop)):
        lines = (tmp_path / f"cfaults-sigma-{k + 1:04d}.txt").read_text().splitlines()
        assert len(lines) == 2 + 1 + len(outputs)
        assert lines[-1].startswith(api.es_format(outputs[-1][0], 11, 3, 2))
