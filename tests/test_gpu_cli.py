"""The relax program end to end on the GPU, against the same deck run
through the Python API (the same library calls, so the log lines and the
files agree exactly), and the velocity / postseismic-displacement tracking
of relax_track_relaxation (src/relax.f90:829-850) against differences of
the displacement field."""
import os
import subprocess

import numpy as np
import pytest
from scipy.io import netcdf_file

from relax_b200 import _lib, api
from relax_b200.api import Input, Relax

from cases import linear_small

pytestmark = pytest.mark.gpu

CLI = os.path.join(os.path.dirname(_lib.LIBPATH), "relax")


def _grd(path):
    with netcdf_file(path, "r", mmap=False) as f:
        return f.variables["z"][:].copy()


def test_tracking_matches_displacement_differences():
    sim = linear_small(sx=64, sz=32, steps=4)
    with Relax(sim) as r:
        r.track_relaxation(vel_planes=sim.sx3h, ur_planes=4, inter_i3=6)
        r.coseismic()
        u0 = r.field("u")[..., :sim.sx1].astype(np.float64)
        prev = u0
        for _ in range(4):
            lg = r.step()
            if lg[0] == 0:
                break
            dt = lg[1]
            u = r.field("u")[..., :sim.sx1].astype(np.float64)
            scale = np.abs(u).max()
            for i3 in (0, 3, 9):
                np.testing.assert_allclose(r.plane("v", i3), (u[:, i3] - prev[:, i3]) / dt, rtol=0,
                                           atol=2e-6 * scale / dt)
            for i3 in (0, 2, 6):
                np.testing.assert_allclose(r.plane("ur", i3), u[:, i3] - u0[:, i3], rtol=0, atol=4e-6 * scale)
            prev = u
        with pytest.raises(_lib.RelaxError):
            r.plane("ur", 5)        # neither in the kept planes nor the slice


def test_cli_run_matches_the_api(tmp_path):
    sim = linear_small(sx=64, sz=32)
    sim.interval, sim.odt = 2.0, 0.5          # Dt = tm/10 = 0.1, outputs every 0.5
    pts = [("GPS1", 1.0, 2.0, 0.0), ("GPS2", -6.0, 4.0, 0.0)]
    cli_dir, api_dir = tmp_path / "cli", tmp_path / "api"
    cli_dir.mkdir()
    api_dir.mkdir()
    deck = sim.to_input(wdir=str(cli_dir), oz=0.0, ozs=2.0, points=pts)
    r = subprocess.run([CLI], input=deck, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.splitlines()
    start = lines.index("# event 001")
    log_lines = [l for l in lines[start + 2:] if not l.startswith(("#", "coseismic", " I "))]
    # the same deck through the API
    inp = Input.parse(sim.to_input(wdir=str(api_dir), oz=0.0, ozs=2.0, points=pts))
    info = inp.info
    want = []
    with Relax.from_input(inp) as rr:
        rr.track_relaxation(vel_planes=sim.sx3h, ur_planes=0, inter_i3=0)
        rr.coseismic()
        want.append(api.format_log(rr.last_log, sim.interval))
        oi = 1
        while True:
            rr.step()
            lg = rr.last_log
            if lg.i == 0:
                break
            want.append(api.format_log(lg, sim.interval))
            t_last = lg.t
            if lg.output:
                last_oi = oi
                oi += 1
        u = rr.plane("u", 0)
        ur = rr.plane("ur", 0)
        v = rr.plane("v", 0)
        sig = rr.plane("sig", 2)
        rr.export_points(np.ctypeslib.as_array(info.pts, (3 * info.npts,)), [n for n, *_ in pts], t_last,
                         api_dir, isnew=True)
    assert log_lines == want
    assert oi > 2
    tag = f"{last_oi:03d}"
    np.testing.assert_array_equal(_grd(cli_dir / f"{tag}-north.grd"), np.fft.fftshift(u[0].T))
    np.testing.assert_array_equal(_grd(cli_dir / f"{tag}-up.grd"), -np.fft.fftshift(u[2].T))
    np.testing.assert_array_equal(_grd(cli_dir / f"{tag}-relax-east.grd"), np.fft.fftshift(ur[1].T))
    np.testing.assert_array_equal(_grd(cli_dir / f"{tag}-s23.grd"), np.fft.fftshift(sig[4].T))
    assert (cli_dir / f"vel-{tag}.vtk").exists() and (cli_dir / f"disp-{tag}.vtk").exists()
    assert (cli_dir / "disp-000.vtk").exists() and (cli_dir / "sigma-0000.vtk").exists()
    # time report: the coseismic line and one per output
    assert len((cli_dir / "time.txt").read_text().splitlines()) == oi
    # the point series: header, t = 0 and one row per step; the last row as the API writes it
    for n, *_ in pts:
        rows = (cli_dir / f"{n}.ned").read_text().splitlines()
        assert len(rows) == 1 + len(want)
        assert rows[-1] == (api_dir / f"{n}.ned").read_text().splitlines()[-1]
    # the velocity of the last step, exported at stride 8 x 8 x 16
    raw = (cli_dir / f"vel-{tag}.vtk").read_bytes().split(b"\n", 9)[9]
    data = np.frombuffer(raw, ">f4").reshape(-1, 3)
    i1 = [(sim.sx1 + k) % sim.sx1 for k in range(-sim.sx1 // 2, sim.sx1 // 2, 8)]
    i2 = [(sim.sx2 + k) % sim.sx2 for k in range(-sim.sx2 // 2, sim.sx2 // 2, 8)]
    first_plane = np.stack([v[c][np.ix_(i2, i1)].ravel() for c in range(3)], axis=1)
    np.testing.assert_array_equal(data[:first_plane.shape[0]], first_plane)

