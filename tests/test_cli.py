"""The relax command-line program (src/relax.f90 with the options of
src/input.f90:64-185) without a GPU: help, version, the echo of a dry run
and input errors."""
import os
import subprocess

import pytest

from relax_b200 import _lib

from cases import linear_small

CLI = os.path.join(os.path.dirname(_lib.LIBPATH), "relax")


def _run(args, stdin=None, cwd=None):
    return subprocess.run([CLI] + args, input=stdin, capture_output=True, text=True, timeout=60, cwd=cwd)


@pytest.fixture(scope="module", autouse=True)
def built():
    if not os.path.exists(CLI):
        _lib.build()
    assert os.path.exists(CLI)


def test_help_and_version():
    r = _run(["--help"])
    assert r.returncode == 0
    assert r.stdout.startswith("usage:")
    assert "--with-transient        include the transient rheology" in r.stdout
    r = _run(["--version"])
    assert r.returncode == 0 and r.stdout.startswith("relax version")


def test_dry_run_reads_stdin_and_echoes(tmp_path):
    sim = linear_small()
    deck = sim.to_input(wdir=str(tmp_path), points=[("GPS1", 1.0, 2.0, 0.0)])
    r = _run(["--dry-run"], stdin=deck)
    assert r.returncode == 0, r.stderr
    out = r.stdout.splitlines()
    assert out[-1] == "dry run: abort calculation"
    assert "   64   64   32" in out
    assert "001 GPS1  1.00E+0  2.00E+0  0.00E+0" in out
    assert (tmp_path / "opts.dat").read_text().splitlines() == [
        "# x1(north) x2(east) x3(down) name(4-char)", "  1.0000E+0  2.0000E+0  0.0000E+0 GPS1"]


def test_input_file_argument_and_errors(tmp_path):
    sim = linear_small()
    deck = sim.to_input(wdir=str(tmp_path))
    path = tmp_path / "relax.inp"
    path.write_text(deck)
    assert _run(["--dry-run", str(path)]).returncode == 0
    bad = deck.replace("1 6.0 1.0 0.0", "2 6.0 1.0 0.0")
    r = _run(["--dry-run"], stdin=bad)
    assert r.returncode == 1
    assert "index misfit" in r.stderr
    r = _run(["--dry-run"], stdin=deck.replace(str(tmp_path), str(tmp_path / "missing")))
    assert r.returncode == 1 and "unable to access" in r.stderr
