"""The C++ host driver (cgli_fu_flow_b200/csrc/driver/cgli_run.cpp): the
reference's step loop of main.cpp on the C ABI, reading and writing the
reference's restart layout."""
import os
import subprocess

import numpy as np
import pytest

from cgli_fu_flow_b200 import build
from cgli_fu_flow_b200 import channel as C


def _driver():
    build.build()
    return build.DRIVER


def test_driver_builds_and_prints_usage():
    r = subprocess.run([_driver(), "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.startswith("usage: cgli_run")


def test_driver_rejects_incomplete_command_line():
    r = subprocess.run([_driver(), "--nx", "8"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "usage" in r.stderr


def test_driver_reports_library_errors(tmp_path):
    """A call the library refuses (here a grid below the smallest accepted
    one; on a machine without a GPU the context cannot be created at all)
    ends the driver with status 2 and the library's message."""
    r = subprocess.run([_driver(), "--nx", "2", "--ny", "4", "--nz", "4", "--dxi", "1e-3", "--det", "0.25",
                        "--dzt", "1e-3", "--dt", "1e-6", "--e", "0.1", "--mu", "1.85e-5", "--pr", "0.72",
                        "--high", "1e-3", "--stretch", "2.0", "--initial", str(tmp_path / "none.bin"),
                        "--steps", "1"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2, (r.returncode, r.stderr)
    assert r.stderr.startswith("cgli_run: cgli_create: ") and len(r.stderr.strip()) > len("cgli_run: cgli_create:")


def _args(ch, initial, output, steps, extra=()):
    f = lambda x: repr(float(x))
    return [_driver(), "--nx", str(ch.nx), "--ny", str(ch.ny), "--nz", str(ch.nz), "--dxi", f(ch.dxi),
            "--det", f(ch.det), "--dzt", f(ch.dzt), "--dt", f(ch.dt), "--e", f(C.PRECOND_EPS), "--mu", f(C.MU0),
            "--pr", f(C.PR), "--high", f(ch.high), "--stretch", f(C.STRETCH), "--twall-lo", f(ch.twall_lo),
            "--twall-hi", f(ch.twall_hi), "--initial", initial, "--output", output, "--steps", str(steps),
            "--target-flux", f(ch.target_flux), "--force-lam", f(ch.force_lam), *extra]


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["lusgs", "dplur"])
def test_driver_matches_python_solver(tmp_path, solver):
    """Three steps with the stopping rule and the mass-flux controller through
    the C++ driver and through the Python wrapper of the same library: the
    same iteration counts, forces and output file, byte for byte."""
    from cgli_fu_flow_b200.solver import Solver
    ch = C.Channel(16, 12, 8)
    q = ch.initial_conserved()
    init, out_d, out_p = (str(tmp_path / n) for n in ("initial.bin", "driver.bin", "python.bin"))
    ch.write_restart(init, q, q, ranks=1, rank=0)
    extra = ["--drop", "1e-2", "--cap", "8"] + (["--dplur"] if solver == "dplur" else [])
    r = subprocess.run(_args(ch, init, out_d, 3, extra), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [ln.split("\t") for ln in r.stdout.strip().splitlines()]
    g = Solver(ch)
    g.read_restart(init, history=False)
    g.set_inner_solver(solver)
    for n in range(3):
        it, _ = g.step(None, drop=1e-2, cap=8)
        assert int(lines[n][1]) == it
        assert float(lines[n][7]) == g.force
    g.write_restart(out_p, history=False)
    with open(out_d, "rb") as a, open(out_p, "rb") as b:
        assert a.read() == b.read()
