"""Restart files in the reference's format (Output.cpp:187-284 writes them,
Initial_condition.cpp:111-236 reads them) and the history sidecar."""
import os

import numpy as np
import pytest

from cgli_fu_flow_b200.channel import Channel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from cgli_fu_flow_b200 import build, solver
    build.build()
    return solver.load_library()


def _interior(ch):
    return np.s_[3:ch.nx + 3, 2:ch.ny + 2, 2:ch.nz + 2]


def _q(g, suffix):
    ch = g.ch
    J = g.get("J")[_interior(ch)]
    return np.stack([g.get(f"U{v}{suffix}")[_interior(ch)] * J for v in range(1, 6)])


def test_restart_file_has_the_reference_layout(lib, tmp_path):
    """Byte for byte the file the reference's writer lays out for the same
    Q^n = U*J and Q^(n-1) = Uq*J (one slab = the whole domain)."""
    from cgli_fu_flow_b200.solver import Solver
    ch = Channel(10, 12, 8)
    g = Solver(ch)
    g.init()
    for _ in range(3):
        g.step(6)
    p, want = str(tmp_path / "LES00003.bin"), str(tmp_path / "expected.bin")
    g.write_restart(p, history=False)
    ch.write_restart(want, _q(g, ""), _q(g, "q"), ranks=1, rank=0)
    assert open(p, "rb").read() == open(want, "rb").read()


def test_restart_round_trip_continues_the_run(lib, tmp_path):
    """A second context started from the file and its history sidecar
    continues the run bit for bit (same iteration counts under the
    running-maximum rule, identical states): the sidecar keeps the raw
    levels with their ghost cells, whose lagged wall rows in the x-ghost
    planes the reference-format file cannot hold."""
    from cgli_fu_flow_b200.solver import Solver
    ch = Channel(10, 12, 8)
    a = Solver(ch)
    a.init()
    a.set_predictor(1)
    for _ in range(3):
        a.step(None, 1e-2, 20)
    p = str(tmp_path / "LES00003.bin")
    a.write_restart(p)
    b = Solver(ch)
    b.read_restart(p, ctrl=a.ctrl)
    assert b.force == a.force
    b.set_predictor(1)
    for _ in range(2):
        ia, _ = a.step(None, 1e-2, 20)
        ib, _ = b.step(None, 1e-2, 20)
        assert ia == ib
    qa, qb = a.q()[(slice(None),) + _interior(ch)], b.q()[(slice(None),) + _interior(ch)]
    assert np.array_equal(qa, qb)


def _ref_present(ch):
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    return os.path.exists(os.path.join(here, "oracle", "_ref", ch.name, "libref.so"))


@pytest.mark.skipif(not _ref_present(Channel(8, 12, 8)), reason="reference build for 8x12x8 not present")
def test_reference_reads_the_gpu_restart(lib, tmp_path):
    """The GPU writes its slab as the middle one of a three-slab file; the
    reference's own reader (Initial_condition.cpp) and the GPU reader both
    load it and continue the run together (both start from the file's
    interior values with the reader's ghost initialisation)."""
    from cgli_fu_flow_b200.solver import Solver
    from oracle.refrun import RefSolver
    ch = Channel(8, 12, 8)
    g = Solver(ch)
    g.init()
    for _ in range(2):
        g.step(6)
    p = str(tmp_path / "LES00002.bin")
    g.write_restart(p, global_nx=3 * ch.nx, x_offset=ch.nx, history=False)
    r = RefSolver(ch, threads=1, build=False)
    r.force, r.ctrl = g.force, dict(g.ctrl)
    r.load(p)
    sl = _interior(ch)
    for v in range(1, 6):
        for sfx in ("", "q"):
            a, b = g.get(f"U{v}{sfx}")[sl], r.array(f"U{v}{sfx}")[sl]
            assert np.abs(a - b).max() <= 4e-16 * np.abs(a).max(), (v, sfx)
    g2 = Solver(ch)
    g2.read_restart(p, global_nx=3 * ch.nx, x_offset=ch.nx, history=False, ctrl=g.ctrl)
    g2.set_force(g.force)
    for v in range(1, 6):
        assert np.array_equal(g2.get(f"U{v}")[sl], r.array(f"U{v}")[sl])
    g2.step(6)
    r.step(6)
    qg, qr = g2.q()[(slice(None),) + sl], r.q()[(slice(None),) + sl]
    for v in range(5):
        assert np.linalg.norm(qg[v] - qr[v]) <= 1e-10 * np.linalg.norm(qr[v]), v
