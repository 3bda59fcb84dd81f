"""DP-LUR inner solver (DPLUSGS.cpp): the CPU restatement against the
reference's own routine, then the CUDA path against the restatement.

DPLUSGS.cpp replaces the two symmetric LU-SGS sweeps of Dual_time_stepping
by four Jacobi relaxations of the same split-Jacobian operator; the
reference's driver leaves its call commented out (main.cpp:268-284).  The
reference build used for pinning fixes the routine's unassigned j_ / k_ loop
indices (oracle/build_ref.py) so that its upper y / z terms read the
neighbours whose state they use."""
import json
import os

import numpy as np
import pytest

from cgli_fu_flow_b200.channel import Channel
from tests.conftest import have_reference

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _fixture():
    with open(os.path.join(GOLDEN, "dplur_channel_8x12x8.json")) as fh:
        return json.load(fh)


def _regions(ch):
    from tests.golden.make_golden import regions
    return regions(ch)


def _digest(a):
    from tests.golden.make_golden import digest
    return digest(a)


def test_dplur_oracle_first_iteration_bit_exact():
    from oracle.oracle import Oracle
    g = _fixture()
    ch = Channel(*g["cells"])
    o = Oracle(ch, inner_solver="dplur")
    o.init()
    er = o.inner_iteration()
    reg = _regions(ch)
    for n, h in g["first"].items():
        assert _digest(o.array(n)[reg["cell"]]) == h, n
    np.testing.assert_allclose(er, g["first_norms"], rtol=1e-13)


def test_dplur_oracle_three_steps_bit_exact():
    from oracle.oracle import Oracle
    g = _fixture()
    ch = Channel(*g["cells"])
    o = Oracle(ch, inner_solver="dplur")
    o.init()
    forces = [o.force]
    for n in range(g["steps"]):
        _, er = o.step(g["iters_per_step"])
        np.testing.assert_allclose(er, g["step_norms"][n], rtol=1e-13)
        forces.append(o.force)
    reg = _regions(ch)
    q = o.q()[(slice(None),) + reg["cell"]]
    assert _digest(q) == g["final_state"]
    assert forces == g["forces"]
    assert np.array_equal(q, np.load(os.path.join(GOLDEN, "dplur_channel_8x12x8.npz"))["q"])


def test_dplur_differs_from_lusgs():
    """The two inner solvers are different iterations: after one inner
    iteration from the same state the updates differ, and the first DP-LUR
    norm is the pressure increment, not the density increment."""
    from oracle.oracle import Oracle
    ch = Channel(8, 12, 8)
    a, b = Oracle(ch), Oracle(ch, inner_solver="dplur")
    a.init(); b.init()
    ea, eb = a.inner_iteration(), b.inner_iteration()
    assert not np.array_equal(a.q(), b.q())
    assert eb[0] > 1e3 * ea[0]


@pytest.mark.skipif(not have_reference(), reason="reference sources not present")
def test_dplur_oracle_matches_reference_second_grid():
    """A non-cubic grid with four OpenMP threads in the reference: two steps
    stay bit-identical, and so do the norms (the reference divides by its
    global 3 Nx)."""
    from oracle.oracle import Oracle
    from oracle.refrun import RefSolver
    ch = Channel(6, 10, 5)
    r = RefSolver(ch, threads=4, inner_solver="dplur")
    r.init()
    o = Oracle(ch, inner_solver="dplur")
    o.init()
    sl = (slice(None),) + _regions(ch)["cell"]
    for _ in range(2):
        _, er_r = r.step(4)
        _, er_o = o.step(4)
        assert np.array_equal(r.q()[sl], o.q()[sl])
        np.testing.assert_allclose(3.0 * er_r, er_o, rtol=1e-14)


@pytest.mark.skipif(not have_reference(), reason="reference sources not present")
@pytest.mark.parametrize("dims,threads", [((3, 6, 4), 2), ((11, 7, 9), 3)])
def test_dplur_oracle_matches_reference_at_edge_sizes(dims, threads):
    """The smallest accepted grid and an odd-sized one: the relaxation's
    neighbour terms at every wall and end row, bit-identical over two
    steps, norms up to the reference's global 3 Nx."""
    from oracle.oracle import Oracle
    from oracle.refrun import RefSolver
    ch = Channel(*dims)
    r = RefSolver(ch, threads=threads, inner_solver="dplur")
    r.init()
    o = Oracle(ch, inner_solver="dplur")
    o.init()
    sl = (slice(None),) + _regions(ch)["cell"]
    for _ in range(2):
        _, er_r = r.step(4)
        _, er_o = o.step(4)
        assert np.array_equal(r.q()[sl], o.q()[sl])
        np.testing.assert_allclose(3.0 * np.asarray(er_r), er_o, rtol=1e-14)


@pytest.mark.skipif(not have_reference(), reason="reference sources not present")
def test_dplur_oracle_matches_reference_wavy_grid():
    from oracle.oracle import Oracle
    from oracle.refrun import RefSolver
    ch = Channel(8, 12, 8, wavy=True)
    r = RefSolver(ch, threads=2, inner_solver="dplur")
    r.init()
    o = Oracle(ch, curved_walls=False, inner_solver="dplur")
    o.init()
    sl = (slice(None),) + _regions(ch)["cell"]
    for _ in range(2):
        r.step(4)
        o.step(4)
        assert np.array_equal(r.q()[sl], o.q()[sl])


# ------------------------------------------------------------------ GPU
# Tolerances as for the LU-SGS path: the relaxation kernel evaluates the
# same expressions with reciprocals and fused multiply-adds, so one call
# agrees to ~1e-13 of each array's scale; whole steps by relative L2 per
# conserved variable.

STAGE_TOL = 1e-12
STEP_TOL = 1e-10


def _rel_max(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _pair(ch, **kw):
    from cgli_fu_flow_b200 import build
    from cgli_fu_flow_b200.solver import Solver
    from oracle.oracle import Oracle
    build.build()
    g = Solver(ch)
    g.init()
    o = Oracle(ch, inner_solver="dplur", **kw)
    o.init()
    return g, o


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(8, 12, 8), (40, 36, 62)])
def test_dplusgs_entry_matches_oracle(dims):
    """cgli_dplusgs after the granular residual entry points: the relaxed
    increment NR, the updated state and the norms.  The second grid has
    ragged relaxation tiles in j and k and two x chunks."""
    ch = Channel(*dims)
    g, o = _pair(ch)
    for fn in ("halo_x", "y_boundary_condition", "z_boundary_condition", "flux_x", "flux_y", "flux_z",
               "viscous_terms"):
        getattr(g, fn)()
    for n in ("halo_x", "bc_y", "bc_z", "flux_x", "flux_y", "flux_z", "viscous", "dts_residual", "dplur_sweeps"):
        o.call(n)
    er_o = np.zeros(5)
    o.L.or_dplur_update(o.s, er_o.ctypes.data)
    er_g = g.dplusgs()
    reg = _regions(ch)["cell"]
    for v in range(1, 6):
        assert _rel_max(g.get(f"NR{v}")[reg], o.array(f"NR{v}")[reg]) <= STAGE_TOL, v
        assert _rel_max(g.get(f"U{v}_")[reg], o.array(f"U{v}_")[reg]) <= STAGE_TOL, v
    np.testing.assert_allclose(er_g, er_o, rtol=1e-9)


@pytest.mark.gpu
def test_dplur_steps_match_reference_fixture():
    """Three steps of ten inner iterations through cgli_step with the DP-LUR
    solver against the reference's DPLUSGS.cpp final state."""
    g0 = _fixture()
    ch = Channel(*g0["cells"])
    g, _ = _pair(ch)
    g.set_inner_solver("dplur")
    for _ in range(g0["steps"]):
        it, _er = g.step(g0["iters_per_step"])
        assert it == g0["iters_per_step"]
    ref = np.load(os.path.join(GOLDEN, "dplur_channel_8x12x8.npz"))["q"]
    q = g.q()[(slice(None),) + _regions(ch)["cell"]]
    for v in range(5):
        assert _rel_l2(q[v], ref[v]) <= STEP_TOL, v


@pytest.mark.gpu
def test_dplur_twenty_steps_match_oracle():
    """Twenty steps on a grid with several relaxation tiles and x chunks,
    with the stopping rule of main.cpp:287-304 deciding the iteration
    counts on both sides."""
    ch = Channel(34, 20, 40)
    g, o = _pair(ch)
    g.set_inner_solver("dplur")
    for s in range(20):
        it_g, _ = g.step(None, drop=1e-2, cap=12)
        it_o, _ = o.step(None, drop=1e-2, cap=12)
        assert it_g == it_o, s
    sl = (slice(None),) + _regions(ch)["cell"]
    for v in range(5):
        assert _rel_l2(g.q()[sl][v], o.q()[sl][v]) <= STEP_TOL, v


@pytest.mark.gpu
def test_dplur_wavy_wall_matches_oracle():
    """General metrics (every metric term live): five steps."""
    ch = Channel(16, 16, 32, wavy=True, wave=0.01)
    g, o = _pair(ch)
    g.set_inner_solver("dplur")
    for _ in range(5):
        g.step(6)
        o.step(6)
    sl = (slice(None),) + _regions(ch)["cell"]
    for v in range(5):
        assert _rel_l2(g.q()[sl][v], o.q()[sl][v]) <= STEP_TOL, v


@pytest.mark.gpu
def test_inner_solver_switch_and_errors():
    """Switching back to LU-SGS gives the LU-SGS result again; DP-LUR is
    refused in mixed precision and an unknown solver is refused."""
    from cgli_fu_flow_b200 import build
    from cgli_fu_flow_b200.solver import CgliError, Solver
    from oracle.oracle import Oracle
    build.build()
    ch = Channel(8, 12, 8)
    g = Solver(ch)
    g.init()
    g.set_inner_solver("dplur")
    g.set_inner_solver("lusgs")
    o = Oracle(ch)
    o.init()
    g.step(5)
    o.step(5)
    sl = (slice(None),) + _regions(ch)["cell"]
    assert _rel_l2(g.q()[sl][0], o.q()[sl][0]) <= STEP_TOL
    with pytest.raises(CgliError):
        g._rc(g.L.cgli_set_inner_solver(g.h, 7))
    m = Solver(ch, 1)
    m.init()
    with pytest.raises(CgliError):
        m.set_inner_solver("dplur")
    er = (__import__("ctypes").c_double * 5)()
    with pytest.raises(CgliError):
        m._rc(m.L.cgli_dplusgs(m.h, er))
