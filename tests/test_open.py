"""The reference's own open configuration: x ends with characteristic inflow
and outflow ghost planes (X_boundary_condition.cpp), one-sided MUSCL
stencils at the ends (Flux_X.cpp:139-216), no x halo and zero implicit halos
(Dual_time_stepping.cpp:204-246), sponge layers (:554-664), walls isothermal
only between them (Y_boundary_condition.cpp:114), end-plane metrics of the
first and last rank (Jacobian.cpp:110-157) and the buoyancy body force
(:831) -- the paths a single rank 0 of 1 takes.

The CPU restatement is pinned bit for bit to the reference built here as
rank 0 of 1 (fixture from tests/golden/make_golden.py --open, and fresh
builds), then the CUDA path is compared with it."""
import json
import os

import numpy as np
import pytest

from cgli_fu_flow_b200.channel import Channel
from tests.conftest import have_reference

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _fixture():
    with open(os.path.join(GOLDEN, "open_16x12x8.json")) as fh:
        return json.load(fh)


def _open_channel(nx=16, ny=12, nz=8, **kw):
    args = dict(x_open=True, nx_inlet=4, nx_outlet=4, buoyancy=True, twall_lo=343.0592)
    args.update(kw)
    return Channel(nx, ny, nz, **args)


def _sl(ch):
    """Interior cells plus the two x-end ghost planes the boundary updates."""
    return (slice(None), slice(2, ch.nx + 4), slice(2, ch.ny + 2), slice(2, ch.nz + 2))


def _digest(a):
    from tests.golden.make_golden import digest
    return digest(a)


@pytest.mark.parametrize("solver", ["lusgs", "dplur"])
def test_open_oracle_matches_reference_fixture(solver):
    from oracle.oracle import Oracle
    g = _fixture()
    ch = _open_channel(*g["cells"])
    o = Oracle(ch, inner_solver=solver)
    o.init()
    forces = [o.force]
    for n in range(g["steps"]):
        _, er = o.step(g["iters_per_step"])
        np.testing.assert_allclose(er, g[solver]["step_norms"][n], rtol=1e-13)
        forces.append(o.force)
    q = o.q()[_sl(ch)]
    assert _digest(q) == g[solver]["final_state"]
    assert forces == g[solver]["forces"]
    assert np.array_equal(q, np.load(os.path.join(GOLDEN, "open_16x12x8.npz"))[solver])


def test_open_ends_are_live():
    """The configuration exercises what it claims: the inlet ghost plane
    moves away from its quiescent start, the sponge terms are non-zero only
    in the inlet and outlet layers, and the heated wall's ghost row differs
    from the adiabatic copy only between the sponges."""
    from oracle.oracle import Oracle
    ch = _open_channel()
    o = Oracle(ch)
    o.init()
    g0 = o.array("U2_")[2].copy()
    o.step(3)
    assert not np.array_equal(o.array("U2_")[2, 2:ch.ny + 2, 2:ch.nz + 2], g0[2:ch.ny + 2, 2:ch.nz + 2])
    for n in ("halo_x", "bc_y", "bc_x", "bc_z", "flux_x", "flux_y", "flux_z", "viscous", "dts_residual"):
        o.call(n)
    sp = np.abs(o.array("Sponge2")[:, 2:ch.ny + 2, 2:ch.nz + 2]).max(axis=(1, 2))
    # the inlet layer is planes 3..nx_inlet+2, the outlet layer starts one
    # plane before the last nx_outlet (Dual_time_stepping.cpp:618: its first
    # plane has the small weight ((0.5)/nx_outlet)^3)
    layers = list(range(3, ch.nx_inlet + 3)) + list(range(ch.nx - ch.nx_outlet + 2, ch.nx + 3))
    assert all(sp[i] > 0 for i in layers)
    assert all(sp[i] == 0 for i in range(ch.nx + 6) if i not in layers)
    assert np.isfinite(o.array("MR1")[3:ch.nx + 3, 2:ch.ny + 2, 2:ch.nz + 2]).all()
    u1 = o.array("U1_")
    inside = [i for i in range(3, ch.nx + 3) if ch.nx_inlet + 2 < i < ch.nx - ch.nx_outlet + 3]
    outside = [i for i in range(3, ch.nx + 3) if i not in inside]
    for i in outside:
        assert np.array_equal(u1[i, 1, 2:ch.nz + 2], u1[i, 2, 2:ch.nz + 2])
    assert all(not np.array_equal(u1[i, 1, 2:ch.nz + 2], u1[i, 2, 2:ch.nz + 2]) for i in inside)


@pytest.mark.skipif(not have_reference(), reason="reference sources not present")
@pytest.mark.parametrize("solver", ["lusgs", "dplur"])
def test_open_oracle_matches_reference_second_grid(solver):
    """Another grid, unequal sponges, no buoyancy (the controlled uniform
    force), four OpenMP threads in the reference: bit-identical over two
    steps."""
    from oracle.oracle import Oracle
    from oracle.refrun import RefSolver
    ch = _open_channel(20, 10, 6, nx_inlet=3, nx_outlet=5, buoyancy=False)
    r = RefSolver(ch, threads=4, inner_solver=solver)
    r.init()
    o = Oracle(ch, inner_solver=solver)
    o.init()
    for _ in range(2):
        _, er_r = r.step(4)
        _, er_o = o.step(4)
        assert np.array_equal(r.q()[_sl(ch)], o.q()[_sl(ch)])
        np.testing.assert_allclose(er_r, er_o, rtol=1e-14)


@pytest.mark.skipif(not have_reference(), reason="reference sources not present")
@pytest.mark.parametrize("solver", ["lusgs", "dplur"])
@pytest.mark.parametrize("dims,sponges", [((8, 6, 4), (2, 2)), ((13, 7, 9), (3, 4))])
def test_open_oracle_matches_reference_at_edge_sizes(solver, dims, sponges):
    """The smallest y and z extents the library accepts, with sponges and a
    heated section a few planes long, and an odd-sized grid, buoyancy on:
    bit-identical over two steps."""
    from oracle.oracle import Oracle
    from oracle.refrun import RefSolver
    ch = _open_channel(*dims, nx_inlet=sponges[0], nx_outlet=sponges[1], buoyancy=True)
    r = RefSolver(ch, threads=3, inner_solver=solver)
    r.init()
    o = Oracle(ch, inner_solver=solver)
    o.init()
    for _ in range(2):
        _, er_r = r.step(4)
        _, er_o = o.step(4)
        assert np.array_equal(r.q()[_sl(ch)], o.q()[_sl(ch)])
        np.testing.assert_allclose(er_r, er_o, rtol=1e-14)


# ------------------------------------------------------------------ GPU
# Tolerances as for the periodic channel: one routine ~1e-13 of the array's
# scale (fused multiply-adds and reciprocals), whole steps by relative L2.

STAGE_TOL = 1e-12
STEP_TOL = 1e-10


def _rel_max(a, b):
    m = np.isfinite(a) & np.isfinite(b)
    return np.abs(a[m] - b[m]).max() / max(np.abs(b[m]).max(), 1e-300)


def _rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _pair(ch, precision=0, solver="lusgs"):
    from cgli_fu_flow_b200 import build
    from cgli_fu_flow_b200.solver import Solver
    from oracle.oracle import Oracle
    build.build()
    g = Solver(ch, precision)
    g.init()
    o = Oracle(ch, inner_solver=solver)
    o.init()
    return g, o


@pytest.mark.gpu
def test_open_metrics_and_initial_state_match_oracle():
    ch = _open_channel()
    g, o = _pair(ch)
    for n in ("J", "xidx", "etdy", "ztdx", "ztdy", "ztdz", "J_u", "etdy_v", "J_v", "J_w"):
        assert np.array_equal(g.get(n), o.array(n)), n
    for n in ("U1_", "U2_", "U5_", "U1", "U1q"):
        a, b = g.get(n), o.array(n)
        assert np.array_equal(np.isfinite(a), np.isfinite(b)), n
        assert np.array_equal(a[np.isfinite(a)], b[np.isfinite(b)]), n


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(16, 12, 8), (37, 20, 34)])
def test_open_routines_match_oracle(dims):
    """Each entry point of the open configuration after two steps (a
    developed state), then one routine-by-routine inner iteration."""
    ch = _open_channel(*dims, nx_inlet=4, nx_outlet=6)
    g, o = _pair(ch)
    for _ in range(2):
        g.step(4)
        o.step(4)
    X = (slice(2, ch.nx + 4), slice(2, ch.ny + 2), slice(2, ch.nz + 2))
    for v in range(1, 6):
        assert _rel_l2(g.get(f"U{v}_")[X], o.array(f"U{v}_")[X]) <= 1e-11, v
    g.set_state(*[np.stack([o.array(f"U{v}{s}") for v in range(1, 6)]) for s in ("_", "", "q")])
    g.halo_x(); g.y_boundary_condition(); g.x_boundary_condition(); g.z_boundary_condition()
    for n in ("halo_x", "bc_y", "bc_x", "bc_z"):
        o.call(n)
    ring = (slice(2, ch.nx + 4), slice(1, ch.ny + 3), slice(1, ch.nz + 3))
    for v in range(1, 6):
        assert _rel_max(g.get(f"U{v}_")[ring], o.array(f"U{v}_")[ring]) <= STAGE_TOL, ("bc", v)
    g.flux_x(); o.call("flux_x")
    fx = (slice(2, ch.nx + 3), slice(1, ch.ny + 1), slice(1, ch.nz + 1))
    for v in range(1, 6):
        assert _rel_max(g.get(f"inFx{v}")[fx], o.array(f"inFx{v}")[fx]) <= STAGE_TOL, ("fx", v)
    g.flux_y(); g.flux_z(); g.viscous_terms()
    for n in ("flux_y", "flux_z", "viscous"):
        o.call(n)
    cell = (slice(3, ch.nx + 3), slice(2, ch.ny + 2), slice(2, ch.nz + 2))
    for v in range(2, 6):
        assert _rel_max(g.get(f"vF{v}")[cell], o.array(f"vF{v}")[cell]) <= STAGE_TOL, ("vF", v)
    er_g = g.dual_time_stepping()
    o.call("dts_residual"); o.call("sweeps")
    er_o = o.update()
    # the sponge's energy term E J - 253250 (Dual_time_stepping.cpp:596, :655)
    # cancels about four digits, so MR carries ten times the stage bar
    for v in range(1, 6):
        assert _rel_max(g.get(f"MR{v}")[cell], o.array(f"MR{v}")[cell]) <= 10 * STAGE_TOL, ("MR", v)
        assert _rel_max(g.get(f"U{v}_")[cell], o.array(f"U{v}_")[cell]) <= STAGE_TOL, ("U_", v)
    np.testing.assert_allclose(er_g, er_o, rtol=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["lusgs", "dplur"])
def test_open_steps_match_reference_fixture(solver):
    """Three steps of ten inner iterations through cgli_step (the fused path
    for LU-SGS) against the reference run as rank 0 of 1."""
    f = _fixture()
    ch = _open_channel(*f["cells"])
    g, _ = _pair(ch)
    g.set_inner_solver(solver)
    for _ in range(f["steps"]):
        g.step(f["iters_per_step"])
    ref = np.load(os.path.join(GOLDEN, "open_16x12x8.npz"))[solver]
    q = g.q()[_sl(ch)]
    for v in range(5):
        assert _rel_l2(q[v], ref[v]) <= STEP_TOL, v


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["lusgs", "dplur"])
def test_open_ten_steps_match_oracle(solver):
    """A grid with several sweep tiles and relaxation tiles, unequal sponges,
    buoyancy, the stopping rule deciding the iteration counts on both
    sides."""
    ch = _open_channel(40, 24, 36, nx_inlet=5, nx_outlet=7)
    g, o = _pair(ch, solver=solver)
    g.set_inner_solver(solver)
    for s in range(10):
        it_g, _ = g.step(None, drop=1e-2, cap=10)
        it_o, _ = o.step(None, drop=1e-2, cap=10)
        assert it_g == it_o, s
    q, r = g.q()[_sl(ch)], o.q()[_sl(ch)]
    for v in range(5):
        assert _rel_l2(q[v], r[v]) <= STEP_TOL, v


@pytest.mark.gpu
def test_open_mixed_precision_within_1e6():
    from cgli_fu_flow_b200.solver import MIXED
    ch = _open_channel(32, 16, 32)
    g, o = _pair(ch, precision=MIXED)
    for _ in range(10):
        g.step(8)
        o.step(8)
    q, r = g.q()[_sl(ch)], o.q()[_sl(ch)]
    errs = [_rel_l2(q[v], r[v]) for v in range(5)]
    print("open, mixed precision, relative L2 per variable after 10 steps:", errs)
    assert max(errs) <= 1e-6


@pytest.mark.gpu
def test_open_parameter_errors():
    from cgli_fu_flow_b200 import build
    from cgli_fu_flow_b200.solver import CgliError, Solver
    build.build()
    with pytest.raises(CgliError):
        Solver(Channel(16, 12, 8, nx_inlet=2))                  # sponge on a periodic slab
    with pytest.raises(CgliError):
        Solver(_open_channel(16, 12, 8, nx_inlet=10, nx_outlet=8))   # layers longer than the slab
