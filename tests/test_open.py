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
