"""The CPU oracle is pinned to the reference: it must reproduce, bit for
bit, the fixtures recorded from the reference's own compiled routines
(tests/golden/make_golden.py), and -- where the reference sources are
present -- a fresh run of the reference built here."""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from cgli_fu_flow_b200.channel import Channel
from tests.conftest import have_reference

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def load(name):
    with open(os.path.join(GOLDEN, name + ".json")) as fh:
        return json.load(fh)


@pytest.fixture(scope="module")
def golden():
    return load("channel_8x12x8")


def regions(ch):
    from tests.golden.make_golden import regions as r
    return r(ch)


def test_oracle_metrics_match_reference_fixture(golden):
    from oracle.oracle import Oracle
    ch = Channel(*golden["cells"])
    o = Oracle(ch)
    reg = regions(ch)
    for name, h in golden["metrics"].items():
        assert digest(o.array(name)[reg["metric"]]) == h, name


def test_oracle_first_iteration_stages_bit_exact(golden):
    from oracle.oracle import Oracle
    from tests.golden.make_golden import STAGES, STAGE_REGION
    ch = Channel(*golden["cells"])
    o = Oracle(ch)
    o.init()
    reg = regions(ch)
    o.call("halo_x"); o.call("bc_y"); o.call("bc_z")
    for st, calls in (("bc", []), ("fx", ["flux_x"]), ("fy", ["flux_y"]), ("fz", ["flux_z"]), ("visc", ["viscous"])):
        for c in calls:
            o.call(c)
        for n in STAGES[st]:
            assert digest(o.array(n)[reg[STAGE_REGION[st]]]) == golden["stages"][st][n], (st, n)
    o.call("dts_residual"); o.call("sweeps")
    er = o.update()
    for n in STAGES["dts"]:
        assert digest(o.array(n)[reg["cell"]]) == golden["stages"]["dts"][n], n
    np.testing.assert_allclose(er, golden["first_norms"], rtol=1e-13)


def test_oracle_three_steps_bit_exact(golden):
    from oracle.oracle import Oracle
    ch = Channel(*golden["cells"])
    o = Oracle(ch)
    o.init()
    forces = [o.force]
    for _ in range(golden["steps"]):
        _, er = o.step(golden["iters_per_step"])
        forces.append(o.force)
    reg = regions(ch)
    q = o.q()[(slice(None),) + reg["cell"]]
    assert digest(q) == golden["final_state"]
    assert forces == golden["forces"]
    ref = np.load(os.path.join(GOLDEN, "channel_8x12x8.npz"))["q"]
    assert np.array_equal(q, ref)


@pytest.mark.skipif(not have_reference(), reason="reference sources not present")
def test_reference_rebuild_reproduces_fixture(golden):
    """Provenance of the fixture: the reference compiled now gives the same
    final-state hash."""
    from oracle.refrun import RefSolver
    ch = Channel(*golden["cells"])
    r = RefSolver(ch, threads=2)
    r.init()
    assert r.lib.ref_check_hyperplanes() == 0
    for _ in range(golden["steps"]):
        r.step(golden["iters_per_step"])
    reg = regions(ch)
    assert digest(r.q()[(slice(None),) + reg["cell"]]) == golden["final_state"]


@pytest.mark.skipif(not have_reference(), reason="reference sources not present")
def test_oracle_matches_reference_on_second_grid():
    """A second, non-cubic grid with more than one OpenMP thread in the
    reference: states stay bit-identical over two steps."""
    from oracle.oracle import Oracle
    from oracle.refrun import RefSolver
    ch = Channel(6, 10, 5)
    r = RefSolver(ch, threads=4)
    r.init()
    o = Oracle(ch)
    o.init()
    reg = regions(ch)
    for _ in range(2):
        r.step(6)
        o.step(6)
        sl = (slice(None),) + reg["cell"]
        assert np.array_equal(r.q()[sl], o.q()[sl])


@pytest.mark.skipif(not have_reference(), reason="reference sources not present")
@pytest.mark.parametrize("dims,threads", [((3, 6, 4), 2), ((11, 7, 9), 3)])
def test_oracle_matches_reference_at_edge_sizes(dims, threads):
    """The smallest grid the library accepts (Nx 3, Ny 6, Nz 4: every wall
    and end stencil of the reduced MUSCL forms is in use) and an odd-sized
    grid: two steps of four inner iterations stay bit-identical, and the
    norms agree (the reference divides by its global 3 Nx, the oracle by
    Nx)."""
    from oracle.oracle import Oracle
    from oracle.refrun import RefSolver
    ch = Channel(*dims)
    r = RefSolver(ch, threads=threads)
    r.init()
    o = Oracle(ch)
    o.init()
    sl = (slice(None),) + regions(ch)["cell"]
    for _ in range(2):
        _, er_r = r.step(4)
        _, er_o = o.step(4)
        assert np.array_equal(r.q()[sl], o.q()[sl])
        np.testing.assert_allclose(3.0 * np.asarray(er_r), er_o, rtol=1e-14)


@pytest.mark.skipif(not have_reference(), reason="reference sources not present")
def test_oracle_matches_reference_on_wavy_wall_grid():
    """Curvilinear metrics (wavy lower wall: every metric term the flat
    channel leaves zero is live) loaded into the reference's own arrays and
    into the oracle: two physical steps of five inner iterations are
    bit-identical."""
    from oracle.oracle import Oracle
    from oracle.refrun import RefSolver
    ch = Channel(8, 12, 8, wavy=True)
    r = RefSolver(ch, threads=2)
    r.init()
    o = Oracle(ch, curved_walls=False)     # the reference's own (flat) wall-face flux
    o.init()
    sl = np.s_[:, 3:ch.nx + 3, 2:ch.ny + 2, 2:ch.nz + 2]
    for _ in range(2):
        r.step(5)
        o.step(5)
        assert np.array_equal(r.q()[sl], o.q()[sl])
