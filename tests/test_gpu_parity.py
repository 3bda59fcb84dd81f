"""GPU parity: every entry point of the C ABI against the CPU oracle (and the
reference fixtures / reference build) on the same seeded inputs.

Tolerances.  The kernels evaluate the reference's expressions in the same
order, but the CUDA compiler fuses multiply-adds, so single-kernel results
agree to a few units in the last place: relative max error 1e-12 per stage
(normalised by the array's largest magnitude).  Whole steps are compared by
relative L2 per conserved variable, 1e-10 after 20 physical steps (the bar
the task sets for the plain FP64 path)."""
import os

import numpy as np
import pytest

from cgli_fu_flow_b200.channel import Channel

pytestmark = pytest.mark.gpu

STAGE_TOL = 1e-12
STEP_TOL = 1e-10


def rel_max(a, b):
    m = np.isfinite(a) & np.isfinite(b)
    scale = max(np.abs(b[m]).max(), 1e-300)
    return np.abs(a[m] - b[m]).max() / scale


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def regions(ch):
    from tests.golden.make_golden import regions as r
    return r(ch)


@pytest.fixture(scope="module")
def lib():
    from cgli_fu_flow_b200 import build, solver
    build.build()
    return solver.load_library()


def pair(ch, precision=0):
    from cgli_fu_flow_b200.solver import Solver
    from oracle.oracle import Oracle
    g = Solver(ch, precision)
    g.init()
    o = Oracle(ch)
    o.init()
    return g, o


@pytest.mark.parametrize("dims", [(8, 12, 8), (12, 16, 10)])
def test_metrics_on_device_match_oracle(lib, dims):
    ch = Channel(*dims)
    g, o = pair(ch)
    for n in ("J", "etdy", "ztdz", "J_u", "etdy_v", "J_v", "ztdz_w", "J_w"):
        assert np.array_equal(g.get(n), o.array(n)), n


@pytest.mark.parametrize("dims", [(8, 12, 8), (12, 16, 10)])
def test_routines_match_oracle(lib, dims):
    ch = Channel(*dims)
    g, o = pair(ch)
    reg = regions(ch)
    g.halo_x(); g.y_boundary_condition(); g.z_boundary_condition()
    o.call("halo_x"); o.call("bc_y"); o.call("bc_z")
    for v in range(1, 6):
        n = f"U{v}_"
        assert rel_max(g.get(n)[reg["bc"]], o.array(n)[reg["bc"]]) <= STAGE_TOL, n
    g.flux_x(); g.flux_y(); g.flux_z()
    o.call("flux_x"); o.call("flux_y"); o.call("flux_z")
    for d, r in (("x", "fx"), ("y", "fy"), ("z", "fz")):
        for v in range(1, 6):
            n = f"inF{d}{v}"
            assert rel_max(g.get(n)[reg[r]], o.array(n)[reg[r]]) <= STAGE_TOL, n
    g.viscous_terms(); o.call("viscous")
    for v in range(2, 6):
        n = f"vF{v}"
        assert rel_max(g.get(n)[reg["cell"]], o.array(n)[reg["cell"]]) <= 1e-11, n
    er_g = g.dual_time_stepping()
    o.call("dts_residual"); o.call("sweeps")
    er_o = o.update()
    for v in range(1, 6):
        for n in (f"MR{v}", f"NR{v}", f"U{v}_"):
            assert rel_max(g.get(n)[reg["cell"]], o.array(n)[reg["cell"]]) <= 1e-10, n
    np.testing.assert_allclose(er_g, er_o, rtol=1e-9)


def test_fused_iteration_matches_oracle(lib):
    ch = Channel(10, 12, 8)
    g, o = pair(ch)
    reg = regions(ch)
    for _ in range(3):
        er_g = g.inner_iteration()
        er_o = o.inner_iteration()
        np.testing.assert_allclose(er_g, er_o, rtol=1e-8)
    sl = (slice(None),) + reg["cell"]
    qg, qo = g.q()[sl], o.q()[sl]
    for v in range(5):
        assert rel_l2(qg[v], qo[v]) <= 1e-12, v


def test_three_steps_match_reference_fixture(lib):
    """Against the state the reference itself produced (tests/golden)."""
    from cgli_fu_flow_b200.solver import Solver
    ch = Channel(8, 12, 8)
    g = Solver(ch)
    g.init()
    for _ in range(3):
        it, _ = g.step(10)
        assert it == 10
    reg = regions(ch)
    q = g.q()[(slice(None),) + reg["cell"]]
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "channel_8x12x8.npz"))["q"]
    for v in range(5):
        assert rel_l2(q[v], ref[v]) <= STEP_TOL, v


def test_twenty_steps_match_oracle(lib):
    """20 physical steps x 10 inner iterations, relative L2 <= 1e-10."""
    ch = Channel(16, 16, 12)
    g, o = pair(ch)
    for _ in range(20):
        g.step(10)
        o.step(10)
    assert abs(g.force - o.force) <= 1e-8 * abs(o.force)
    reg = regions(ch)
    sl = (slice(None),) + reg["cell"]
    qg, qo = g.q()[sl], o.q()[sl]
    for v in range(5):
        assert rel_l2(qg[v], qo[v]) <= STEP_TOL, v


def test_adaptive_inner_loop_matches_oracle(lib):
    """The residual-drop stopping rule picks the same iteration counts."""
    ch = Channel(10, 12, 8)
    g, o = pair(ch)
    for _ in range(3):
        it_g, _ = g.step(None, drop=1e-2, cap=30)
        it_o, _ = o.step(None, drop=1e-2, cap=30)
        assert it_g == it_o
    reg = regions(ch)
    sl = (slice(None),) + reg["cell"]
    qg, qo = g.q()[sl], o.q()[sl]
    for v in range(5):
        assert rel_l2(qg[v], qo[v]) <= STEP_TOL, v


def _ref_lib_present(ch):
    return os.path.exists(os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref", ch.name,
                                       "libref.so"))


@pytest.mark.skipif(not _ref_lib_present(Channel(64, 64, 64)), reason="reference build for 64^3 not present")
def test_c1_twenty_steps_match_reference_build(lib):
    """The 64^3 channel, 20 steps x 10 inner iterations, GPU FP64 against the
    reference's own CPU build (OpenMP on every host core)."""
    from cgli_fu_flow_b200.solver import Solver
    from oracle.refrun import RefSolver
    ch = Channel(64, 64, 64)
    g = Solver(ch)
    g.init()
    r = RefSolver(ch, threads=os.cpu_count() or 1, build=False)
    r.init()
    for _ in range(20):
        g.step(10)
        r.step(10)
    reg = regions(ch)
    sl = (slice(None),) + reg["cell"]
    qg, qr = g.q()[sl], r.q()[sl]
    errs = [rel_l2(qg[v], qr[v]) for v in range(5)]
    print("C1 20-step relative L2 per variable:", errs)
    assert max(errs) <= STEP_TOL


@pytest.mark.skipif(not _ref_lib_present(Channel(256, 192, 192)),
                    reason="reference build for 256x192x192 not present")
def test_c2_twenty_steps_match_reference_build(lib):
    """The plain-FP64-at-scale channel at its own size, 256 x 192 x 192
    cells: 20 physical steps x 10 inner iterations on the GPU against the
    reference's own CPU build (OpenMP on every host core, several minutes).
    At this size the wavefront runs 32 x 12 tiles of 8 x 16 columns and the
    channel's per-row metric tables are in use, as in the benchmark."""
    from cgli_fu_flow_b200.solver import Solver
    from oracle.refrun import RefSolver
    ch = Channel(256, 192, 192)
    g = Solver(ch)
    g.init()
    r = RefSolver(ch, threads=os.cpu_count() or 1, build=False)
    r.init()
    for _ in range(20):
        g.step(10)
        r.step(10)
    reg = regions(ch)
    sl = (slice(None),) + reg["cell"]
    qg, qr = g.q()[sl], r.q()[sl]
    errs = [rel_l2(qg[v], qr[v]) for v in range(5)]
    print("C2 20-step relative L2 per variable:", errs)
    g.close()
    assert max(errs) <= STEP_TOL


def test_extrapolated_predictor_matches_oracle(lib):
    """Second-order extrapolated initial guess: same states as the oracle
    with the same predictor."""
    ch = Channel(10, 12, 8)
    g, o = pair(ch)
    g.set_predictor(1)
    for _ in range(4):
        g.step(8)
        o.step(8, predictor=1)
    reg = regions(ch)
    sl = (slice(None),) + reg["cell"]
    qg, qo = g.q()[sl], o.q()[sl]
    for v in range(5):
        assert rel_l2(qg[v], qo[v]) <= STEP_TOL, v


MIXED_TOL = 1e-6


def test_mixed_precision_hundred_steps_within_1e6_of_fp64_oracle(lib):
    """FP32 sweeps and split Jacobians, FP64 residual, filter-free update:
    after 100 physical steps x 10 inner iterations the state differs from the
    FP64 CPU oracle by at most 1e-6 (relative L2, every variable)."""
    from cgli_fu_flow_b200.solver import Solver, MIXED
    from oracle.oracle import Oracle
    ch = Channel(16, 24, 16)
    g = Solver(ch, MIXED)
    g.init()
    o = Oracle(ch)
    o.init()
    for _ in range(100):
        g.step(10)
        o.step(10)
    reg = regions(ch)
    sl = (slice(None),) + reg["cell"]
    qg, qo = g.q()[sl], o.q()[sl]
    errs = [rel_l2(qg[v], qo[v]) for v in range(5)]
    print("mixed vs FP64 oracle after 100 steps, relative L2 per variable:", errs)
    assert max(errs) <= MIXED_TOL


def test_copy_state_continues_the_same_run(lib):
    """Two contexts continued from one point by cgli_copy_state produce the
    same states as the original context (bit for bit: same kernels, same
    order)."""
    from cgli_fu_flow_b200.solver import Solver
    ch = Channel(10, 12, 8)
    a = Solver(ch)
    a.init()
    a.set_predictor(1)
    for _ in range(3):
        a.step(None, 1e-2, 20)
    b = Solver(ch)
    b.copy_state_from(a)
    b.set_predictor(1)
    for _ in range(2):
        ia, _ = a.step(None, 1e-2, 20)
        ib, _ = b.step(None, 1e-2, 20)
        assert ia == ib
    sl = (slice(None),) + regions(ch)["cell"]
    assert np.array_equal(a.q()[sl], b.q()[sl])


@pytest.mark.parametrize("precision", [0, 1])
def test_wavy_wall_general_metrics_match_oracle(lib, precision):
    """The curvilinear (wavy lower wall) grid takes the general-metric paths
    of every kernel (3-D metric arrays in the sweeps, non-zero etdx in the
    fluxes and viscous terms, the curved-wall pressure force): FP64 within
    1e-10 of the oracle after three steps of ten inner iterations, the mixed
    path within 1e-6.  Wall amplitude 0.01 h, where the scheme is stable."""
    from cgli_fu_flow_b200.solver import Solver
    from oracle.oracle import Oracle
    ch = Channel(16, 16, 32, wavy=True, wave=0.01)
    g = Solver(ch, precision)
    g.init()
    o = Oracle(ch)
    o.init()
    for _ in range(3):
        g.step(10)
        o.step(10)
    reg = regions(ch)
    sl = (slice(None),) + reg["cell"]
    qg, qo = g.q()[sl], o.q()[sl]
    errs = [rel_l2(qg[v], qo[v]) for v in range(5)]
    print("wavy wall, precision", precision, "relative L2 per variable:", errs)
    assert max(errs) <= (STEP_TOL if precision == 0 else MIXED_TOL)


def test_wavy_wall_specified_amplitude_first_step(lib):
    """The specified 0.05 h wall: the reference's scheme diverges after one
    to two steps on it (oracle and reference alike), so parity is checked on
    the first step (eight inner iterations), where every curvilinear term is
    at full strength."""
    from cgli_fu_flow_b200.solver import Solver
    from oracle.oracle import Oracle
    ch = Channel(16, 16, 12, wavy=True)
    g = Solver(ch)
    g.init()
    o = Oracle(ch)
    o.init()
    for _ in range(8):
        np.testing.assert_allclose(g.inner_iteration(), o.inner_iteration(), rtol=1e-8)
    sl = (slice(None),) + regions(ch)["cell"]
    qg, qo = g.q()[sl], o.q()[sl]
    assert max(rel_l2(qg[v], qo[v]) for v in range(5)) <= 1e-12


def test_statistics_match_restatement(lib):
    """Running sums of Statistic.cpp:120-160 over three steps against the
    numpy restatement applied to the same converged levels."""
    from cgli_fu_flow_b200.solver import Solver
    from oracle.stats_oracle import samples, sums
    ch = Channel(10, 12, 8)
    g = Solver(ch)
    g.init()
    J = g.get("J")
    want = np.zeros((11, ch.nx, ch.ny))
    for _ in range(3):
        g.step(6)
        g.accumulate_statistics()
        want += sums(g.q(), J, ch.nx, ch.ny, ch.nz)
    got, n = g.statistics()
    assert n == 3
    assert np.abs(got[:11] - want).max() <= 1e-12 * np.abs(want).max()
    # no cell at reference index k = 150 on this grid: the samples stay zero
    assert np.array_equal(got[11:], samples(g.q(), J, ch.nx, ch.ny, ch.nz))
    g.reset_statistics()
    assert g.statistics()[1] == 0 and not g.statistics()[0].any()


def test_mixed_mean_velocity_profile_within_half_percent(lib):
    """The mixed-precision acceptance criterion on a small channel: the mean streamwise
    velocity profile over x, z and the steps of the mixed path agrees with
    the FP64 path's within 0.5 % (max over the wall-normal cells, relative to
    the bulk velocity)."""
    from cgli_fu_flow_b200.solver import Solver, MIXED
    ch = Channel(16, 24, 32)
    prof = []
    for prec in (0, MIXED):
        g = Solver(ch, prec)
        g.init()
        for _ in range(30):
            g.step(None, 1e-3, 30)
            g.accumulate_statistics()
        prof.append(g.mean_profiles()["U"])
    diff = np.abs(prof[1] - prof[0]).max() / ch.u_b
    print("mean U profile, mixed vs FP64, max difference / U_b:", diff)
    assert diff <= 5e-3


def test_host_driven_loop_with_set_levels_matches_resident_run(lib):
    """A loop that keeps the time levels on the host (cgli_get_state after
    each step, cgli_set_levels before the next) reproduces the device-resident
    run bit for bit, stopping-rule iteration counts included (the running
    maxima carry on through cgli_set_levels)."""
    import numpy as np
    from cgli_fu_flow_b200.solver import Solver
    ch = Channel(16, 12, 8)
    a, b = Solver(ch), Solver(ch)
    a.init(); b.init()
    shape = (5,) + ch.shape
    qn = np.stack([b.get(f"U{v}") for v in range(1, 6)])
    qm = np.stack([b.get(f"U{v}q") for v in range(1, 6)])
    out = np.empty(shape)
    for _ in range(4):
        it_a, _ = a.step(None, drop=1e-2, cap=10)
        b.set_levels(np.ascontiguousarray(qn), np.ascontiguousarray(qm))
        it_b, _ = b.step(None, drop=1e-2, cap=10)
        assert it_a == it_b
        b.q_into(out)
        qm, qn = qn, out.copy()
    sl = (slice(None), slice(3, ch.nx + 3), slice(2, ch.ny + 2), slice(2, ch.nz + 2))
    assert np.array_equal(a.q()[sl], b.q()[sl])


def test_sweep_time_counts_the_passes_of_every_iteration(lib):
    """cgli_sweep_time: events inside the iteration graph time the four
    wavefront passes of every inner iteration; reset clears the totals."""
    from cgli_fu_flow_b200.solver import Solver
    g = Solver(Channel(16, 12, 8))
    g.init()
    g.sweep_time(reset=True)
    it, _ = g.step(None, drop=1e-2, cap=6)
    ms, passes = g.sweep_time(reset=True)
    assert passes == 4 * it and ms > 0
    assert g.sweep_time() == (0.0, 0)
