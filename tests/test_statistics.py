"""The running statistics against the reference's own Statistic().

Statistic.cpp:12-506 accumulates per (i, j) the sums over k of U, V, W, T,
UU, VV, WW, TT, UV, UT, VT (and keeps U, T of the cell k = 150), and every
statistic_step-th step writes the means of the x planes at its observation
positions to st_obs<n>_<step>.dat (:160-331).  The reference build runs it
after each step with five observation planes; its files pin the numpy
restatement (oracle/stats_oracle.py, CPU) and the GPU's sums (cgli_statistics_*).
The grid has Nz = 152 so that the k = 150 sample exists."""
import os

import numpy as np
import pytest

from cgli_fu_flow_b200.channel import Channel
from tests.conftest import have_reference

DIMS = (8, 12, 152)
STEPS = 3
ITERS = 4
PLANES = [3, 4, 6, 9, 10]      # interior x planes (3 .. Nx+2) the reference writes out


def _ref_lib_present(ch):
    return os.path.exists(os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref", ch.name,
                                       "libref.so"))


def _reference_run(ch, build):
    """The reference run: STEPS steps of ITERS inner iterations, Statistic()
    after each; returns the written planes and the converged levels."""
    from oracle.refrun import RefSolver
    r = RefSolver(ch, threads=os.cpu_count() or 1, build=build)
    r.init()
    levels, written = [], None
    for step in range(1, STEPS + 1):
        r.step(ITERS)
        levels.append(r.q())
        out = r.statistic(step, STEPS, PLANES)
        if step < STEPS:
            assert out is None, "the reference writes only every statistic_step-th step"
        else:
            written = out
    assert written is not None and sorted(written) == PLANES
    return written, levels, r.array("J").copy()


def _means(sums, samples, steps, nz, i):
    """The 13 rows the reference writes for plane i: means of the 11 sums
    over k and the steps, then U and T at k = 150."""
    il = i - 3
    return np.concatenate([sums[:, il, :] / (steps * nz), samples[:, il, :]])


@pytest.mark.skipif(not have_reference(), reason="reference sources not present")
def test_restatement_matches_reference_statistic():
    from oracle.stats_oracle import samples, sums
    ch = Channel(*DIMS)
    written, levels, J = _reference_run(ch, build=True)
    acc = sum(sums(q, J, ch.nx, ch.ny, ch.nz) for q in levels)
    smp = samples(levels[-1], J, ch.nx, ch.ny, ch.nz)
    for i in PLANES:
        want = written[i]
        got = _means(acc, smp, STEPS, ch.nz, i)
        # the files carry 16 decimals: compare at that absolute precision
        scale = np.abs(want).max(axis=1, keepdims=True)
        assert np.all(np.abs(got - want) <= 1e-14 * scale + 2e-16), i


@pytest.mark.gpu
@pytest.mark.skipif(not _ref_lib_present(Channel(*DIMS)), reason="reference build for 8x12x152 not present")
def test_gpu_statistics_match_reference_statistic(cuda_lib):
    from cgli_fu_flow_b200.solver import Solver
    ch = Channel(*DIMS)
    written, _, _ = _reference_run(ch, build=False)
    g = Solver(ch)
    g.init()
    for _ in range(STEPS):
        g.step(ITERS)
        g.accumulate_statistics()
    vals, n = g.statistics()
    g.close()
    assert n == STEPS
    sums, smp = vals[:11], vals[11:]
    for i in PLANES:
        want = written[i]
        got = _means(sums, smp, STEPS, ch.nz, i)
        scale = np.abs(want).max(axis=1, keepdims=True)
        err = (np.abs(got - want) / scale).max()
        # the GPU state after three steps agrees with the reference build to
        # about 1e-13 relative; the statistics inherit that
        assert err <= 1e-10, (i, err)
