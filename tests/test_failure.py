"""Failure detection without a GPU fault.

The reference has no error path: its OpenMP barriers wait without limit and
a diverging run just prints non-finite norms (Dual_time_stepping.cpp:1761-1791,
main.cpp:313).  The library bounds every device-side wait of the wavefront
passes and turns both conditions into return codes:

* a wait on another tile that runs out (here forced with a wait limit of 0
  polls, so that such waits give up at once) records a timeout; the pass
  then runs to its end without waiting, the update leaves the state alone,
  the call returns CGLI_ETIMEOUT and the context keeps working;
* a non-finite state (NaN in Q) or a degenerate metric (J = 0 in one cell)
  gives non-finite update norms: CGLI_EDIVERGED.

Nothing here faults or hangs the GPU: the timeout is a bounded poll that
gives up, the divergence is plain IEEE arithmetic."""
import numpy as np
import pytest

from cgli_fu_flow_b200.channel import Channel

pytestmark = pytest.mark.gpu

ETIMEOUT = -6
EDIVERGED = -5


def interior(ch):
    return np.s_[:, 3:ch.nx + 3, 2:ch.ny + 2, 2:ch.nz + 2]


@pytest.fixture(scope="module")
def lib(cuda_lib):
    return cuda_lib


@pytest.mark.parametrize("dims", [(24, 40, 16), (32, 40, 16)])
def test_wait_that_runs_out_reports_timeout_and_keeps_the_state(lib, dims):
    from cgli_fu_flow_b200.solver import CgliError, Solver
    # 3 x 3 and 4 x 3 tiles of the 8 x 16 wavefront: every kind of wait
    # occurs (with four tiles along x, also the waits inside a cluster of
    # tiles when the library is built with clusters)
    ch = Channel(*dims)
    g = Solver(ch)
    g.init()
    sl = interior(ch)
    q0 = g.q()[sl].copy()
    g.set_wait_limit(0)
    for _ in range(2):   # the status word is cleared after each report
        with pytest.raises(CgliError) as ei:
            g.inner_iteration()
        assert ei.value.code == ETIMEOUT
        assert np.array_equal(g.q()[sl], q0), "a pass that gave up must leave the state unchanged"
    with pytest.raises(CgliError):
        g.set_wait_limit(-1)
    # the context works again: the default limit, a fresh start, four
    # iterations equal to those of a context that never timed out
    g.set_wait_limit(4194304)
    g.init()
    h = Solver(ch)
    h.init()
    ig, _ = g.step(4)
    ih, _ = h.step(4)
    assert ig == ih == 4
    assert np.array_equal(g.q()[sl], h.q()[sl])
    g.close()
    h.close()


def test_timeout_in_mixed_precision(lib):
    from cgli_fu_flow_b200.solver import MIXED, CgliError, Solver
    ch = Channel(32, 40, 16)
    g = Solver(ch, MIXED)
    g.init()
    g.set_wait_limit(0)
    with pytest.raises(CgliError) as ei:
        g.inner_iteration()
    assert ei.value.code == ETIMEOUT
    g.set_wait_limit(4194304)
    er = g.inner_iteration()
    assert np.all(np.isfinite(er))
    g.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_nan_in_the_state_reports_divergence(lib, precision):
    from cgli_fu_flow_b200.solver import CgliError, Solver
    ch = Channel(8, 12, 8)     # one wavefront tile: no hand-over waits
    g = Solver(ch, precision)
    q = ch.initial_conserved().copy()
    q[2, 4, 5, 3] = np.nan            # rho v of one interior cell
    g.init(q)
    with pytest.raises(CgliError) as ei:
        g.inner_iteration()
    assert ei.value.code == EDIVERGED
    g.close()


def test_zero_jacobian_reports_divergence(lib):
    from cgli_fu_flow_b200.solver import CgliError, Solver
    ch = Channel(8, 12, 8)
    g = Solver(ch)
    g.init()
    J = g.get("J")
    J[3 + 2, 2 + 6, 2 + 4] = 0.0
    g.set("J", J)
    with pytest.raises(CgliError) as ei:
        g.inner_iteration()
    assert ei.value.code == EDIVERGED
    g.close()
