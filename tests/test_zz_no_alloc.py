"""The entry point that allocates nothing: cgli_update_norms_noalloc.

It serves callers that cannot call cudaMalloc when they need the step (a
host code whose pool owns every device buffer, a loop that must not pay an
allocation's synchronisation, a process that has committed the whole GPU);
it keeps its per-row partial sums in a static device array.  Here it is
called through the C ABI on device arrays the test owns, twice in a row, and
must reproduce the update and the five norms of the context path
(cgli_dual_time_stepping) on the same inputs.  This file is collected last so
a run that stops at the first failure has run every other test first."""
import ctypes

import numpy as np
import pytest

from cgli_fu_flow_b200.channel import Channel

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _ptrs(ts):
    return (ctypes.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


def _one_iteration_inputs(sol):
    """Runs the reference-granularity entry points of one inner iteration up
    to the update and returns (U_ before the update, NR, norms, U_ after)."""
    sol.halo_x()
    sol.y_boundary_condition()
    sol.z_boundary_condition()
    sol.flux_x()
    sol.flux_y()
    sol.flux_z()
    sol.viscous_terms()
    before = sol.q()
    er = sol.dual_time_stepping()
    nr = np.stack([sol.get(f"NR{v}") for v in range(1, 6)])
    after = sol.q()
    return before, nr, er, after


def test_update_norms_noalloc_matches_context_path_twice():
    import torch
    from cgli_fu_flow_b200 import build
    from cgli_fu_flow_b200.solver import Solver, load_library
    build.build()
    L = load_library()
    ch = Channel(12, 16, 10)
    sol = Solver(ch)
    sol.init()
    J = torch.from_numpy(sol.get("J")).cuda()
    sl = np.s_[:, 3:ch.nx + 3, 2:ch.ny + 2, 2:ch.nz + 2]
    for call in range(2):
        before, nr, er_ctx, after = _one_iteration_inputs(sol)
        U = [torch.from_numpy(np.ascontiguousarray(before[v])).cuda() for v in range(5)]
        N = [torch.from_numpy(np.ascontiguousarray(nr[v])).cuda() for v in range(5)]
        torch.cuda.synchronize()
        er = (ctypes.c_double * 5)()
        rc = L.cgli_update_norms_noalloc(ch.nx, ch.ny, ch.nz, _ptrs(U), J.data_ptr(), _ptrs(N), er, None)
        assert rc == 0, L.cgli_last_error().decode()
        torch.cuda.synchronize()
        got = np.stack([u.cpu().numpy() for u in U])
        np.testing.assert_allclose(np.array(er[:]), er_ctx, rtol=TOL, err_msg=f"norms, call {call + 1}")
        for v in range(5):
            a, b = got[sl][v], after[sl][v]
            assert np.abs(a - b).max() <= TOL * np.abs(b).max(), (call, v)
    sol.close()


def test_update_norms_noalloc_rejects_oversized_grid():
    from cgli_fu_flow_b200.solver import load_library
    L = load_library()
    dummy = (ctypes.c_void_p * 5)(*([1] * 5))
    er = (ctypes.c_double * 5)()
    rc = L.cgli_update_norms_noalloc(1024, 256, 8, dummy, ctypes.c_void_p(1), dummy, er, None)
    assert rc == -1
    assert b"CGLI_NOALLOC_MAX_ROWS" in L.cgli_last_error()
