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


def _update_restated(q, J, nr):
    """The update and norms of Dual_time_stepping.cpp:1702-1782 in numpy, on
    interior arrays (5, nx, ny, nz), J and nr likewise."""
    KG = 1.4
    rho_old = q[0] * J
    u0, v0, w0 = q[1] / q[0], q[2] / q[0], q[3] / q[0]
    p_old = (q[4] * J - 0.5 * rho_old * (u0 * u0 + v0 * v0 + w0 * w0)) * (KG - 1)
    t_old = p_old / rho_old
    p = p_old + nr[0] * J
    u, v, w = u0 + nr[1] * J, v0 + nr[2] * J, w0 + nr[3] * J
    t = t_old + nr[4] * J
    rho = p / t
    out = np.stack([rho / J, rho * u / J, rho * v / J, rho * w / J,
                    (p / (KG - 1) + 0.5 * rho * (u * u + v * v + w * w)) / J])
    n = q[0].size
    er = [np.sqrt(np.sum((a - b) ** 2)) / n for a, b in ((rho, rho_old), (u, u0), (v, v0), (w, w0), (t, t_old))]
    return out, np.array(er)


def _synthetic(nx, ny, nz, seed):
    """A smooth positive state Q/J, J and small increments NR in the
    reference layout [Nx+6][Ny+4][Nz+4]."""
    rng = np.random.default_rng(seed)
    shape = (nx + 6, ny + 4, nz + 4)
    J = 1.0 + 0.1 * rng.random(shape)
    rho = 1.18 * (1 + 0.01 * rng.random(shape))
    u, v, w = 60 + rng.random(shape), rng.random(shape), rng.random(shape)
    p = 101300.0 * (1 + 0.01 * rng.random(shape))
    q = np.stack([rho, rho * u, rho * v, rho * w, p / 0.4 + 0.5 * rho * (u * u + v * v + w * w)]) / J
    nr = np.stack([1e-3 * p, 1e-2 * u, 1e-2 * v, 1e-2 * w, 1e-3 * p / rho]) * (rng.random((5,) + shape) - 0.5)
    return q, J, nr


def test_update_norms_noalloc_grid_wider_than_a_grid_dimension():
    """Nx above 65535 (a limit of the second and third grid dimensions):
    within the row limit, the call runs and matches the restated update."""
    import torch
    from cgli_fu_flow_b200.solver import load_library
    L = load_library()
    nx, ny, nz = 70000, 1, 4
    q, J, nr = _synthetic(nx, ny, nz, 7)
    U = [torch.from_numpy(np.ascontiguousarray(q[v])).cuda() for v in range(5)]
    N = [torch.from_numpy(np.ascontiguousarray(nr[v])).cuda() for v in range(5)]
    Jd = torch.from_numpy(J).cuda()
    er = (ctypes.c_double * 5)()
    rc = L.cgli_update_norms_noalloc(nx, ny, nz, _ptrs(U), Jd.data_ptr(), _ptrs(N), er, None)
    assert rc == 0, L.cgli_last_error().decode()
    got = np.stack([u.cpu().numpy() for u in U])
    sl = np.s_[:, 3:nx + 3, 2:ny + 2, 2:nz + 2]
    want, er_want = _update_restated(q[sl], J[sl[1:]], nr[sl])
    np.testing.assert_allclose(np.array(er[:]), er_want, rtol=1e-10)
    for v in range(5):
        assert np.abs(got[sl][v] - want[v]).max() <= TOL * np.abs(want[v]).max(), v


RESET_PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include <cuda_runtime.h>
#include "cgli_fu_flow.h"
/* two calls on the same inputs with a device reset between them: the second
   must find the static array at its address in the new context */
static int run(int nx, int ny, int nz, const double *hq, const double *hJ, const double *hn, double er[5]) {
  size_t n = (size_t)(nx + 6) * (ny + 4) * (nz + 4), b = n * sizeof(double);
  double *U[5], *N[5], *J;
  for (int v = 0; v < 5; v++) {
    if (cudaMalloc((void **)&U[v], b) || cudaMalloc((void **)&N[v], b)) return 10;
    cudaMemcpy(U[v], hq + v * n, b, cudaMemcpyHostToDevice);
    cudaMemcpy(N[v], hn + v * n, b, cudaMemcpyHostToDevice);
  }
  if (cudaMalloc((void **)&J, b)) return 11;
  cudaMemcpy(J, hJ, b, cudaMemcpyHostToDevice);
  int rc = cgli_update_norms_noalloc(nx, ny, nz, U, J, (const double *const *)N, er, NULL);
  if (rc) { fprintf(stderr, "%s\n", cgli_last_error()); return 12; }
  for (int v = 0; v < 5; v++) { cudaFree(U[v]); cudaFree(N[v]); }
  cudaFree(J);
  return cudaGetLastError() == cudaSuccess ? 0 : 13;
}
int main(int argc, char **argv) {
  int nx = atoi(argv[1]), ny = atoi(argv[2]), nz = atoi(argv[3]);
  size_t n = (size_t)(nx + 6) * (ny + 4) * (nz + 4);
  double *q = malloc(5 * n * 8), *J = malloc(n * 8), *nr = malloc(5 * n * 8);
  FILE *f = fopen(argv[4], "rb");
  if (!f || fread(q, 8, 5 * n, f) != 5 * n || fread(J, 8, n, f) != n || fread(nr, 8, 5 * n, f) != 5 * n) return 2;
  fclose(f);
  double a[5], b[5];
  int rc = run(nx, ny, nz, q, J, nr, a);
  if (rc) return rc;
  if (cudaDeviceReset() != cudaSuccess) return 3;
  rc = run(nx, ny, nz, q, J, nr, b);
  if (rc) return rc;
  for (int v = 0; v < 5; v++) printf("%.17g %.17g\n", a[v], b[v]);
  return 0;
}
"""


def test_update_norms_noalloc_after_a_device_reset(tmp_path):
    """A caller that resets its device between two calls (cudaDeviceReset
    ends the process's context; the module and its static array are loaded
    again, possibly elsewhere): the second call must use the new address.
    Runs as a separate C program so that the reset touches no other user of
    the device in the test process."""
    import os
    import shutil
    import subprocess
    from cgli_fu_flow_b200 import build
    if shutil.which("gcc") is None:
        pytest.skip("gcc not present")
    build.build()
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(repo, "cgli_fu_flow_b200")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    src = tmp_path / "reset.c"
    src.write_text(RESET_PROGRAM)
    exe = tmp_path / "reset"
    r = subprocess.run(["gcc", "-std=c99", "-I", os.path.join(repo, "include"), "-I", os.path.join(cuda, "include"),
                        str(src), "-o", str(exe), "-L", libdir, "-lcgli_fu_flow", f"-Wl,-rpath,{libdir}",
                        "-L", os.path.join(cuda, "lib64"), "-lcudart", f"-Wl,-rpath,{os.path.join(cuda, 'lib64')}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    nx, ny, nz = 12, 16, 10
    q, J, nr = _synthetic(nx, ny, nz, 11)
    data = tmp_path / "in.bin"
    with open(data, "wb") as fh:
        fh.write(q.tobytes() + J.tobytes() + nr.tobytes())
    r = subprocess.run([str(exe), str(nx), str(ny), str(nz), str(data)], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, (r.returncode, r.stderr)
    vals = np.array([[float(x) for x in line.split()] for line in r.stdout.split("\n") if line.strip()])
    sl = np.s_[:, 3:nx + 3, 2:ny + 2, 2:nz + 2]
    _, er_want = _update_restated(q[sl], J[sl[1:]], nr[sl])
    assert np.array_equal(vals[:, 0], vals[:, 1]), vals
    np.testing.assert_allclose(vals[:, 0], er_want, rtol=1e-10)
