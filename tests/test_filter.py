"""Filter sensor (Filter.cpp:12-1720): the oracle against the reference's own
output, then the CUDA kernels against the oracle.

The sensor's output is a choice between two values per face, decided by a
ratio that the kernels compute with the reference's operations in the
reference's order without fused multiply-adds, so the bar is exact equality
of EpX/EpY/EpZ at every threshold."""
import os

import numpy as np
import pytest

from cgli_fu_flow_b200.channel import Channel
from oracle import filter_oracle as F

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "filter_channel_8x12x8.npz")
E_HIGH, E_LOW = 2.0, 1.0


def oracle_input(ch):
    """Seeded field after halo exchange and boundary conditions (the
    reference's ref_halo_bc stage, reproduced bit for bit by the oracle)."""
    from oracle.oracle import Oracle
    o = Oracle(ch)
    o.init()
    for n in ("halo_x", "bc_y", "bc_z"):
        o.call(n)
    U = [o.array(f"U{v}_").copy() for v in range(1, 6)]
    return U, o.array("J").copy(), ch.y_point()


def codes(ep, masks):
    out = []
    for e, m in zip(ep, masks):
        c = np.zeros(e.shape, np.uint8)
        c[m & (e == E_LOW)] = 1
        c[m & (e == E_HIGH)] = 2
        out.append(c)
    return out


def test_filter_oracle_matches_reference_fixture():
    from tests.golden.make_golden import digest
    fx = np.load(FIX)
    ch = Channel(8, 12, 8)
    U, J, yp = oracle_input(ch)
    assert digest(np.stack(U)) == str(fx["input_sha256"][0])
    masks = F.face_masks(ch.nx, ch.ny, ch.nz, J.shape, x_ends=None)
    for n, crit in enumerate(fx["crits"]):
        ep, _, _ = F.filter_ep(U, J, yp, ch.nx, ch.ny, ch.nz, crit, E_HIGH, E_LOW, x_ends=None)
        got = codes(ep, masks)
        for f in range(3):
            assert np.array_equal(got[f], fx["codes"][n, f]), (n, "XYZ"[f])
    # each threshold splits the faces: both values occur
    assert (fx["codes"] == 1).any() and (fx["codes"] == 2).any()


def test_filter_oracle_periodic_x_ends():
    """With the periodic image in x, the first and last EpX faces are the same
    physical face (between the last and the first interior plane)."""
    ch = Channel(8, 12, 8)
    U, J, yp = oracle_input(ch)
    RX, RY, RZ = F.sensor(U, J, yp, ch.nx, ch.ny, ch.nz, x_ends="periodic")
    g = ch.nx + 2
    a, b = RX[2, 1:ch.ny + 1, 1:ch.nz + 1], RX[g, 1:ch.ny + 1, 1:ch.nz + 1]
    assert np.isfinite(a).all() and np.array_equal(a, b)
    # the other faces do not depend on the x-end choice
    R0 = F.sensor(U, J, yp, ch.nx, ch.ny, ch.nz, x_ends=None)
    assert np.array_equal(RX[3:g], R0[0][3:g], equal_nan=True)
    assert np.array_equal(RY, R0[1], equal_nan=True) and np.array_equal(RZ, R0[2], equal_nan=True)


from oracle.build_ref import REF_SRC as REF  # noqa: E402  (the reference tree the recipe reads)


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference sources not present")
def test_filter_oracle_matches_reference_build_second_grid():
    from oracle.refrun import RefSolver
    ch = Channel(16, 24, 12)
    r = RefSolver(ch, threads=1, build=True)
    r.init()
    r.lib.ref_halo_bc()
    U = [r.array(f"U{v}_").copy() for v in range(1, 6)]
    J, yp = r.array("J").copy(), ch.y_point()
    R = F.sensor(U, J, yp, ch.nx, ch.ny, ch.nz, x_ends=None)
    M = F.face_masks(ch.nx, ch.ny, ch.nz, J.shape, x_ends=None)
    for q in (0.25, 0.5, 0.75):
        crit = float(np.quantile(R[0][M[0]], q))
        ref = r.filter(yp, crit, E_HIGH, E_LOW)
        mine, _, _ = F.filter_ep(U, J, yp, ch.nx, ch.ny, ch.nz, crit, E_HIGH, E_LOW, x_ends=None)
        for f in range(3):
            assert np.array_equal(ref[f][M[f]], mine[f][M[f]]), (q, "XYZ"[f])


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference sources not present")
@pytest.mark.parametrize("dims", [(11, 14, 9), (8, 6, 5)])
def test_filter_oracle_matches_reference_build_odd_sizes(dims):
    """Odd extents and the smallest wall-normal extent, on a state two steps
    from the seeded field: EpX/EpY/EpZ bit-identical at three thresholds."""
    from oracle.refrun import RefSolver
    ch = Channel(*dims)
    r = RefSolver(ch, threads=2, build=True)
    r.init()
    r.step(2)
    r.lib.ref_halo_bc()
    U = [r.array(f"U{v}_").copy() for v in range(1, 6)]
    J, yp = r.array("J").copy(), ch.y_point()
    R = F.sensor(U, J, yp, ch.nx, ch.ny, ch.nz, x_ends=None)
    M = F.face_masks(ch.nx, ch.ny, ch.nz, J.shape, x_ends=None)
    for q in (0.25, 0.5, 0.75):
        crit = float(np.quantile(R[0][M[0]], q))
        ref = r.filter(yp, crit, E_HIGH, E_LOW)
        mine, _, _ = F.filter_ep(U, J, yp, ch.nx, ch.ny, ch.nz, crit, E_HIGH, E_LOW, x_ends=None)
        for f in range(3):
            assert np.array_equal(ref[f][M[f]], mine[f][M[f]]), (q, "XYZ"[f])


# ------------------------------------------------------------------ GPU

def _gpu(ch):
    from cgli_fu_flow_b200 import build
    from cgli_fu_flow_b200.solver import Solver
    build.build()
    g = Solver(ch)
    g.init()
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(8, 12, 8), (20, 36, 40)])
def test_filter_gpu_matches_oracle(dims):
    ch = Channel(*dims)
    g = _gpu(ch)
    g.halo_x(); g.y_boundary_condition(); g.z_boundary_condition()
    U = [g.get(f"U{v}_") for v in range(1, 6)]
    J, yp = g.get("J"), ch.y_point()
    R = F.sensor(U, J, yp, ch.nx, ch.ny, ch.nz)
    M = F.face_masks(ch.nx, ch.ny, ch.nz, J.shape)
    for q in (0.1, 0.5, 0.9):
        crit = float(np.quantile(R[0][M[0]], q))
        got = g.filter(yp, crit, E_HIGH, E_LOW)
        want, _, _ = F.filter_ep(U, J, yp, ch.nx, ch.ny, ch.nz, crit, E_HIGH, E_LOW)
        for f in range(3):
            assert np.array_equal(got[f][M[f]], want[f][M[f]]), (q, "XYZ"[f])
            assert (got[f][~M[f]] == 0).all()


@pytest.mark.gpu
def test_filter_gpu_matches_reference_fixture():
    fx = np.load(FIX)
    ch = Channel(8, 12, 8)
    g = _gpu(ch)
    g.halo_x(); g.y_boundary_condition(); g.z_boundary_condition()
    M = F.face_masks(ch.nx, ch.ny, ch.nz, ch.shape, x_ends=None)
    yp = ch.y_point()
    for n, crit in enumerate(fx["crits"]):
        got = codes(g.filter(yp, crit, E_HIGH, E_LOW), M)
        for f in range(3):
            assert np.array_equal(got[f], fx["codes"][n, f]), (n, "XYZ"[f])


@pytest.mark.gpu
def test_filter_gpu_on_evolved_state():
    """After three physical steps on the GPU (a turbulent-looking field with
    stale ghost planes, read as stored like the reference does)."""
    ch = Channel(16, 16, 12)
    g = _gpu(ch)
    for _ in range(3):
        g.step(6)
    U = [g.get(f"U{v}_") for v in range(1, 6)]
    J, yp = g.get("J"), ch.y_point()
    R = F.sensor(U, J, yp, ch.nx, ch.ny, ch.nz)
    M = F.face_masks(ch.nx, ch.ny, ch.nz, J.shape)
    crit = float(np.median(R[1][M[1]]))
    got = g.filter(yp, crit, E_HIGH, E_LOW)
    want, _, _ = F.filter_ep(U, J, yp, ch.nx, ch.ny, ch.nz, crit, E_HIGH, E_LOW)
    for f in range(3):
        assert np.array_equal(got[f][M[f]], want[f][M[f]]), "XYZ"[f]


@pytest.mark.gpu
def test_filter_requires_y_point():
    from cgli_fu_flow_b200.solver import CgliError
    g = _gpu(Channel(8, 12, 8))
    with pytest.raises(CgliError):
        g._rc(g.L.cgli_filter(g.h, 1.0, E_HIGH, E_LOW))
