"""CPU-only checks of the product library: it loads, exports every entry
point the header declares, and its host-side set-up code (analytic metrics,
hyperplane enumeration) and workload definitions are right.  No kernel runs."""
import hashlib
import json
import os
import re

import numpy as np
import pytest

from cgli_fu_flow_b200 import channel as C
from cgli_fu_flow_b200.channel import Channel

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(REPO, "include", "cgli_fu_flow.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\s*\*|long long)\s*(cgli_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol(cuda_lib):
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(cuda_lib, s), s
    from cgli_fu_flow_b200.solver import EXPORTS
    assert sorted(EXPORTS) == syms


def test_host_metrics_match_reference_fixture(cuda_lib):
    from cgli_fu_flow_b200.solver import channel_metric_host
    from tests.golden.make_golden import regions
    golden = json.load(open(os.path.join(REPO, "tests", "golden", "channel_8x12x8.json")))
    ch = Channel(*golden["cells"])
    reg = regions(ch)
    for name, h in golden["metrics"].items():
        a = channel_metric_host(ch, name)[reg["metric"]]
        assert hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest() == h, name


def test_host_metrics_match_oracle_everywhere(cuda_lib):
    from cgli_fu_flow_b200.solver import channel_metric_host
    from oracle.oracle import Oracle
    ch = Channel(10, 14, 6)
    o = Oracle(ch)
    names = ["J", "J_u", "J_v", "J_w"] + [m + s for m in ("xidx", "xidy", "xidz", "etdx", "etdy", "etdz",
                                                         "ztdx", "ztdy", "ztdz") for s in ("", "_u", "_v", "_w")]
    for n in names:
        assert np.array_equal(channel_metric_host(ch, n), o.array(n)), n


def brute_force_hyperplanes(nx, ny, nz):
    """Hyperplane.cpp:50-78 as written: for every m scan all cells."""
    ie, jn, kn = nx + 2, ny + 1, nz + 1
    cells, counts = [], {}
    for m in range(7, ie + jn + kn + 1):
        mi = 0
        for i in range(3, ie + 1):
            for j in range(2, jn + 1):
                for k in range(2, kn + 1):
                    if i + j + k == m:
                        cells.append((i, j, k))
                        mi += 1
        counts[m] = (len(cells), mi)
    return cells, counts


@pytest.mark.parametrize("dims", [(3, 6, 4), (5, 7, 9), (8, 12, 8)])
def test_hyperplane_enumeration_matches_reference_order(cuda_lib, dims):
    from cgli_fu_flow_b200.solver import hyperplane_lists
    nijk, ijk = hyperplane_lists(*dims)
    cells, counts = brute_force_hyperplanes(*dims)
    assert [tuple(x) for x in ijk[1:]] == cells
    for m, (end, cnt) in counts.items():
        assert tuple(nijk[m]) == (end, cnt)


def test_hyperplane_rejects_short_buffers(cuda_lib):
    import ctypes
    buf = np.zeros(4, dtype=np.int32)
    rc = cuda_lib.cgli_hyperplane(4, 6, 4, buf.ctypes.data, 4, buf.ctypes.data, 4)
    assert rc == -1


def test_create_rejects_too_small_grid(cuda_lib):
    import ctypes
    from cgli_fu_flow_b200.solver import Params
    p = Params(4, 5, 4, 1e-3, 0.2, 1e-3, 1e-6, 1e-3, 1.85e-5, 0.72, 298.0, 298.0, 0.0, 0)
    h = ctypes.c_void_p()
    assert cuda_lib.cgli_create(ctypes.byref(p), ctypes.byref(h)) == -1
    assert b"grid too small" in cuda_lib.cgli_last_error()


def test_initial_field_properties():
    ch = Channel(16, 12, 8)
    rho, u, v, w, p = ch.initial_primitives()
    y = ch.cell_y()
    ulam = 1.5 * ch.u_b * (1.0 - (y / ch.h - 1.0) ** 2)
    for comp, base in ((u, ulam), (v, 0 * ulam), (w, 0 * ulam)):
        pert = comp - base[None, :, None]
        assert 0.05 * ch.u_b < np.abs(pert).max() <= 0.125 * ch.u_b  # +-10 % plus the removed plane mean
        np.testing.assert_allclose(pert.mean(axis=(0, 2)), 0, atol=1e-12 * ch.u_b)
    assert np.all(rho == ch.rho0) and np.all(p == C.P0)
    # the seeded generator is deterministic
    assert np.array_equal(Channel(16, 12, 8).initial_conserved(), ch.initial_conserved())
    # walls at y = 0 and y = 2h
    assert 0 < y[0] < y[-1] < ch.high


def test_channel_constants():
    ch = Channel(64, 64, 64)
    assert abs(ch.u_b / ch.c0 - 0.2) < 1e-12
    assert abs(ch.rho0 * ch.u_b * 2 * ch.h / C.MU0 - 5600) < 1e-6
    assert abs(ch.dt * ch.u_b / ch.dxi - 1.0) < 1e-12


def test_force_controller_steers_toward_target():
    ch = Channel(8, 12, 8)
    st = {}
    f_hi = C.force_update(st, ch.target_flux * 1.01, ch)
    assert f_hi < ch.force_lam
    st = {}
    f_lo = C.force_update(st, ch.target_flux * 0.99, ch)
    assert f_lo > ch.force_lam


def test_wavefront_step_count():
    """Dependent steps of one wavefront pass of ti x tj tiles (the profiling
    runner's per-step figure): nz + ti + tj - 2 for one tile, plus ti per
    extra tile in x and tj per extra tile in y (ragged tiles count whole)."""
    from cgli_fu_flow_b200.run import wavefront_steps
    assert wavefront_steps(8, 16, 192, 8, 16) == 214
    assert wavefront_steps(256, 192, 192, 8, 16) == 256 + 192 + 192 - 2
    assert wavefront_steps(9, 17, 10, 8, 16) == 10 + 22 + 8 + 16
    # other tile shapes the library can be built with
    assert wavefront_steps(256, 192, 192, 16, 16) == 256 + 192 + 192 - 2
    assert wavefront_steps(20, 20, 8, 16, 16) == 8 + 30 + 16 + 16
    assert wavefront_steps(9, 40, 10, 8, 32) == 10 + 38 + 8 + 32


def test_library_reports_its_tile_shape(cuda_lib):
    """The tile shape comes from the library itself (set at build time)."""
    from cgli_fu_flow_b200.solver import FP64, MIXED, CgliError, sweep_tile_shape
    for precision in (FP64, MIXED):
        ti, tj = sweep_tile_shape(precision)
        assert ti >= 1 and tj >= 1 and (ti * tj) % 32 == 0
    with pytest.raises(CgliError):
        sweep_tile_shape(7)
