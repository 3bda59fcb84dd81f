"""Generates the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own hot-path routines, compiled here by
oracle/build_ref.py from the reference sources, on the seeded channel
workload of cgli_fu_flow_b200.channel, and records for every stage of the
first inner iteration and for three physical steps:
  * the SHA-256 of the exact float64 bytes of each array (interior region),
  * the five update norms and the driving-force sequence,
  * the full final state Q^(n+1) of the interior cells (npz).
The oracle must reproduce every hash bit for bit; the GPU path is compared
with the stored state within tolerance.

It also records the reference's filter sensor (Filter.cpp) on the seeded
field at five thresholds (filter_<workload>.npz), and the DP-LUR inner
solver of DPLUSGS.cpp run in place of Dual_time_stepping (dplur_<workload>:
the first iteration's MR / NR / U_ hashes, three steps' norms, forces and
final state).

The reference's own open configuration (inflow / outflow x ends with
characteristic boundaries, sponge layers, heated-section walls, buoyancy),
run as a single rank 0 of 1: open_<workload> (three steps' norms and final
state with each inner solver).

Usage:  python tests/golden/make_golden.py [--filter | --dplur | --open] [nx ny nz]
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from cgli_fu_flow_b200.channel import Channel  # noqa: E402
from oracle.refrun import RefSolver  # noqa: E402

STEPS = 3
ITERS = 10


def regions(ch):
    nx, ny, nz = ch.nx, ch.ny, ch.nz
    return {
        "cell": np.s_[3:nx + 3, 2:ny + 2, 2:nz + 2],
        "bc": np.s_[0:nx + 6, 1:ny + 3, 1:nz + 3],
        "fx": np.s_[2:nx + 3, 1:ny + 1, 1:nz + 1],
        "fy": np.s_[2:nx + 2, 1:ny + 2, 1:nz + 1],
        "fz": np.s_[2:nx + 2, 1:ny + 1, 1:nz + 2],
        "metric": np.s_[0:nx + 6, 1:ny + 3, 1:nz + 3],
    }


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


STAGES = {
    "bc": [f"U{v}_" for v in range(1, 6)],
    "fx": [f"inFx{v}" for v in range(1, 6)],
    "fy": [f"inFy{v}" for v in range(1, 6)],
    "fz": [f"inFz{v}" for v in range(1, 6)],
    "visc": [f"vF{v}" for v in range(2, 6)],
    "dts": [f"MR{v}" for v in range(1, 6)] + [f"NR{v}" for v in range(1, 6)] + [f"U{v}_" for v in range(1, 6)],
}
STAGE_REGION = {"bc": "bc", "fx": "fx", "fy": "fy", "fz": "fz", "visc": "cell", "dts": "cell"}
METRICS = ["J", "xidx", "etdy", "ztdy", "ztdz", "J_u", "etdy_u", "J_v", "etdy_v", "J_w", "etdy_w", "ztdz_w"]


def main(nx=8, ny=12, nz=8):
    ch = Channel(nx, ny, nz)
    reg = regions(ch)
    r = RefSolver(ch, threads=1)
    r.init()
    out = {"workload": ch.name, "cells": [nx, ny, nz], "steps": STEPS, "iters_per_step": ITERS,
           "hyperplane_mismatches": int(r.lib.ref_check_hyperplanes()),
           "metrics": {m: digest(r.array(m)[reg["metric"]]) for m in METRICS}, "stages": {}}
    r.lib.ref_halo_bc()
    out["stages"]["bc"] = {n: digest(r.array(n)[reg["bc"]]) for n in STAGES["bc"]}
    for st, fn in (("fx", "ref_flux_x"), ("fy", "ref_flux_y"), ("fz", "ref_flux_z"), ("visc", "ref_viscous")):
        getattr(r.lib, fn)()
        out["stages"][st] = {n: digest(r.array(n)[reg[STAGE_REGION[st]]]) for n in STAGES[st]}
    import ctypes
    er = (ctypes.c_double * 5)()
    r.lib.ref_dts(er)
    out["stages"]["dts"] = {n: digest(r.array(n)[reg["cell"]]) for n in STAGES["dts"]}
    # the reference divides the norms by its global X_out = 3 Nx
    out["first_norms"] = [3.0 * x for x in er[:]]
    # restart and run whole steps
    r2 = RefSolver(ch, threads=1, build=False)
    r2.init()
    forces, norms = [r2.force], []
    for _ in range(STEPS):
        _, e = r2.step(ITERS)
        norms.append([3.0 * x for x in e])
        forces.append(r2.force)
    out["step_norms"] = norms
    out["forces"] = forces
    q = r2.q()[(slice(None),) + reg["cell"]]
    out["final_state"] = digest(q)
    base = os.path.join(HERE, ch.name)
    np.savez_compressed(base + ".npz", q=q)
    with open(base + ".json", "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", base + ".json", base + ".npz")


FILTER_QUANTILES = (0.1, 0.3, 0.5, 0.7, 0.9)
FILTER_E_HIGH, FILTER_E_LOW = 2.0, 1.0


def filter_input(ch, U_from):
    """The filter fixture's input: the seeded initial field after the halo
    exchange and the wall / periodic boundary conditions, with Y_point from
    Channel.y_point()."""
    return [U_from(f"U{v}_") for v in range(1, 6)], ch.y_point()


def main_filter(nx=8, ny=12, nz=8):
    """EpX/EpY/EpZ of the reference's Filter.cpp at five thresholds (the 10..90 %
    quantiles of the face ratios, so each threshold splits the faces), coded
    0 = face not in the reference's range (or an x-end face whose E planes
    the reference leaves unset), 1 = E_low, 2 = E_high."""
    from oracle import filter_oracle as F
    ch = Channel(nx, ny, nz)
    r = RefSolver(ch, threads=1)
    r.init()
    r.lib.ref_halo_bc()
    U, yp = filter_input(ch, lambda n: r.array(n).copy())
    J = r.array("J").copy()
    R = F.sensor(U, J, yp, ch.nx, ch.ny, ch.nz, x_ends=None)
    M = F.face_masks(ch.nx, ch.ny, ch.nz, J.shape, x_ends=None)
    fin = R[0][M[0] & np.isfinite(R[0])]
    crits = [float(np.quantile(fin, q)) for q in FILTER_QUANTILES]
    codes = np.zeros((len(crits), 3) + J.shape, np.uint8)
    for n, crit in enumerate(crits):
        ep = r.filter(yp, crit, FILTER_E_HIGH, FILTER_E_LOW)
        for f in range(3):
            codes[n, f][M[f] & (ep[f] == FILTER_E_LOW)] = 1
            codes[n, f][M[f] & (ep[f] == FILTER_E_HIGH)] = 2
    base = os.path.join(HERE, "filter_" + ch.name)
    np.savez_compressed(base + ".npz", codes=codes, crits=np.array(crits),
                        input_sha256=np.array([digest(np.stack(U))]))
    print("wrote", base + ".npz")


def main_dplur(nx=8, ny=12, nz=8):
    """DPLUSGS.cpp (with the loop-index fix of oracle/build_ref.py) in place of
    Dual_time_stepping: one inner iteration's arrays, then three steps of
    ITERS inner iterations with the driving-force update."""
    import ctypes
    ch = Channel(nx, ny, nz)
    reg = regions(ch)
    r = RefSolver(ch, threads=1, inner_solver="dplur")
    r.init()
    er = (ctypes.c_double * 5)()
    r.lib.ref_inner_iteration_dplusgs(er)
    out = {"workload": ch.name, "cells": [nx, ny, nz], "steps": STEPS, "iters_per_step": ITERS,
           "first": {n: digest(r.array(n)[reg["cell"]]) for n in STAGES["dts"]},
           "first_norms": [3.0 * x for x in er[:]]}
    r2 = RefSolver(ch, threads=1, build=False, inner_solver="dplur")
    r2.init()
    forces, norms = [r2.force], []
    for _ in range(STEPS):
        _, e = r2.step(ITERS)
        norms.append([3.0 * x for x in e])
        forces.append(r2.force)
    out["step_norms"] = norms
    out["forces"] = forces
    q = r2.q()[(slice(None),) + reg["cell"]]
    out["final_state"] = digest(q)
    base = os.path.join(HERE, "dplur_" + ch.name)
    np.savez_compressed(base + ".npz", q=q)
    with open(base + ".json", "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", base + ".json", base + ".npz")


def open_channel(nx=16, ny=12, nz=8):
    """The open-configuration fixture's workload: 4-cell inlet and outlet
    sponges, heated lower wall at the reference's 343.0592 K, buoyancy."""
    return Channel(nx, ny, nz, x_open=True, nx_inlet=4, nx_outlet=4, buoyancy=True, twall_lo=343.0592)


def main_open(nx=16, ny=12, nz=8):
    ch = open_channel(nx, ny, nz)
    out = {"workload": ch.name, "cells": [nx, ny, nz], "nx_inlet": ch.nx_inlet, "nx_outlet": ch.nx_outlet,
           "twall_lo": ch.twall_lo, "buoyancy": True, "steps": STEPS, "iters_per_step": ITERS}
    arrays = {}
    sl = (slice(None), slice(2, nx + 4), slice(2, ny + 2), slice(2, nz + 2))   # with the x-end ghost planes
    for solver in ("lusgs", "dplur"):
        r = RefSolver(ch, threads=1, inner_solver=solver)
        r.init()
        norms, forces = [], [r.force]
        for _ in range(STEPS):
            _, e = r.step(ITERS)
            norms.append(list(e))
            forces.append(r.force)
        q = r.q()[sl]
        out[solver] = {"step_norms": norms, "forces": forces, "final_state": digest(q)}
        arrays[solver] = q
    base = os.path.join(HERE, "open_" + f"{nx}x{ny}x{nz}")
    np.savez_compressed(base + ".npz", **arrays)
    with open(base + ".json", "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", base + ".json", base + ".npz")


if __name__ == "__main__":
    argv = sys.argv[1:]
    which = main
    if argv and argv[0] == "--filter":
        which, argv = main_filter, argv[1:]
    elif argv and argv[0] == "--dplur":
        which, argv = main_dplur, argv[1:]
    elif argv and argv[0] == "--open":
        which, argv = main_open, argv[1:]
    args = [int(a) for a in argv[0:3]] or ([16, 12, 8] if which is main_open else [8, 12, 8])
    which(*args)
