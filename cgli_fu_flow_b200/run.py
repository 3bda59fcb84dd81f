"""Runs one of the seeded channel workloads on the GPU and prints what each
step or inner iteration did.

    python -m cgli_fu_flow_b200.run (--workload c2 | --dims NX NY NZ)
        [--precision fp64|mixed] [--inner lusgs|dplur] [--predictor 0|1]
        (--steps N | --iterations N | --stages REPS) [--drop 1e-3] [--cap 30]

--steps N runs N physical steps with the stopping rule (iterations per step,
the last norms and the device time of the step); --iterations N runs N bare
inner iterations from the seeded field (the five norms of each), the form
used for kernel profiles; --stages REPS runs two inner iterations, then times
each stage of one inner iteration REPS times (cgli_profile_stages) and also
reports the wavefront passes per dependent step of the tile wavefront (the
tile shape the library was built with, cgli_sweep_tile_shape).  --dims runs the seeded channel on any grid instead of a named
workload.  One JSON line per step / iteration / stage report.
"""
from __future__ import annotations

import argparse
import json

from . import channel as C


def wavefront_steps(nx: int, ny: int, nz: int, ti: int, tj: int) -> int:
    """Hyperplane steps of one wavefront pass of ti x tj tiles: the last
    tile starts ti (tj) steps after its x (y) neighbour and runs nz + ti +
    tj - 2 steps."""
    nti, ntj = -(-nx // ti), -(-ny // tj)
    return nz + ti + tj - 2 + ti * (nti - 1) + tj * (ntj - 1)


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(prog="python -m cgli_fu_flow_b200.run")
    ap.add_argument("--workload", default="c1", choices=sorted(C.WORKLOADS))
    ap.add_argument("--dims", type=int, nargs=3, metavar=("NX", "NY", "NZ"), default=None)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--inner", default="lusgs", choices=["lusgs", "dplur"])
    ap.add_argument("--predictor", type=int, default=0, choices=[0, 1])
    g = ap.add_mutually_exclusive_group()
    g.add_argument("--steps", type=int, default=0)
    g.add_argument("--iterations", type=int, default=0)
    g.add_argument("--stages", type=int, default=0, metavar="REPS")
    ap.add_argument("--drop", type=float, default=1e-3)
    ap.add_argument("--cap", type=int, default=30)
    a = ap.parse_args(argv)
    from .solver import FP64, MIXED, Solver
    ch = C.Channel(*a.dims) if a.dims else C.workload(a.workload)
    sol = Solver(ch, FP64 if a.precision == "fp64" else MIXED)
    sol.init()
    sol.set_inner_solver(a.inner)
    sol.set_predictor(a.predictor)
    if a.iterations:
        for n in range(a.iterations):
            er = sol.inner_iteration()
            print(json.dumps({"iteration": n + 1, "norms": [float(x) for x in er]}), flush=True)
    if a.stages:
        from .solver import sweep_tile_shape
        for _ in range(2):
            sol.inner_iteration()
        st = sol.profile_stages(a.stages)
        ti, tj = sweep_tile_shape(FP64 if a.precision == "fp64" else MIXED)
        nsteps = wavefront_steps(ch.nx, ch.ny, ch.nz, ti, tj)
        print(json.dumps({"cells": [ch.nx, ch.ny, ch.nz], "stage_ms": {k: round(v, 4) for k, v in st.items()},
                          "tile": [ti, tj], "wavefront_steps": nsteps,
                          "us_per_wavefront_step": {d: round(st[f"sweep_{d}"] * 1e3 / nsteps, 3)
                                                    for d in ("forward", "backward")}}), flush=True)
    for n in range(a.steps):
        sol.event(0)
        it, er = sol.step(None, a.drop, a.cap)
        sol.event(1)
        print(json.dumps({"step": n + 1, "inner_iterations": it, "norms": [float(x) for x in er],
                          "ms": round(sol.elapsed_ms(0, 1), 3)}), flush=True)
    sol.close()


if __name__ == "__main__":
    main()
