"""Runs one of the seeded channel workloads on the GPU and prints what each
step or inner iteration did.

    python -m cgli_fu_flow_b200.run --workload c2 [--precision fp64|mixed]
        [--inner lusgs|dplur] [--predictor 0|1|2] (--steps N | --iterations N)
        [--drop 1e-3] [--cap 30]

--steps N runs N physical steps with the stopping rule (iterations per step,
the last norms and the device time of the step); --iterations N runs N bare
inner iterations from the seeded field (the five norms of each), the form
used for kernel profiles.  One JSON line per step / iteration.
"""
from __future__ import annotations

import argparse
import json

from . import channel as C


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(prog="python -m cgli_fu_flow_b200.run")
    ap.add_argument("--workload", default="c1", choices=sorted(C.WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--inner", default="lusgs", choices=["lusgs", "dplur"])
    ap.add_argument("--predictor", type=int, default=0, choices=[0, 1])
    g = ap.add_mutually_exclusive_group()
    g.add_argument("--steps", type=int, default=0)
    g.add_argument("--iterations", type=int, default=0)
    ap.add_argument("--drop", type=float, default=1e-3)
    ap.add_argument("--cap", type=int, default=30)
    a = ap.parse_args(argv)
    from .solver import FP64, MIXED, Solver
    ch = C.workload(a.workload)
    sol = Solver(ch, FP64 if a.precision == "fp64" else MIXED)
    sol.init()
    sol.set_inner_solver(a.inner)
    sol.set_predictor(a.predictor)
    if a.iterations:
        for n in range(a.iterations):
            er = sol.inner_iteration()
            print(json.dumps({"iteration": n + 1, "norms": [float(x) for x in er]}), flush=True)
    for n in range(a.steps):
        sol.event(0)
        it, er = sol.step(None, a.drop, a.cap)
        sol.event(1)
        print(json.dumps({"step": n + 1, "inner_iterations": it, "norms": [float(x) for x in er],
                          "ms": round(sol.elapsed_ms(0, 1), 3)}), flush=True)
    sol.close()


if __name__ == "__main__":
    main()
