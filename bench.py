"""Benchmark of the per-step hot path: Mcell-steps/s on the seeded channel.

A step is one physical time step of the dual-time scheme on the
256 x 192 x 192 channel (the plain-FP64-at-scale workload): inner LU-SGS
iterations until every one of the five update norms, divided by its running
maximum over the run (the reference's rule), is below 1e-3 (capped at 30),
then the time-level shift and the driving-force update.  All state stays
resident on the GPU for `value` (plain FP64, the reference's algorithm, from
the seeded field); `e2e` repeats the measurement through the C ABI with the
step's inputs copied from pinned host memory and its result copied back
every step.

`arms` compares, from one common point of a run (after `--collect` steps
with second-order extrapolation in mixed precision, whose converged levels
train the learned initial guess with Adam on the GPU), the same number of
steps in: plain FP64 (previous-level guess), mixed precision with
extrapolation, mixed precision with the learned guess, and plain FP64 with
the DP-LUR inner solver of DPLUSGS.cpp in place of the LU-SGS sweeps (its
stopping norms are those of DPLUSGS.cpp, squared increments with the
pressure first), with each arm's state error against the FP64 arm.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With N > 1 (torchrun) every rank runs an independent replica of the workload
(the solver does not shard: one x-slab per GPU with no exchange is the
reference's own decomposition collapsed to one slab), `value` sums the ranks'
cell-steps over the slowest rank's time.  `--impl reference` times the
reference's own CPU build (compiled here from its sources into oracle/_ref)
on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

from cgli_fu_flow_b200 import channel as C  # noqa: E402

METRIC = "Mcell-steps/s at fixed inner-residual drop (1e-3, cap 30)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(C.WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--drop", type=float, default=1e-3)
    ap.add_argument("--cap", type=int, default=30)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-iters", type=int, default=4, help="reference inner iterations in the CPU sample")
    ap.add_argument("--arms", default="all", choices=["all", "none"])
    ap.add_argument("--collect", type=int, default=48, help="steps before the common point of the arms")
    ap.add_argument("--skip", type=int, default=16, help="first steps (initial transient) not used for training")
    ap.add_argument("--train-steps", type=int, default=600)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--subbox-pairs", type=int, default=2000,
                    help="also train the learned guess on this many (history, converged level) pairs of a seeded run of "
                         "a 64 x Ny x 64 sub-box of the channel with its cell sizes (0: off), and add arms with it")
    ap.add_argument("--subbox-train-steps", type=int, default=2000)
    ap.add_argument("--tight-drop", type=float, default=1e-9,
                    help="stopping rule of the arms' second matrix: the drop under which the converged state no "
                         "longer depends on the predictor or the sweep precision")
    ap.add_argument("--tight-cap", type=int, default=200)
    ap.add_argument("--truth-drop", type=float, default=1e-11, help="the arms' reference run (FP64)")
    ap.add_argument("--truth-cap", type=int, default=250)
    ap.add_argument("--extras", action=argparse.BooleanOptionalAction, default=True,
                    help="after the timed region, also run the 384x256x256 mixed-precision profile check and the "
                         "wavy-wall workload (the line's `extras`)")
    ap.add_argument("--extras-steps", type=int, default=100, help="steps of the 384x256x256 profile check")
    ap.add_argument("--profile-check", type=int, default=0, metavar="STEPS",
                    help="instead of timing: run FP64 and mixed STEPS steps each and compare the mean streamwise "
                         "velocity profiles over x, z and the steps (the mixed-precision acceptance criterion of the 384x256x256 channel: 0.5 %%)")
    return ap.parse_args()


# --------------------------------------------------------------- plumbing
class Dist:
    """One process per GPU (RANK / LOCAL_RANK / WORLD_SIZE from the launcher).
    The replicas share no data; the process group only carries the barriers
    around the timed region and the max / sum of the timings.  backend
    "nccl" on GPUs; "gloo" (CPU tensors) runs the same plumbing without a
    GPU, as the tests do."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self.device = "cuda" if backend == "nccl" else "cpu"
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            # a short timeout: a rank that never arrives ends the others'
            # next collective with an error instead of a hang
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist
            self.torch = torch

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if not self.dist:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.dist:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None


def aggregate(dist: Dist, ms: float, cells_steps: float) -> tuple[float, float]:
    """Whole-job throughput of the replicas: the cell-steps of all ranks over
    the slowest rank's device time.  Returns (max ms, Mcell-steps/s)."""
    ms_max = dist.max(ms)
    total = dist.sum(cells_steps)
    return ms_max, total / (ms_max / 1e3) / 1e6


class Clocks:
    """Samples nvidia-smi every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def launches_per_iteration(ch) -> int:
    """Kernels of one fused LU-SGS inner iteration: x halo, Y and Z boundaries,
    three fluxes, three viscous kernels, the residual, four (halo products +
    wavefront pass) pairs, the update and the norm reduction; an open slab
    adds the X boundary and the sponge target reduction and drops the x halo.
    A step adds the bulk-flux pair and the time-level shift."""
    return 21 + (1 if ch.x_open else 0)


def workload_label(ch) -> str:
    if ch.x_open:
        return (f"open channel {ch.nx}x{ch.ny}x{ch.nz} cells (the reference's own configuration: inflow / outflow, "
                f"sponges of {ch.nx_inlet} and {ch.nx_outlet} cells, lower wall {ch.twall_lo} K between them, "
                f"{'buoyancy' if ch.buoyancy else 'uniform force'}), Mach 0.2, Re_b 5600")
    if ch.wavy:
        return f"wavy-wall channel {ch.nx}x{ch.ny}x{ch.nz} cells (amplitude {ch.wave} h), Mach 0.2, Re_b 5600"
    return f"channel {ch.nx}x{ch.ny}x{ch.nz} cells, Mach 0.2, Re_b 5600"


def bench_config(a, ch) -> dict:
    """The workload of a bench line, the same object in both arms."""
    return {"workload": workload_label(ch), "cells": ch.cells, "precision": a.precision,
            "inner": f"until every one of the five update norms is below {a.drop:g} of its running maximum over "
                     f"the run (main.cpp:287-297), cap {a.cap}",
            "start": "seeded field", "l2": "inputs larger than L2 (state and records ~0.8 GB per field group)"}


# ------------------------------------------------------------ GPU arm
def run_gpu(a, dist: Dist) -> dict | None:
    from cgli_fu_flow_b200.solver import Solver, FP64, MIXED
    ch = C.workload(a.workload)
    prec = FP64 if a.precision == "fp64" else MIXED
    sol = Solver(ch, prec)
    q0 = ch.initial_conserved()
    sol.init(q0)
    iters = []
    for _ in range(a.warmup):
        sol.step(None, a.drop, a.cap)
    clocks = Clocks(dist.local)
    dist.barrier()
    sol.sweep_time(reset=True)
    sol.event(0)
    clocks.start()
    for _ in range(a.steps):
        it, _ = sol.step(None, a.drop, a.cap)
        iters.append(it)
    sol.event(1)
    ms = sol.elapsed_ms(0, 1)
    sweep_ms, sweep_passes = sol.sweep_time()
    ck = clocks.stop()
    dist.barrier()
    ms_max, value = aggregate(dist, ms, float(ch.cells) * a.steps)
    mean_iters = float(np.mean(iters))

    # per-stage device times of one inner iteration (the roofline kernels)
    stages = sol.profile_stages(reps=2)

    # end to end through the C ABI with host buffers
    e2e = None
    if not a.no_e2e:
        e2e = run_e2e(a, ch, prec, dist)
    sol.close()
    arms = run_arms(a, ch, dist) if a.arms == "all" else None
    if dist.rank != 0:
        return None
    from cgli_fu_flow_b200 import roofline
    # the roofline kernel's mean launch: the wavefront passes of every inner
    # iteration of the timed steps, from events around them in the graph
    roof = roofline.sweep_roofline(ch, sweep_ms / max(sweep_passes, 1), a.precision)
    roof["launches_timed"] = sweep_passes
    out = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "Mcell-steps/s",
        "n_gpus": dist.world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": round(ms_max / a.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if a.precision == "fp64" else "f64 residual / f32 sweeps",
        "data": "synthetic: seeded Poiseuille + 10% uniform perturbation channel (no dataset involved)",
        "config": bench_config(a, ch),
        "parallelism": "replicas" if dist.world > 1 else "single GPU",
        "mean_inner_iterations": round(mean_iters, 2), "inner_iterations": iters,
        "clocks": ck,
        "stage_ms": {k: round(v, 4) for k, v in stages.items()},
        "roofline": roof,
        "roofline_residual": roofline.residual_roofline(ch, stages),
        "gpu_launches": int(sum(launches_per_iteration(ch) * n + 3 for n in iters)),
    }
    if e2e:
        out["e2e"] = e2e
    if arms:
        out["arms"] = arms
    return out


def _timed_steps(sol, a, dist, drop=None, cap=None):
    iters = []
    drop = a.drop if drop is None else drop
    cap = a.cap if cap is None else cap
    dist.barrier()
    sol.event(0)
    for _ in range(a.steps):
        it, _ = sol.step(None, drop, cap)
        iters.append(it)
    sol.event(1)
    ms = dist.max(sol.elapsed_ms(0, 1))
    return ms, iters


PREDICTORS = ("previous level", "extrapolation", "learned")


def run_arms(a, ch, dist) -> dict:
    """Precision x predictor from one common point of a run (module
    docstring): FP64 and mixed precision, each with the previous-level,
    extrapolated and learned initial guess, at the headline stopping rule
    and at the tight rule; plus FP64 with the DP-LUR inner solver.  Every
    arm runs the same W + K steps from the common point; its state after
    them is compared with a reference run converged far below either rule
    (FP64, previous-level guess, `--truth-drop`)."""
    from cgli_fu_flow_b200.cnn import (CNN_FLOP_PER_CELL, CNN_TC_FLOP_PER_CELL, Network, init_params,
                                       physical_levels, scales_from_levels)
    from cgli_fu_flow_b200.solver import FP64, MIXED, Solver
    base = Solver(ch, MIXED)
    base.init(ch.initial_conserved())
    base.set_predictor(1)
    net = Network(ch.nx, ch.ny, ch.nz)
    net.reserve_levels(a.collect - a.skip)
    net.set_params(init_params(0))
    # scales from the first and the last quadruple of the training levels
    quads = sorted({a.skip, max(a.skip, a.collect - 4)})
    keep = {k for q in quads for k in range(q, q + 4)}
    host = {}
    t0 = time.perf_counter()
    for k in range(a.collect):
        base.step(None, a.drop, a.cap)
        if k >= a.skip:
            net.push_level(base)
            if k in keep:
                host[k] = physical_levels(base, np.float32)
    collect_s = time.perf_counter() - t0
    sc = [scales_from_levels([host[k] for k in range(q, q + 4)]) for q in quads]
    net.set_scales(*[np.mean([x[i] for x in sc], axis=0) for i in range(len(sc[0]))])
    del host
    npairs = net.levels - 3
    ntrain = max(1, npairs - 4)       # the last four pairs are held out
    t0 = time.perf_counter()
    loss = net.train(a.train_steps, a.lr, 20261203, 0, ntrain)
    train_s = time.perf_counter() - t0
    held = float(np.mean([net.pair_loss(p) for p in range(ntrain, npairs)]))
    out = {"common_point": f"after {a.collect} steps from the seeded field (mixed precision, extrapolated guess, "
                           f"headline rule)",
           "steps_per_arm": f"{a.warmup} untimed + {a.steps} timed",
           "learned_guess": {"training_pairs": ntrain, "training_steps_of_run": [a.skip, a.collect],
                             "adam_steps": a.train_steps, "lr": a.lr,
                             "final_mean_loss": round(loss, 5), "held_out_loss_last_4_pairs": round(held, 5),
                             "collect_s": round(collect_s, 2), "train_s": round(train_s, 2),
                             "loss_unit": "mean squared extrapolation correction / its RMS (1.0 = extrapolation)"}}
    sl = (slice(None), slice(3, ch.nx + 3), slice(2, ch.ny + 2), slice(2, ch.nz + 2))
    net_box = None
    if a.subbox_pairs > 0 and ch.nx % 64 == 0 and ch.nz % 64 == 0:
        net_box, out["learned_guess_subbox"] = train_on_subbox(a, ch)

    def run(prec, pred, drop, cap, inner="lusgs", learned=None):
        s = Solver(ch, prec)
        s.copy_state_from(base)
        if pred == 2:
            s.set_learned_guess(learned or net)
        s.set_predictor(pred)
        if inner == "dplur":
            s.set_inner_solver("dplur")
        for _ in range(a.warmup):
            s.step(None, drop, cap)
        ms, iters = _timed_steps(s, a, dist, drop, cap)
        value = dist.sum(float(ch.cells) * a.steps) / (ms / 1e3) / 1e6
        res = {"value": round(value, 3), "unit": "Mcell-steps/s", "ms_per_step": round(ms / a.steps, 3),
               "mean_inner_iterations": round(float(np.mean(iters)), 2), "inner_iterations": iters,
               "precision": "fp64" if prec == FP64 else "mixed", "predictor": PREDICTORS[pred],
               "inner_solver": "DP-LUR (DPLUSGS.cpp: 4 Jacobi relaxations; norms of squared "
                               "p, u, v, w, T increments)" if inner == "dplur" else "LU-SGS"}
        if pred == 2:
            inf_ms = (learned or net).time_inference(s, 3)
            res["inference"] = {"ms": round(inf_ms, 3),
                                "tensor_tflops": round(ch.cells * CNN_TC_FLOP_PER_CELL / (inf_ms / 1e3) / 1e12, 1),
                                "real_tflops": round(ch.cells * CNN_FLOP_PER_CELL / (inf_ms / 1e3) / 1e12, 1)}
        q = s.q()[sl]
        s.close()
        return res, q

    def rel(q, ref):
        return max(float(np.linalg.norm(q[v] - ref[v]) / np.linalg.norm(ref[v])) for v in range(5))

    truth, q_truth = run(FP64, 0, a.truth_drop, a.truth_cap)
    out["truth"] = {"rule": f"drop {a.truth_drop:g}, cap {a.truth_cap}", "precision": "fp64",
                    "predictor": "previous level", "mean_inner_iterations": truth["mean_inner_iterations"],
                    "inner_iterations": truth["inner_iterations"]}
    for rule, drop, cap in (("headline", a.drop, a.cap), ("tight", a.tight_drop, a.tight_cap)):
        arms = {"rule": f"every norm below {drop:g} of its running maximum, cap {cap}"}
        qs = {}
        # the full matrix at the headline rule; at the tight rule the FP64
        # path and the mixed path with either guess
        matrix = [(p, g) for p in (FP64, MIXED) for g in (0, 1, 2)] if rule == "headline" else \
            [(FP64, 0), (MIXED, 1), (MIXED, 2)]
        for prec, pred in matrix:
            name = f"{'fp64' if prec == FP64 else 'mixed'}_{['previous', 'extrapolation', 'learned'][pred]}"
            arms[name], qs[name] = run(prec, pred, drop, cap)
        if rule == "headline":
            arms["fp64_dplur"], qs["fp64_dplur"] = run(FP64, 0, drop, cap, "dplur")
        if net_box is not None:
            arms["mixed_learned_subbox"], qs["mixed_learned_subbox"] = run(MIXED, 2, drop, cap, learned=net_box)
            arms["mixed_learned_subbox"]["predictor"] = "learned (trained on the sub-box run)"
        for name, q in qs.items():
            arms[name]["state_rel_l2_vs_truth"] = rel(q, q_truth)
            arms[name]["state_rel_l2_vs_fp64_previous"] = rel(q, qs["fp64_previous"])
        base_v = arms["fp64_previous"]["value"]
        arms["speedup_vs_fp64_previous"] = {n: round(arms[n]["value"] / base_v, 3)
                                            for n in qs if n != "fp64_previous"}
        out[rule] = arms
    base.close()
    net.close()
    if net_box is not None:
        net_box.close()
    return out


def train_on_subbox(a, ch):
    """The learned guess trained on `a.subbox_pairs` pairs: a seeded run of a
    periodic 64 x Ny x 64 sub-box of the channel with the same cell sizes and
    time step (mixed precision, extrapolated guess, headline rule) stores
    skip + pairs + 3 converged levels on the device, the network of the
    sub-box trains on all its pairs, and its parameters and scales go to a
    network of the full grid (the network is convolutional: its weights do
    not depend on the grid).  Returns (network, training record)."""
    from cgli_fu_flow_b200.cnn import Network, init_params, physical_levels, scales_from_levels
    from cgli_fu_flow_b200.solver import MIXED, Solver
    sub = C.Channel(64, ch.ny, 64, lx_scale=64 / ch.nx, lz_scale=64 / ch.nz)
    s = Solver(sub, MIXED)
    s.init(sub.initial_conserved())
    s.set_predictor(1)
    nlev = a.subbox_pairs + 3
    nb = Network(sub.nx, sub.ny, sub.nz)
    nb.reserve_levels(nlev)
    nb.set_params(init_params(0))
    quads = [a.skip, a.skip + nlev // 2, a.skip + nlev - 4]
    keep = {k for q in quads for k in range(q, q + 4)}
    host, iters = {}, []
    t0 = time.perf_counter()
    for k in range(a.skip + nlev):
        it, _ = s.step(None, a.drop, a.cap)
        iters.append(it)
        if k >= a.skip:
            nb.push_level(s)
            if k in keep:
                host[k] = physical_levels(s, np.float32)
    collect_s = time.perf_counter() - t0
    sc = [scales_from_levels([host[k] for k in range(q, q + 4)]) for q in quads]
    scales = [np.mean([x[i] for x in sc], axis=0) for i in range(len(sc[0]))]
    nb.set_scales(*scales)
    t0 = time.perf_counter()
    loss = nb.train(a.subbox_train_steps, a.lr, 20261204, 0, a.subbox_pairs)
    train_s = time.perf_counter() - t0
    theta = nb.get_params()
    s.close()
    nb.close()
    full = Network(ch.nx, ch.ny, ch.nz)
    full.set_params(theta)
    full.set_scales(*scales)
    return full, {"workload": f"periodic sub-box {sub.nx}x{sub.ny}x{sub.nz} cells with the channel's cell sizes "
                              f"(Lx x {64 / ch.nx:g}, Lz x {64 / ch.nz:g})",
                  "training_pairs": a.subbox_pairs, "training_steps_of_run": [a.skip, a.skip + nlev],
                  "adam_steps": a.subbox_train_steps, "lr": a.lr, "final_mean_loss": round(float(loss), 5),
                  "mean_inner_iterations_of_run": round(float(np.mean(iters)), 2),
                  "collect_s": round(collect_s, 2), "train_s": round(train_s, 2)}


def run_e2e(a, ch, prec, dist: Dist) -> dict:
    """The same steps through the C ABI with the time levels kept on the host
    in pinned buffers: every step uploads Q^n and Q^(n-1) with
    cgli_set_levels, runs cgli_step, and downloads Q^(n+1) with
    cgli_get_state; the host rotates its three buffers (no host copies)."""
    import torch
    from cgli_fu_flow_b200.solver import Solver, reference_state
    sol = Solver(ch, prec)
    J = sol.get("J")
    U_, U, Uq = reference_state(ch, J, ch.initial_conserved(), ch.initial_conserved())
    shape = (5,) + ch.shape
    pin = [torch.empty(shape, dtype=torch.float64, pin_memory=True) for _ in range(3)]
    buf = [t.numpy() for t in pin]
    buf[0][:] = U
    buf[1][:] = Uq
    sol.set_state(U_, U, Uq)       # a fresh run: the stopping rule's running maxima start here

    def one_step(b):
        sol.set_levels(b[0], b[1])
        sol.step(None, a.drop, a.cap)
        sol.q_into(b[2])
        return [b[2], b[0], b[1]]  # Q^(n+1), Q^n, free

    for _ in range(max(1, min(a.warmup, 2))):
        buf = one_step(buf)
    n = ch.shape[0] * ch.shape[1] * ch.shape[2] * 8
    dist.barrier()
    sol.event(2)
    for _ in range(a.steps):
        buf = one_step(buf)
    sol.event(3)
    ms = dist.max(sol.elapsed_ms(2, 3))
    sol.close()
    value = dist.sum(float(ch.cells) * a.steps) / (ms / 1e3) / 1e6
    return {"value": round(value, 3), "unit": "Mcell-steps/s", "h2d_bytes_per_step": 10 * n,
            "d2h_bytes_per_step": 5 * n}


# ------------------------------------------------------------ CPU reference
def reference_build(ch) -> tuple[str, str] | None:
    """The reference's compiled routines for the workload: the -O3 timing
    build (the reference Makefile's flags) if present, else the pinning
    build; (flavor, path) or None."""
    from oracle import build_ref
    for flavor in ("perf", "pin"):
        path = build_ref.lib_path(ch.name, flavor)
        if os.path.exists(path):
            return flavor, path
    return None


def cpu_reference_sample(ch, iters: int, warm: int = 1) -> dict:
    """Times the reference's own compiled routines (oracle/_ref) on `iters`
    inner iterations of the workload with every host core (OpenMP)."""
    from oracle.refrun import RefSolver
    cores = os.cpu_count() or 1
    flavor, _ = reference_build(ch)
    r = RefSolver(ch, threads=cores, build=False, flavor=flavor)
    r.init()
    for _ in range(warm):
        r.inner_iteration()
    t = time.perf_counter()
    for _ in range(iters):
        r.inner_iteration()
    dt = (time.perf_counter() - t) / iters
    return {"sec_per_inner_iteration": dt, "cores": cores, "build": flavor}


BUILD_NAMES = {"perf": "g++ -O3 -fopenmp, the reference Makefile's optimisation level",
               "pin": "g++ -O2 -fopenmp -ffp-contract=off, the build the oracle is pinned to"}


def run_reference(a, dist: Dist) -> dict | None:
    """The reference's own CPU implementation of the step on the host cores:
    whole physical steps of its compiled routines from the seeded field, each
    iterated with its own stopping rule (main.cpp:287-304: every norm below
    `drop` of its running maximum, cap), W untimed, then K timed by wall
    clock -- the same steps of the same run as the GPU arm's, so the same
    inner-iteration counts."""
    if dist.rank != 0:
        return None
    ch = C.workload(a.workload)
    found = reference_build(ch)
    if found is None:
        return {"impl": "reference", "unavailable": f"reference build for {ch.name} missing (build() compiles it "
                                                    "where the reference sources are present)"}
    flavor, path = found
    from oracle.refrun import RefSolver
    cores = os.cpu_count() or 1
    r = RefSolver(ch, threads=cores, build=False, flavor=flavor)
    r.init()
    warm_iters, iters = [], []
    t0 = time.perf_counter()
    for _ in range(a.warmup):
        it, _ = r.step(None, a.drop, a.cap)
        warm_iters.append(it)
    warm_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    for _ in range(a.steps):
        it, _ = r.step(None, a.drop, a.cap)
        iters.append(it)
    sec = time.perf_counter() - t0
    value = ch.cells * a.steps / sec / 1e6
    sample = (f"{a.steps} whole physical steps (after {a.warmup} untimed) of the reference's routines "
              f"({BUILD_NAMES[flavor]}; OpenMP on {cores} threads; single process, no MPI library here) on the "
              f"{ch.nx}x{ch.ny}x{ch.nz} channel from the seeded field, each iterated to its own stopping rule; "
              f"wall clock")
    return {"impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": "Mcell-steps/s",
            "n_gpus": dist.world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": round(sec / a.steps * 1e3, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic: seeded Poiseuille + 10% uniform perturbation "
                                                         "channel (no dataset involved)",
            "config": bench_config(a, ch), "parallelism": f"host cores (OpenMP, {cores} threads)",
            "mean_inner_iterations": round(float(np.mean(iters)), 2), "inner_iterations": iters,
            "warmup_inner_iterations": warm_iters, "warmup_s": round(warm_s, 1),
            "cpu_baseline": {"value": round(value, 5), "unit": "Mcell-steps/s", "cores": cores,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": round(value, 5), "unit": "Mcell-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_profile_check(ch, steps: int, drop: float, cap: int) -> dict:
    """Mean streamwise velocity profile of mixed precision against FP64 on
    the same workload (each from the seeded field, same stopping rule, on-
    device statistics every step), the final states' relative L2 difference
    and each precision's throughput over the steps (CUDA events)."""
    from cgli_fu_flow_b200.solver import FP64, MIXED, Solver
    prof, q, iters, ms = {}, {}, {}, {}
    for name, prec in (("fp64", FP64), ("mixed", MIXED)):
        g = Solver(ch, prec)
        g.init()
        it = []
        g.event(0)
        for _ in range(steps):
            n, _ = g.step(None, drop, cap)
            it.append(n)
            g.accumulate_statistics()
        g.event(1)
        ms[name] = g.elapsed_ms(0, 1)
        prof[name] = g.mean_profiles()["U"]
        sl = (slice(None), slice(3, ch.nx + 3), slice(2, ch.ny + 2), slice(2, ch.nz + 2))
        q[name] = g.q()[sl]
        iters[name] = it
        g.close()
    diff = float(np.abs(prof["mixed"] - prof["fp64"]).max() / ch.u_b)
    rel = [float(np.linalg.norm(q["mixed"][v] - q["fp64"][v]) / np.linalg.norm(q["fp64"][v])) for v in range(5)]
    return {"check": "mean streamwise velocity profile over x, z and the steps: mixed vs FP64 (criterion 0.5 % "
                     "of U_b)", "workload": workload_label(ch), "steps": steps,
            "rule": f"every norm below {drop:g} of its running maximum, cap {cap}",
            "max_profile_difference_over_u_b": diff, "criterion": 0.005, "passed": diff <= 0.005,
            "state_rel_l2_mixed_vs_fp64": max(rel), "state_rel_l2_mixed_vs_fp64_per_variable": rel,
            "mean_inner_iterations": {k: round(float(np.mean(v)), 2) for k, v in iters.items()},
            "value": {k: round(ch.cells * steps / (v / 1e3) / 1e6, 3) for k, v in ms.items()},
            "unit": "Mcell-steps/s (statistics included)"}


def run_wavy(a) -> dict:
    """The curvilinear workload: FP64 and mixed precision on the wavy-wall
    channel, W + K steps each from the seeded field at the headline rule,
    throughput over the K timed steps and the final states' difference."""
    from cgli_fu_flow_b200.solver import FP64, MIXED, Solver
    ch = C.workload("c4")
    out, q = {"workload": workload_label(ch)}, {}
    for name, prec in (("fp64", FP64), ("mixed", MIXED)):
        g = Solver(ch, prec)
        g.init()
        for _ in range(a.warmup):
            g.step(None, a.drop, a.cap)
        it = []
        g.event(0)
        for _ in range(a.steps):
            n, _ = g.step(None, a.drop, a.cap)
            it.append(n)
        g.event(1)
        ms = g.elapsed_ms(0, 1)
        q[name] = g.q()[(slice(None), slice(3, ch.nx + 3), slice(2, ch.ny + 2), slice(2, ch.nz + 2))]
        g.close()
        out[name] = {"value": round(ch.cells * a.steps / (ms / 1e3) / 1e6, 3), "unit": "Mcell-steps/s",
                     "mean_inner_iterations": round(float(np.mean(it)), 2), "inner_iterations": it}
    out["state_rel_l2_mixed_vs_fp64"] = max(float(np.linalg.norm(q["mixed"][v] - q["fp64"][v]) /
                                              np.linalg.norm(q["fp64"][v])) for v in range(5))
    return out


def main():
    a = parse()
    dist = Dist()
    if a.profile_check:
        if dist.rank == 0:
            print(json.dumps(run_profile_check(C.workload(a.workload), a.profile_check, a.drop, a.cap)), flush=True)
        dist.close()
        return
    try:
        if a.impl == "reference":
            out = run_reference(a, dist)
        else:
            out = run_gpu(a, dist)
            if out is not None and not a.no_cpu_baseline and dist.world == 1:
                ch = C.workload(a.workload)
                if reference_build(ch) is not None:
                    smp = cpu_reference_sample(ch, a.cpu_iters)
                    m_it = out["mean_inner_iterations"]
                    v = ch.cells / (smp["sec_per_inner_iteration"] * m_it) / 1e6
                    out["cpu_baseline"] = {
                        "value": round(v, 5), "unit": "Mcell-steps/s", "cores": smp["cores"], "kind": "reference",
                        "sample": f"{a.cpu_iters} inner iterations of the reference's compiled routines on the same "
                                  f"workload ({BUILD_NAMES[smp['build']]}; {smp['sec_per_inner_iteration']:.2f} s "
                                  f"each, OpenMP on {smp['cores']} threads), times the {m_it:g} inner iterations "
                                  f"per step that this run's timed steps needed (the reference needs the same "
                                  f"count: its numerics match to 1e-10)"}
                else:
                    out["cpu_baseline"] = {"value": None, "unit": "Mcell-steps/s", "cores": 0, "kind": "reference",
                                           "sample": "reference build missing"}
            if out is not None and a.extras and dist.world == 1:
                # the other two configurations, after the timed region
                out["extras"] = {"mixed_384x256x256": run_profile_check(C.workload("c3"), a.extras_steps, a.drop,
                                                                         a.cap),
                                 "wavy_256x256x128": run_wavy(a)}
        if out is not None:
            print(json.dumps(out), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
