"""ctypes driver for the reference oracle library (oracle/_ref/<name>/libref.so).

Test infrastructure only: used by tests/, by the CPU-baseline leg of bench.py
and by tests/golden/make_golden.py.  It reproduces the reference driver loop
of main.cpp:152-420 on top of the harness entry points: inner iterations
until the workload's stopping rule, then the end-of-step block.
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

from . import build_ref


class RefSolver:
    """One reference process (rank 1 of 3, periodic x) for one workload."""

    def __init__(self, ch, threads: int = 0, build: bool = True, inner_solver: str = "lusgs",
                 flavor: str = "pin"):
        """inner_solver: "lusgs" (Dual_time_stepping, the reference's default)
        or "dplur" (DPLUSGS.cpp, the call main.cpp:268-284 leaves commented).
        flavor: "pin" (the build the oracle is pinned to) or "perf" (-O3, the
        reference Makefile's flags, for timing)."""
        if inner_solver not in ("lusgs", "dplur"):
            raise ValueError(inner_solver)
        self.inner_solver = inner_solver
        params = build_ref.params_for(ch)
        if build:
            path = build_ref.build(params, ch.name, flavor=flavor)
        else:
            path = build_ref.lib_path(ch.name, flavor)
        self.path = path
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.ref_array.restype = ctypes.POINTER(ctypes.c_double)
        L.ref_array.argtypes = [ctypes.c_char_p]
        L.ref_init.argtypes = [ctypes.c_char_p, ctypes.c_double, ctypes.c_double]
        L.ref_setup.argtypes = [ctypes.c_double, ctypes.c_double]
        L.ref_load.argtypes = [ctypes.c_char_p]
        L.ref_set_force.argtypes = [ctypes.c_double]
        L.ref_set_buoyancy.argtypes = [ctypes.c_int]
        L.ref_bulk_flux.restype = ctypes.c_double
        L.ref_check_hyperplanes.restype = ctypes.c_long
        L.ref_filter.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.ref_statistic.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        self.ch = ch
        dims = (ctypes.c_int * 6)()
        L.ref_dims(dims)
        self.shape = (dims[3], dims[4], dims[5])
        assert self.shape == ch.shape, (self.shape, ch.shape)
        if threads:
            L.ref_set_threads(threads)
        self.force = ch.force_lam
        self.ctrl = {}

    def init(self, q_n: np.ndarray | None = None, q_nm1: np.ndarray | None = None) -> None:
        """Loads the seeded initial field through the reference's own restart
        reader (Initial_condition.cpp:111-236)."""
        ch = self.ch
        if q_n is None:
            q_n = ch.initial_conserved()
        if q_nm1 is None:
            q_nm1 = q_n
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "initial.bin")
            if ch.x_open:
                ch.write_restart(path, q_n, q_nm1, ranks=1, rank=0)
            else:
                ch.write_restart(path, q_n, q_nm1)
            self.lib.ref_setup(ch.dt, _c().PRECOND_EPS)
            if ch.wavy:
                from .oracle import load_wavy_metrics
                load_wavy_metrics(self.array, ch)
            self.lib.ref_load(path.encode())
        self.lib.ref_set_force(self.force)
        self.lib.ref_set_buoyancy(int(ch.buoyancy))

    def load(self, path: str) -> None:
        """Set-up, then the initial field read from a restart file written
        elsewhere (the reference's own reader, Initial_condition.cpp:111-236)."""
        ch = self.ch
        self.lib.ref_setup(ch.dt, _c().PRECOND_EPS)
        if ch.wavy:
            from .oracle import load_wavy_metrics
            load_wavy_metrics(self.array, ch)
        self.lib.ref_load(path.encode())
        self.lib.ref_set_force(self.force)

    def array(self, name: str) -> np.ndarray:
        """A live view of one reference array, shape (X_np, Y_m, Z_m)."""
        p = self.lib.ref_array(name.encode())
        if not p:
            raise KeyError(name)
        n = int(np.prod(self.shape))
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(self.shape)

    def q(self, which: str = "_") -> np.ndarray:
        suffix = {"_": "_", "n": "", "nm1": "q"}[which]
        return np.stack([self.array(f"U{v}{suffix}").copy() for v in range(1, 6)])

    def inner_iteration(self) -> np.ndarray:
        er = (ctypes.c_double * 5)()
        if self.inner_solver == "dplur":
            self.lib.ref_inner_iteration_dplusgs(er)
        else:
            self.lib.ref_inner_iteration(er)
        return np.array(er[:])

    def end_step(self, update_force: bool = True) -> None:
        qb = self.lib.ref_bulk_flux()
        self.lib.ref_end_step()
        if update_force:
            self.force = _c().force_update(self.ctrl, qb, self.ch)
            self.lib.ref_set_force(self.force)

    def filter(self, y_point: np.ndarray, roe_criterion: float, e_high: float, e_low: float):
        """Filter.cpp on the current U_ with the given Y_point; returns copies
        of EpX, EpY, EpZ."""
        self.array("Y_point")[...] = y_point
        self.lib.ref_filter(roe_criterion, e_high, e_low)
        return [self.array(n).copy() for n in ("EpX", "EpY", "EpZ")]

    def statistic(self, step: int, statistic_step: int, planes: list[int]) -> dict | None:
        """Statistic.cpp on the current U_ (call after each step).  On every
        statistic_step-th step the reference writes, for up to five x planes,
        the means over k and the accumulated steps of U, V, W, T, UU, VV, WW,
        TT, UV, UT, VT and the instantaneous U, T at k = 150; returns
        {plane i: array (13, Ny)} then, None otherwise.  Planes are the
        slab's interior indices i = 3 .. Nx+2 (periodic slab only)."""
        assert not self.ch.x_open and len(planes) <= 5
        nx, ny = self.ch.nx, self.ch.ny
        # the reference finds plane i where (ii-2) dx <= obs <= (ii-1) dx with
        # ii = i + gstart of this rank (rank 1 of 3 equal slabs: gstart = Nx)
        obs = [(i + nx - 1.5) * self.ch.dxi for i in planes] + [-1e30] * (5 - len(planes))
        cwd = os.getcwd()
        with tempfile.TemporaryDirectory() as td:
            os.chdir(td)
            try:
                self.lib.ref_statistic(step, statistic_step, (ctypes.c_double * 5)(*obs))
            finally:
                os.chdir(cwd)
            out = {}
            for n, i in enumerate(planes, start=1):
                path = os.path.join(td, f"st_obs{n}_{step:05d}.dat")
                if os.path.exists(path):
                    out[i] = np.loadtxt(path).reshape(13, ny)
        return out or None

    def step(self, fixed_iters: int | None = 10, drop: float = 1e-3, cap: int = 30) -> tuple[int, np.ndarray]:
        """One physical step.  fixed_iters=N runs exactly N inner iterations;
        fixed_iters=None iterates until every one of the five update norms,
        divided by its running maximum over the run, is below `drop`, or `cap`."""
        # main.cpp:287-304: norms over their running maximum over the run
        if not hasattr(self, "Emax"):
            self.Emax = np.zeros(5)
        it = 0
        while True:
            it += 1
            er = self.inner_iteration()
            self.Emax = np.maximum(self.Emax, er)
            rel = np.where(self.Emax > 0, er / np.where(self.Emax > 0, self.Emax, 1.0), 0.0)
            if fixed_iters is not None:
                if it >= fixed_iters:
                    break
            elif np.all(rel < drop) or it >= cap:
                break
        self.end_step()
        return it, er


def _c():
    from cgli_fu_flow_b200 import channel
    return channel
