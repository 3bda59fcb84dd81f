"""ctypes wrapper for the C restatement oracle (oracle/cgli_oracle.c).

Test infrastructure only (tests/, __graft_entry__.smoke(), bench.py's
CPU-baseline leg).  `build()` compiles the C file into oracle/_build/.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
SRC = os.path.join(HERE, "cgli_oracle.c")


def build() -> str:
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-o", LIB, SRC, "-lm"],
                       check=True)
    return LIB


class _Params(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dxi", ctypes.c_double), ("det", ctypes.c_double), ("dzt", ctypes.c_double),
                ("dt", ctypes.c_double), ("e", ctypes.c_double),
                ("mu", ctypes.c_double), ("pr", ctypes.c_double),
                ("twall_lo", ctypes.c_double), ("twall_hi", ctypes.c_double),
                ("force", ctypes.c_double), ("curved_walls", ctypes.c_int),
                ("x_open", ctypes.c_int), ("nx_inlet", ctypes.c_int), ("nx_outlet", ctypes.c_int),
                ("buoyancy", ctypes.c_int)]


_lib = None


def _load():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(build())
        L.or_create.restype = ctypes.c_void_p
        L.or_create.argtypes = [ctypes.POINTER(_Params)]
        L.or_destroy.argtypes = [ctypes.c_void_p]
        L.or_array.restype = ctypes.POINTER(ctypes.c_double)
        L.or_array.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.or_metrics.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        L.or_initial.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.or_set_force.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.or_bulk_flux.restype = ctypes.c_double
        L.or_bulk_flux.argtypes = [ctypes.c_void_p]
        for name in ("or_halo_x", "or_bc_y", "or_bc_x", "or_bc_z", "or_flux_x", "or_flux_y", "or_flux_z",
                     "or_viscous", "or_dts_residual", "or_dplur_residual", "or_sweeps", "or_end_step"):
            getattr(L, name).argtypes = [ctypes.c_void_p]
        L.or_update.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.or_inner_iteration.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.or_dplur_sweeps.argtypes = [ctypes.c_void_p]
        L.or_dplur_update.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.or_dplur_inner_iteration.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        _lib = L
    return _lib


def load_wavy_metrics(array, ch) -> None:
    """Overwrites the 40 metric arrays with the wavy-wall workload's (the
    workload definition, generated once on the host and fed to the oracle,
    the reference build and the GPU path alike)."""
    from cgli_fu_flow_b200.solver import METRIC_NAMES, channel_metric_host
    for name in METRIC_NAMES:
        array(name)[...] = channel_metric_host(ch, name)


class Oracle:
    """CPU restatement of one slab of the reference solver for one workload."""

    def __init__(self, ch, e: float | None = None, curved_walls: bool | None = None, inner_solver: str = "lusgs"):
        """inner_solver: "lusgs" (Dual_time_stepping) or "dplur" (DPLUSGS)."""
        from cgli_fu_flow_b200 import channel as C
        if inner_solver not in ("lusgs", "dplur"):
            raise ValueError(inner_solver)
        self.inner_solver = inner_solver
        self.C = C
        self.ch = ch
        self.L = _load()
        p = _Params(ch.nx, ch.ny, ch.nz, ch.dxi, ch.det, ch.dzt, ch.dt,
                    C.PRECOND_EPS if e is None else e, C.MU0, C.PR, ch.twall_lo, ch.twall_hi, ch.force_lam,
                    int(ch.wavy if curved_walls is None else curved_walls),
                    int(ch.x_open), ch.nx_inlet, ch.nx_outlet, int(ch.buoyancy))
        self.s = self.L.or_create(ctypes.byref(p))
        self.shape = ch.shape
        self.force = ch.force_lam
        self.ctrl = {}
        self.L.or_metrics(self.s, ch.high, C.STRETCH)
        if ch.wavy:
            load_wavy_metrics(self.array, ch)

    def __del__(self):
        if getattr(self, "s", None):
            self.L.or_destroy(self.s)
            self.s = None

    def array(self, name: str) -> np.ndarray:
        p = self.L.or_array(self.s, name.encode())
        if not p:
            raise KeyError(name)
        n = int(np.prod(self.shape))
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(self.shape)

    def q(self, which: str = "_") -> np.ndarray:
        suffix = {"_": "_", "n": "", "nm1": "q"}[which]
        return np.stack([self.array(f"U{v}{suffix}").copy() for v in range(1, 6)])

    def init(self, q_n: np.ndarray | None = None, q_nm1: np.ndarray | None = None) -> None:
        if q_n is None:
            q_n = self.ch.initial_conserved()
        if q_nm1 is None:
            q_nm1 = q_n
        a = np.ascontiguousarray(q_n, dtype=np.float64)
        b = np.ascontiguousarray(q_nm1, dtype=np.float64)
        self.L.or_initial(self.s, a.ctypes.data, b.ctypes.data)
        self.L.or_set_force(self.s, self.force)

    def call(self, name: str) -> None:
        getattr(self.L, "or_" + name)(self.s)

    def update(self) -> np.ndarray:
        er = np.zeros(5)
        self.L.or_update(self.s, er.ctypes.data)
        return er

    def inner_iteration(self) -> np.ndarray:
        er = np.zeros(5)
        fn = self.L.or_dplur_inner_iteration if self.inner_solver == "dplur" else self.L.or_inner_iteration
        fn(self.s, er.ctypes.data)
        return er

    def bulk_flux(self) -> float:
        return self.L.or_bulk_flux(self.s)

    def end_step(self, update_force: bool = True) -> None:
        qb = self.bulk_flux()
        self.L.or_end_step(self.s)
        if update_force:
            self.force = self.C.force_update(self.ctrl, qb, self.ch)
            self.L.or_set_force(self.s, self.force)

    def predict(self) -> None:
        """Second-order extrapolated initial guess on the interior cells,
        3Q^n - 3Q^(n-1) + Q^(n-2) (2Q^n - Q^(n-1) with one level of history),
        with Q^(n-2) kept on the Python side."""
        ch = self.ch
        sl = np.s_[3:ch.nx + 3, 2:ch.ny + 2, 2:ch.nz + 2]
        hist = getattr(self, "history", 0)
        for v in range(1, 6):
            u_, u, uq = self.array(f"U{v}_"), self.array(f"U{v}"), self.array(f"U{v}q")
            if hist >= 2:
                u_[sl] = 3 * u[sl] - 3 * uq[sl] + self.uqq[v - 1][sl]
            elif hist == 1:
                u_[sl] = 2 * u[sl] - uq[sl]

    def step(self, fixed_iters: int | None = 10, drop: float = 1e-3, cap: int = 30, predictor: int = 0):
        if predictor:
            self.predict()
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
        self.uqq = [self.array(f"U{v}q").copy() for v in range(1, 6)]
        self.end_step()
        self.history = getattr(self, "history", 0) + 1
        return it, er
