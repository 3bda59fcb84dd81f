"""Python mirror of the reference solver's per-step interface over the C ABI
of include/cgli_fu_flow.h (libcgli_fu_flow.so, built in this directory).

The method names follow the reference routines (Flux_X, Viscous_terms,
Dual_time_stepping, ...); arrays cross the boundary in the reference layout
[X_np][Y_m][Z_m] as numpy float64.  There is no CPU fallback: constructing a
Solver without the CUDA library or without a GPU raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import channel as C

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcgli_fu_flow.so")

FP64 = 0
MIXED = 1

_ERRORS = {-1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "ESTATE", -5: "EDIVERGED", -6: "ETIMEOUT"}


class CgliError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dxi", ctypes.c_double), ("det", ctypes.c_double), ("dzt", ctypes.c_double),
                ("dt", ctypes.c_double), ("e", ctypes.c_double),
                ("mu", ctypes.c_double), ("pr", ctypes.c_double),
                ("twall_lo", ctypes.c_double), ("twall_hi", ctypes.c_double),
                ("force", ctypes.c_double), ("precision", ctypes.c_int), ("curved_walls", ctypes.c_int),
                ("x_open", ctypes.c_int), ("nx_inlet", ctypes.c_int), ("nx_outlet", ctypes.c_int),
                ("buoyancy", ctypes.c_int), ("high", ctypes.c_double)]


EXPORTS = [
    "cgli_create", "cgli_destroy", "cgli_last_error", "cgli_device_bytes", "cgli_set_array",
    "cgli_get_array", "cgli_channel_metrics", "cgli_set_state", "cgli_get_state", "cgli_halo_x",
    "cgli_y_boundary_condition", "cgli_z_boundary_condition", "cgli_flux_x", "cgli_flux_y",
    "cgli_flux_z", "cgli_viscous_terms", "cgli_dual_time_stepping", "cgli_inner_iteration",
    "cgli_driven_force", "cgli_end_step", "cgli_set_force", "cgli_step", "cgli_hyperplane",
    "cgli_channel_metrics_host", "cgli_profile_stages", "cgli_event_record", "cgli_event_elapsed",
    "cgli_update_norms_noalloc", "cgli_set_predictor", "cgli_filter",
    "cgli_cnn_param_count", "cgli_cnn_create", "cgli_cnn_destroy", "cgli_cnn_last_error", "cgli_cnn_set_params",
    "cgli_cnn_get_params", "cgli_cnn_set_scales", "cgli_cnn_forward_host", "cgli_cnn_loss_grad_host",
    "cgli_cnn_reserve_levels", "cgli_cnn_levels", "cgli_cnn_push_level_host", "cgli_cnn_push_level",
    "cgli_cnn_pair_loss", "cgli_cnn_train", "cgli_set_learned_guess", "cgli_step_norms",
    "cgli_copy_state", "cgli_cnn_time_inference", "cgli_wavy_channel_metrics", "cgli_wavy_channel_metrics_host",
    "cgli_statistics_accumulate", "cgli_statistics_get", "cgli_statistics_reset",
    "cgli_write_restart", "cgli_read_restart", "cgli_write_history", "cgli_read_history",
    "cgli_dplusgs", "cgli_set_inner_solver", "cgli_x_boundary_condition", "cgli_set_levels",
    "cgli_sweep_time", "cgli_set_wait_limit", "cgli_sweep_tile_shape",
]

INNER_SOLVERS = {"lusgs": 0, "dplur": 1}

_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libcgli_fu_flow.so and declares every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: build it with python -m cgli_fu_flow_b200.build")
    L = ctypes.CDLL(path)
    P = ctypes.c_void_p
    D = ctypes.c_double
    DP = ctypes.POINTER(ctypes.c_double)
    L.cgli_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(P)]
    L.cgli_destroy.argtypes = [P]
    L.cgli_last_error.restype = ctypes.c_char_p
    L.cgli_device_bytes.restype = ctypes.c_longlong
    L.cgli_device_bytes.argtypes = [P]
    L.cgli_set_array.argtypes = [P, ctypes.c_char_p, P]
    L.cgli_get_array.argtypes = [P, ctypes.c_char_p, P]
    L.cgli_channel_metrics.argtypes = [P, D, D]
    L.cgli_set_state.argtypes = [P, P, P, P]
    L.cgli_get_state.argtypes = [P, P]
    L.cgli_set_levels.argtypes = [P, P, P]
    L.cgli_sweep_time.argtypes = [P, DP, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
    for n in ("cgli_halo_x", "cgli_y_boundary_condition", "cgli_z_boundary_condition", "cgli_flux_x",
              "cgli_flux_y", "cgli_flux_z", "cgli_viscous_terms", "cgli_end_step"):
        getattr(L, n).argtypes = [P]
    L.cgli_dual_time_stepping.argtypes = [P, DP]
    L.cgli_inner_iteration.argtypes = [P, DP]
    L.cgli_driven_force.argtypes = [P, DP]
    L.cgli_set_force.argtypes = [P, D]
    L.cgli_step.argtypes = [P, ctypes.c_int, D, ctypes.c_int, ctypes.POINTER(ctypes.c_int), DP]
    L.cgli_hyperplane.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, P, ctypes.c_long, P, ctypes.c_long]
    L.cgli_profile_stages.argtypes = [P, ctypes.c_int, DP]
    L.cgli_set_predictor.argtypes = [P, ctypes.c_int]
    L.cgli_set_wait_limit.argtypes = [P, ctypes.c_int]
    L.cgli_sweep_tile_shape.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    L.cgli_filter.argtypes = [P, D, D, D]
    F = ctypes.c_float
    FP = ctypes.POINTER(ctypes.c_float)
    LL = ctypes.c_longlong
    L.cgli_cnn_param_count.restype = LL
    L.cgli_cnn_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(P)]
    L.cgli_cnn_destroy.argtypes = [P]
    L.cgli_cnn_last_error.restype = ctypes.c_char_p
    L.cgli_cnn_set_params.argtypes = [P, P]
    L.cgli_cnn_get_params.argtypes = [P, P]
    L.cgli_cnn_set_scales.argtypes = [P, P, P, P, P, P]
    L.cgli_cnn_forward_host.argtypes = [P, P, P]
    L.cgli_cnn_loss_grad_host.argtypes = [P, P, P, FP, P]
    L.cgli_cnn_reserve_levels.argtypes = [P, ctypes.c_int]
    L.cgli_cnn_levels.argtypes = [P]
    L.cgli_cnn_levels.restype = LL
    L.cgli_cnn_push_level_host.argtypes = [P, P]
    L.cgli_cnn_push_level.argtypes = [P, P]
    L.cgli_cnn_pair_loss.argtypes = [P, LL, FP]
    L.cgli_cnn_train.argtypes = [P, ctypes.c_int, F, ctypes.c_ulonglong, LL, LL, FP]
    L.cgli_set_learned_guess.argtypes = [P, P]
    L.cgli_step_norms.argtypes = [P, P, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.cgli_copy_state.argtypes = [P, P]
    L.cgli_statistics_accumulate.argtypes = [P]
    L.cgli_statistics_get.argtypes = [P, P, ctypes.POINTER(ctypes.c_longlong)]
    L.cgli_statistics_reset.argtypes = [P]
    L.cgli_write_restart.argtypes = [P, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
    L.cgli_read_restart.argtypes = [P, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
    L.cgli_write_history.argtypes = [P, ctypes.c_char_p]
    L.cgli_read_history.argtypes = [P, ctypes.c_char_p]
    L.cgli_cnn_time_inference.argtypes = [P, P, ctypes.c_int, FP]
    L.cgli_update_norms_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P, DP, P]
    L.cgli_event_record.argtypes = [P, ctypes.c_int]
    L.cgli_event_elapsed.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.cgli_channel_metrics_host.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, D, D, D, ctypes.c_char_p, P]
    L.cgli_wavy_channel_metrics.argtypes = [P, D, D, D]
    L.cgli_wavy_channel_metrics_host.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, D, D, D, D, D,
                                                 ctypes.c_char_p, P]
    _lib = L
    return L


def _ptrs(arrs) -> ctypes.Array:
    return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def reference_state(ch: C.Channel, J: np.ndarray, q_n: np.ndarray, q_nm1: np.ndarray):
    """U_, U, Uq in the reference layout as Initial_condition.cpp:56-221 and
    main.cpp:127-141 leave them for an interior slab read from a restart file:
    interior planes filled with the quiescent state over all rows (divided by
    the cell's J, which is zero -- hence inf/nan -- on the outermost ring,
    exactly as in the reference with value-initialised arrays), interior
    cells from the restart data divided by J, x ghost planes zero.  An open
    slab (the first and the last rank) also gets the quiescent state on its
    end planes 2 and Nx+3 (Initial_condition.cpp:57-61)."""
    X, Y, Z = ch.shape
    nx, ny, nz = ch.nx, ch.ny, ch.nz
    U = np.zeros((5, X, Y, Z))
    Uq = np.zeros((5, X, Y, Z))
    T = 298.0592
    P = 101300.0
    rho = P / T / C.R_GAS
    quiet = [rho, rho * 0.0, rho * 0.0, rho * 0.0, P / (C.GAMMA - 1) + 0.5 * rho * 0.0]
    lo, hi = (2, nx + 4) if ch.x_open else (3, nx + 3)
    with np.errstate(divide="ignore", invalid="ignore"):
        for v in range(5):
            U[v, lo:hi] = quiet[v] / J[lo:hi]
            Uq[v, lo:hi] = quiet[v] / J[lo:hi]
            Jint = J[3:nx + 3, 2:ny + 2, 2:nz + 2]
            U[v, 3:nx + 3, 2:ny + 2, 2:nz + 2] = q_n[v] / Jint
            Uq[v, 3:nx + 3, 2:ny + 2, 2:nz + 2] = q_nm1[v] / Jint
    U_ = U.copy()
    return U_, U, Uq


class Solver:
    """One device context for one channel workload."""

    def __init__(self, ch: C.Channel, precision: int = FP64, e: float | None = None):
        self.L = load_library()
        self.ch = ch
        self.shape = ch.shape
        self.n = int(np.prod(self.shape))
        p = Params(ch.nx, ch.ny, ch.nz, ch.dxi, ch.det, ch.dzt, ch.dt,
                   C.PRECOND_EPS if e is None else e, C.MU0, C.PR, ch.twall_lo, ch.twall_hi, ch.force_lam, precision,
                   int(ch.wavy), int(ch.x_open), ch.nx_inlet, ch.nx_outlet, int(ch.buoyancy), ch.high)
        h = ctypes.c_void_p()
        self._rc(self.L.cgli_create(ctypes.byref(p), ctypes.byref(h)))
        self.h = h
        self.force = ch.force_lam
        self.ctrl: dict = {}
        if ch.wavy:
            self._rc(self.L.cgli_wavy_channel_metrics(self.h, ch.high, C.STRETCH, ch.amplitude))
        else:
            self._rc(self.L.cgli_channel_metrics(self.h, ch.high, C.STRETCH))

    def _rc(self, rc: int) -> None:
        if rc != 0:
            raise CgliError(rc, self.L.cgli_last_error().decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.cgli_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        return self.L.cgli_device_bytes(self.h)

    # ----------------------------------------------------------- arrays
    def get(self, name: str) -> np.ndarray:
        out = np.empty(self.shape)
        self._rc(self.L.cgli_get_array(self.h, name.encode(), out.ctypes.data))
        return out

    def set(self, name: str, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == self.shape, (a.shape, self.shape)
        self._rc(self.L.cgli_set_array(self.h, name.encode(), a.ctypes.data))

    def set_state(self, U_: np.ndarray, U: np.ndarray, Uq: np.ndarray) -> None:
        arrs = [np.ascontiguousarray(x[v], dtype=np.float64) for x in (U_, U, Uq) for v in range(5)]
        self._keep = arrs
        self._rc(self.L.cgli_set_state(self.h, _ptrs(arrs[0:5]), _ptrs(arrs[5:10]), _ptrs(arrs[10:15])))

    def init(self, q_n: np.ndarray | None = None, q_nm1: np.ndarray | None = None) -> None:
        """Seeded initial field through the reference's restart semantics."""
        if q_n is None:
            q_n = self.ch.initial_conserved()
        if q_nm1 is None:
            q_nm1 = q_n
        U_, U, Uq = reference_state(self.ch, self.get("J"), q_n, q_nm1)
        self.set_state(U_, U, Uq)
        self.set_force(self.force)

    def q(self) -> np.ndarray:
        out = [np.empty(self.shape) for _ in range(5)]
        self._rc(self.L.cgli_get_state(self.h, _ptrs(out)))
        return np.stack(out)

    def set_levels(self, qn: np.ndarray, qnm1: np.ndarray) -> None:
        """cgli_set_levels: Q^n/J and Q^(n-1)/J, each (5, X_np, Y_m, Z_m)
        contiguous (e.g. pinned), for a host-driven loop."""
        for x in (qn, qnm1):
            assert x.shape == (5,) + self.shape and x.flags.c_contiguous and x.dtype == np.float64
        self._rc(self.L.cgli_set_levels(self.h, _ptrs([qn[v] for v in range(5)]), _ptrs([qnm1[v] for v in range(5)])))

    def q_into(self, out: np.ndarray) -> None:
        """cgli_get_state into a caller's contiguous (5, X_np, Y_m, Z_m) array
        (e.g. pinned host memory), without allocating."""
        assert out.shape == (5,) + self.shape and out.flags.c_contiguous and out.dtype == np.float64
        self._rc(self.L.cgli_get_state(self.h, _ptrs([out[v] for v in range(5)])))

    # ---------------------------------------------------- reference routines
    def halo_x(self):
        self._rc(self.L.cgli_halo_x(self.h))

    def y_boundary_condition(self):
        self._rc(self.L.cgli_y_boundary_condition(self.h))

    def x_boundary_condition(self):
        """X_boundary_condition.cpp (open slab; a no-op on a periodic one)."""
        self._rc(self.L.cgli_x_boundary_condition(self.h))

    def z_boundary_condition(self):
        self._rc(self.L.cgli_z_boundary_condition(self.h))

    def flux_x(self):
        self._rc(self.L.cgli_flux_x(self.h))

    def flux_y(self):
        self._rc(self.L.cgli_flux_y(self.h))

    def flux_z(self):
        self._rc(self.L.cgli_flux_z(self.h))

    def viscous_terms(self):
        self._rc(self.L.cgli_viscous_terms(self.h))

    def dual_time_stepping(self) -> np.ndarray:
        er = (ctypes.c_double * 5)()
        self._rc(self.L.cgli_dual_time_stepping(self.h, er))
        return np.array(er[:])

    def dplusgs(self) -> np.ndarray:
        """DPLUSGS.cpp in place of dual_time_stepping (reads the same inF / vF)."""
        er = (ctypes.c_double * 5)()
        self._rc(self.L.cgli_dplusgs(self.h, er))
        return np.array(er[:])

    def set_inner_solver(self, name: str) -> None:
        """"lusgs" (Dual_time_stepping's sweeps, the default) or "dplur"
        (DPLUSGS's Jacobi relaxations; double precision only)."""
        if name not in INNER_SOLVERS:
            raise ValueError(name)
        self._rc(self.L.cgli_set_inner_solver(self.h, INNER_SOLVERS[name]))

    def inner_iteration(self) -> np.ndarray:
        er = (ctypes.c_double * 5)()
        self._rc(self.L.cgli_inner_iteration(self.h, er))
        return np.array(er[:])

    def event(self, slot: int) -> None:
        """Records CUDA event `slot` on the context's stream."""
        self._rc(self.L.cgli_event_record(self.h, slot))

    def sweep_time(self, reset: bool = False) -> tuple[float, int]:
        """(ms, passes): device time of the wavefront passes of every inner
        iteration since the last reset (events inside the iteration graph)."""
        ms = ctypes.c_double()
        n = ctypes.c_longlong()
        self._rc(self.L.cgli_sweep_time(self.h, ctypes.byref(ms), ctypes.byref(n), int(reset)))
        return ms.value, n.value

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = ctypes.c_float()
        self._rc(self.L.cgli_event_elapsed(self.h, a, b, ctypes.byref(ms)))
        return ms.value

    STAGES = ["halo_bc", "flux_x", "flux_y", "flux_z", "viscous", "residual", "sweep_forward", "sweep_backward"]

    def profile_stages(self, reps: int = 3) -> dict:
        """Mean milliseconds per stage of one fast-path inner iteration."""
        ms = (ctypes.c_double * 8)()
        self._rc(self.L.cgli_profile_stages(self.h, reps, ms))
        return dict(zip(self.STAGES, ms[:]))

    def bulk_flux(self) -> float:
        q = ctypes.c_double()
        self._rc(self.L.cgli_driven_force(self.h, ctypes.byref(q)))
        return q.value

    def set_force(self, f: float) -> None:
        self.force = f
        self._rc(self.L.cgli_set_force(self.h, f))

    def end_step(self, update_force: bool = True) -> None:
        qb = self.bulk_flux()
        self._rc(self.L.cgli_end_step(self.h))
        if update_force:
            self.set_force(C.force_update(self.ctrl, qb, self.ch))

    def set_predictor(self, mode: int) -> None:
        """0: previous time level (reference); 1: second-order extrapolation;
        2: extrapolation plus the learned correction (set_learned_guess)."""
        self._rc(self.L.cgli_set_predictor(self.h, mode))

    def set_wait_limit(self, polls: int) -> None:
        """Polls before a wavefront wait gives up (cgli_set_wait_limit)."""
        self._rc(self.L.cgli_set_wait_limit(self.h, polls))

    def write_restart(self, path: str, global_nx: int | None = None, x_offset: int = 0,
                      history: bool = True) -> None:
        """The reference's LES%05d.bin layout (this slab of a global_nx-plane
        file); with history, also `path + '.history'` (Q^(n-2), force, norm
        maxima, step count)."""
        self._rc(self.L.cgli_write_restart(self.h, path.encode(), global_nx or self.ch.nx, x_offset))
        if history:
            self._rc(self.L.cgli_write_history(self.h, (path + ".history").encode()))

    def read_restart(self, path: str, global_nx: int | None = None, x_offset: int = 0,
                     history: bool = True, ctrl: dict | None = None) -> None:
        self._rc(self.L.cgli_read_restart(self.h, path.encode(), global_nx or self.ch.nx, x_offset))
        if history:
            self._rc(self.L.cgli_read_history(self.h, (path + ".history").encode()))
            import struct
            with open(path + ".history", "rb") as fh:
                self.force = struct.unpack("<8s4i6d", fh.read(72))[5]
        if ctrl is not None:
            self.ctrl = dict(ctrl)

    STATS = ("U", "V", "W", "T", "UU", "VV", "WW", "TT", "UV", "UT", "VT")
    SAMPLES = ("UI", "TI")      # instantaneous U and T at reference index k = 150

    def accumulate_statistics(self) -> None:
        """Adds the current level to the running sums (Statistic.cpp:120-160)."""
        self._rc(self.L.cgli_statistics_accumulate(self.h))

    def statistics(self) -> tuple[np.ndarray, int]:
        """The running sums (11, Nx, Ny) followed by the two instantaneous
        samples (13 rows in all), and the number of accumulated steps."""
        out = np.zeros((len(self.STATS) + len(self.SAMPLES), self.ch.nx, self.ch.ny))
        n = ctypes.c_longlong()
        self._rc(self.L.cgli_statistics_get(self.h, out.ctypes.data, ctypes.byref(n)))
        return out, int(n.value)

    def reset_statistics(self) -> None:
        self._rc(self.L.cgli_statistics_reset(self.h))

    def mean_profiles(self) -> dict:
        """Means over x, z and the accumulated steps, per wall-normal cell:
        the reference's (i, j) means (sums / (steps Nz)) averaged over i."""
        sums, n = self.statistics()
        m = sums[:len(self.STATS)].mean(axis=1) / (max(n, 1) * self.ch.nz)
        return dict(zip(self.STATS, m))

    def copy_state_from(self, other: "Solver") -> None:
        """Continue `other`'s run from its current point (levels, force and
        its controller, norm maxima, history)."""
        self._rc(self.L.cgli_copy_state(self.h, other.h))
        self.force = other.force
        self.ctrl = dict(other.ctrl)

    def step_norms(self) -> np.ndarray:
        """(iterations, 5) norms of every inner iteration of the last step."""
        buf = np.zeros((64, 5))
        n = ctypes.c_int()
        self._rc(self.L.cgli_step_norms(self.h, buf.ctypes.data, 64, ctypes.byref(n)))
        if n.value > 64:
            buf = np.zeros((n.value, 5))
            self._rc(self.L.cgli_step_norms(self.h, buf.ctypes.data, n.value, ctypes.byref(n)))
        return buf[:n.value].copy()

    def set_learned_guess(self, net) -> None:
        """Attach a cgli_fu_flow_b200.cnn.Network (None detaches)."""
        self._rc(self.L.cgli_set_learned_guess(self.h, net.h if net is not None else None))
        self._net = net

    def filter(self, y_point: np.ndarray, roe_criterion: float, e_high: float, e_low: float) -> list[np.ndarray]:
        """Filter.cpp's sensor on the current U_ (cgli_filter): EpX, EpY, EpZ
        in the reference layout."""
        self.set("Y_point", y_point)
        self._rc(self.L.cgli_filter(self.h, roe_criterion, e_high, e_low))
        return [self.get(n) for n in ("EpX", "EpY", "EpZ")]

    def step(self, fixed_iters: int | None = 10, drop: float = 1e-3, cap: int = 30, update_force: bool = True):
        """One physical step on the device (inner loop in C++), then the
        force controller update from the converged bulk flux."""
        it = ctypes.c_int()
        er = (ctypes.c_double * 5)()
        self._rc(self.L.cgli_step(self.h, fixed_iters or 0, drop, cap, ctypes.byref(it), er))
        if update_force:
            # the time-level shift leaves U_ = Q^(n+1): the converged bulk flux
            self.set_force(C.force_update(self.ctrl, self.bulk_flux(), self.ch))
        return it.value, np.array(er[:])


def sweep_tile_shape(precision: int = FP64) -> tuple[int, int]:
    """(ti, tj): the wavefront tile the loaded library was built with for
    passes of the given precision."""
    L = load_library()
    ti, tj = ctypes.c_int(), ctypes.c_int()
    rc = L.cgli_sweep_tile_shape(precision, ctypes.byref(ti), ctypes.byref(tj))
    if rc:
        raise CgliError(rc, L.cgli_last_error().decode())
    return ti.value, tj.value


def hyperplane_lists(nx: int, ny: int, nz: int):
    """Nijk, ijk of Hyperplane.cpp through the C ABI (host only)."""
    L = load_library()
    nijk = np.zeros((nx + 2 + ny + 1 + nz + 1 + 1, 2), dtype=np.int32)
    ijk = np.zeros((nx * ny * nz + 1, 3), dtype=np.int32)
    rc = L.cgli_hyperplane(nx, ny, nz, nijk.ctypes.data, nijk.size, ijk.ctypes.data, ijk.size)
    if rc:
        raise CgliError(rc, L.cgli_last_error().decode())
    return nijk, ijk


METRIC_NAMES = ["J", "J_u", "J_v", "J_w"] + [m + s for m in ("xidx", "xidy", "xidz", "etdx", "etdy", "etdz",
                                                               "ztdx", "ztdy", "ztdz") for s in ("", "_u", "_v", "_w")]


def channel_metric_host(ch: C.Channel, name: str) -> np.ndarray:
    """One metric array from the library's host-side generator (no GPU):
    the reference's channel metrics, or the wavy-wall ones for ch.wavy."""
    L = load_library()
    out = np.empty(ch.shape)
    if ch.wavy:
        rc = L.cgli_wavy_channel_metrics_host(ch.nx, ch.ny, ch.nz, ch.dxi, ch.det, ch.high, C.STRETCH, ch.amplitude,
                                              name.encode(), out.ctypes.data)
    else:
        rc = L.cgli_channel_metrics_host(ch.nx, ch.ny, ch.nz, ch.det, ch.high, C.STRETCH, name.encode(),
                                         out.ctypes.data)
    if rc:
        raise CgliError(rc, L.cgli_last_error().decode())
    return out
