"""Python mirror of the learned initial guess (cgli_cnn_* of the C ABI).

The network predicts the correction of second-order extrapolation of
Q^(n+1) from Q^n, Q^(n-1), Q^(n-2) (architecture in
include/cgli_fu_flow.h); its forward, backward and Adam steps run on the
GPU's tensor cores through libcgli_fu_flow.so.  No CPU fallback.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .solver import CgliError, load_library

CIN = (15, 32, 32, 32, 32)
COUT = (32, 32, 32, 32, 5)


def init_params(seed: int = 0) -> np.ndarray:
    """He-style uniform initialisation of the hidden layers; the output layer
    starts at zero, so the untrained network returns plain extrapolation."""
    rng = np.random.default_rng(seed)
    parts = []
    for l, (ci, co) in enumerate(zip(CIN, COUT)):
        lim = float(np.sqrt(6.0 / (27 * ci))) if l < len(CIN) - 1 else 0.0
        parts.append(rng.uniform(-lim, lim, size=27 * co * ci))
        parts.append(np.zeros(co))
    return np.concatenate(parts).astype(np.float32)


class Network:
    """One network on the current device for one grid (Ny % 4 == 0, Nz % 32 == 0)."""

    def __init__(self, nx: int, ny: int, nz: int):
        self.L = load_library()
        self.dims = (nx, ny, nz)
        self.cells = nx * ny * nz
        h = ctypes.c_void_p()
        self._rc(self.L.cgli_cnn_create(nx, ny, nz, ctypes.byref(h)))
        self.h = h
        self.nparams = int(self.L.cgli_cnn_param_count())

    def _rc(self, rc: int) -> None:
        if rc != 0:
            raise CgliError(rc, self.L.cgli_cnn_last_error().decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.cgli_cnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- parameters
    def set_params(self, theta: np.ndarray) -> None:
        t = np.ascontiguousarray(theta, dtype=np.float32)
        assert t.size == self.nparams
        self._rc(self.L.cgli_cnn_set_params(self.h, t.ctypes.data))

    def get_params(self) -> np.ndarray:
        t = np.zeros(self.nparams, np.float32)
        self._rc(self.L.cgli_cnn_get_params(self.h, t.ctypes.data))
        return t

    def set_scales(self, mean, std, d1, d2, oscale) -> None:
        """Input scales of the level (mean, std) and of its first and second
        time differences (RMS d1, d2); output scale of the correction."""
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (mean, std, d1, d2, oscale)]
        self._rc(self.L.cgli_cnn_set_scales(self.h, *[x.ctypes.data for x in a]))

    # ---- host-data entry points (tests)
    def forward(self, x0: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x0, dtype=np.float32)
        out = np.zeros((5,) + self.dims, np.float32)
        self._rc(self.L.cgli_cnn_forward_host(self.h, x.ctypes.data, out.ctypes.data))
        return out

    def loss_grad(self, x0: np.ndarray, target: np.ndarray):
        x = np.ascontiguousarray(x0, dtype=np.float32)
        t = np.ascontiguousarray(target, dtype=np.float32)
        loss = ctypes.c_float()
        g = np.zeros(self.nparams, np.float32)
        self._rc(self.L.cgli_cnn_loss_grad_host(self.h, x.ctypes.data, t.ctypes.data, ctypes.byref(loss), g.ctypes.data))
        return float(loss.value), g

    # ---- training data and training
    def reserve_levels(self, count: int) -> None:
        self._rc(self.L.cgli_cnn_reserve_levels(self.h, count))

    @property
    def levels(self) -> int:
        return int(self.L.cgli_cnn_levels(self.h))

    def push_level(self, solver) -> None:
        """Store the solver's current level Q^n (call after each step)."""
        self._rc(self.L.cgli_cnn_push_level(self.h, solver.h))

    def push_level_host(self, q: np.ndarray) -> None:
        a = np.ascontiguousarray(q, dtype=np.float32)
        self._rc(self.L.cgli_cnn_push_level_host(self.h, a.ctypes.data))

    def time_inference(self, solver, reps: int = 3) -> float:
        """Mean device ms of one inference on the solver's current levels."""
        ms = ctypes.c_float()
        self._rc(self.L.cgli_cnn_time_inference(self.h, solver.h, reps, ctypes.byref(ms)))
        return float(ms.value)

    def pair_loss(self, pair: int) -> float:
        loss = ctypes.c_float()
        self._rc(self.L.cgli_cnn_pair_loss(self.h, pair, ctypes.byref(loss)))
        return float(loss.value)

    def train(self, steps: int, lr: float, seed: int, first_pair: int, npairs: int) -> float:
        loss = ctypes.c_float()
        self._rc(self.L.cgli_cnn_train(self.h, steps, lr, seed, first_pair, npairs, ctypes.byref(loss)))
        return float(loss.value)


def physical_levels(solver, dtype=np.float64) -> np.ndarray:
    """Q = U*J of the solver's current level on the interior, (5, nx, ny, nz)."""
    ch = solver.ch
    sl = np.s_[3:ch.nx + 3, 2:ch.ny + 2, 2:ch.nz + 2]
    J = solver.get("J")[sl]
    return np.stack([(solver.get(f"U{v}")[sl] * J).astype(dtype) for v in range(1, 6)])


# real multiply-adds per cell of one inference (15->32, 3 x 32->32, 32->5,
# 27 taps) and the ones the tensor cores execute (every layer padded to 32x32)
CNN_FLOP_PER_CELL = 2 * 27 * (15 * 32 + 3 * 32 * 32 + 32 * 5)
CNN_TC_FLOP_PER_CELL = 2 * 27 * 32 * 32 * 5


def scales_from_levels(levels: list[np.ndarray]):
    """Per-variable input scales over the given consecutive levels -- the
    levels' mean and std, the RMS of their first and of their second time
    differences -- and the output scale: the RMS of the extrapolation
    residual over consecutive quadruples.  Returns (mean, std, d1, d2, oscale)."""
    q = np.stack(levels)
    mean = q.mean(axis=(0, 2, 3, 4))
    std = q.std(axis=(0, 2, 3, 4))

    def rms(xs):
        r = np.stack(xs)
        return np.sqrt((r ** 2).mean(axis=(0, 2, 3, 4)))

    d1 = rms([levels[i + 1] - levels[i] for i in range(len(levels) - 1)])
    d2 = rms([(levels[i + 2] - levels[i + 1]) - (levels[i + 1] - levels[i]) for i in range(len(levels) - 2)])
    osc = rms([levels[i + 3] - (3 * levels[i + 2] - 3 * levels[i + 1] + levels[i]) for i in range(len(levels) - 3)])
    pos = lambda a: np.where(a > 0, a, 1.0)
    return mean, pos(std), pos(d1), pos(d2), pos(osc)
