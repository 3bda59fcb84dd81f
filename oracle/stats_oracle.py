"""CPU restatement of the running statistics of Statistic.cpp:120-160.

Test infrastructure only (tests/): per interior (i, j) the sums over k of
U, V, W, T, UU, VV, WW, TT, UV, UT, VT of one level U_ (Q/J, reference
layout), with the reference's expressions: U = U2_/U1_ (J cancels),
P = (U5_ - 0.5 U1_ |u|^2)(K - 1) J, T = P / (U1_ R) / J; and the
instantaneous U, T of the cell at reference index k = 150 (:155-158).
Pinned to the reference's own Statistic() (tests/test_statistics.py).
"""
from __future__ import annotations

import numpy as np

KG, RG = 1.4, 287.0


def sums(U_: np.ndarray, J: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    sl = np.s_[3:nx + 3, 2:ny + 2, 2:nz + 2]
    rho = U_[0][sl]
    u, v, w = U_[1][sl] / rho, U_[2][sl] / rho, U_[3][sl] / rho
    vv = u * u + v * v + w * w
    Jc = J[sl]
    P = (U_[4][sl] - 0.5 * rho * vv) * (KG - 1) * Jc
    T = P / (rho * RG) / Jc
    q = [u, v, w, T, u * u, v * v, w * w, T * T, u * v, u * T, v * T]
    return np.stack([x.sum(axis=2) for x in q])


def primitives(U_: np.ndarray, J: np.ndarray, nx: int, ny: int, nz: int):
    """U, T on the interior cells (Nx, Ny, Nz)."""
    sl = np.s_[3:nx + 3, 2:ny + 2, 2:nz + 2]
    rho = U_[0][sl]
    u, v, w = U_[1][sl] / rho, U_[2][sl] / rho, U_[3][sl] / rho
    vv = u * u + v * v + w * w
    P = (U_[4][sl] - 0.5 * rho * vv) * (KG - 1) * J[sl]
    return u, P / (rho * RG) / J[sl]


def samples(U_: np.ndarray, J: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    """(2, Nx, Ny): U and T of the cell at reference index k = 150 (zero when
    the slab has no such cell, Nz < 149)."""
    out = np.zeros((2, nx, ny))
    if nz >= 149:
        u, T = primitives(U_, J, nx, ny, nz)
        out[0], out[1] = u[:, :, 148], T[:, :, 148]
    return out
