"""CPU restatement of the running statistics of Statistic.cpp:120-160.

Test infrastructure only (tests/): per interior (i, j) the sums over k of
U, V, W, T, UU, VV, WW, TT, UV, UT, VT of one level U_ (Q/J, reference
layout), with the reference's expressions: U = U2_/U1_ (J cancels),
P = (U5_ - 0.5 U1_ |u|^2)(K - 1) J, T = P / (U1_ R) / J.
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
