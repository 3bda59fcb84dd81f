"""CPU restatement of the reference's high-order filter sensor, Filter.cpp:12-1720.

Test infrastructure only: imported by tests/ and tests/golden/make_golden.py
as the expected values for the CUDA filter kernels, never by the product.

numpy float64, every expression evaluated in the order Filter.cpp writes it
(numpy does not fuse multiply-adds), so the result is bit-identical to the
reference compiled with -ffp-contract=off.  Arrays are in the reference
layout [X_np][Y_m][Z_m] (X_np = Nx+6, Y_m = Ny+4, Z_m = Nz+4); `ny`, `nz`
below are the reference's `ny = Y_out+1`, `nz = Z_out+1` (Resolution.h:16-17)
and `gend` = Nx+2, the last interior x plane of the single periodic slab.

What the sensor computes (per scale s in {h, 2h}):
  * six filter levels L1..L6, each an x pass, a y pass on the stretched grid
    and a z pass (Filter.cpp:143-754 for h, :821-1429 for 2h); level 3 is
    exchanged periodically in x before level 4 (:431-466, :1105-1139);
  * the high-pass fU = 6 L1 - 15 L2 + 20 L3 - 15 L4 + 6 L5 - L6 (:769, :1444);
  * E_s = |u - u_filtered|^2 per cell (:796-800, :1471-1475), ghosts in y and
    z copied from the nearest interior cell (:1521-1552);
  * per face Ep = E_high if (E_h sum)/(E_2h sum) over the two cells of the
    face >= Roe_criterion, else E_low (:1563-1645).
Only the momentum components feed E, so the energy variable U5 (which the
reference filters too, without using the result) is not filtered here.

Ghost semantics reproduced from the reference: every scratch array starts
as a copy of U_ (Filter.cpp:121-138) and the passes only overwrite j=2..ny,
k=2..nz, so the y pass reads U_ at the wall rows j=1, nyy and the z pass
reads U_ at k=1, nzz on every level.

The two x-end faces of EpX (i = 2 and i = gend) read E at planes 2 and
gend+1, which the reference sets only on the first and last MPI rank
(Filter.cpp:1486-1512) and leaves unset on every other rank.  On the single
periodic slab they are defined here as the periodic images (E[2] = E[gend],
E[gend+1] = E[3]) when x_ends="periodic", and left as NaN (so that those two
faces are excluded from comparisons) when x_ends=None.
"""
from __future__ import annotations

import numpy as np

# (x/z weights, y weights) of the two scales: h uses (1,6,1)/8 with the
# y pass 0.125*(2b/a, 6, 2c/a); 2h uses (1,2,1)/4 with 0.5*(b/a, 1, c/a)
SCALES = ("h", "2h")
HIGH_PASS = (6.0, -15.0, 20.0, -15.0, 6.0, -1.0)


def level_ranges(nx: int) -> list[tuple[int, int]]:
    """x-plane ranges [i0, i1] of the six levels on an interior rank
    (Filter.cpp:146-153, 174-183, 212-221, 345-349, 474-481, 571-578, 670-674)."""
    g = nx + 2
    return [(1, g + 2), (2, g + 1), (3, g), (1, g + 2), (2, g + 1), (3, g)]


def _x_pass(scale, P, out, i0, i1, ny, nz):
    sl = np.s_[2:ny + 1, 2:nz + 1]
    a, b, c = P[i0 - 1:i1, 2:ny + 1, 2:nz + 1], P[i0:i1 + 1, 2:ny + 1, 2:nz + 1], P[i0 + 1:i1 + 2, 2:ny + 1, 2:nz + 1]
    if scale == "h":
        out[(slice(i0, i1 + 1),) + sl] = 0.125 * (a + 6 * b + c)          # Filter.cpp:160
    else:
        out[(slice(i0, i1 + 1),) + sl] = 0.25 * (a + 2 * b + c)           # Filter.cpp:841


def _y_pass(scale, Gx, out, J, Yp, i0, i1, ny, nz):
    I = slice(i0, i1 + 1)
    K = slice(2, nz + 1)
    jm, jc, jp = slice(1, ny), slice(2, ny + 1), slice(3, ny + 2)
    a = Yp[I, jp, K] - Yp[I, jm, K]                                          # Filter.cpp:187-191
    b = Yp[I, jp, K] - Yp[I, jc, K]
    c = Yp[I, jc, K] - Yp[I, jm, K]
    gm, gc, gp = Gx[I, jm, K], Gx[I, jc, K], Gx[I, jp, K]
    Jm, Jc, Jp = J[I, jm, K], J[I, jc, K], J[I, jp, K]
    if scale == "h":
        out[I, jc, K] = 0.125 * (2 * b / a * gm * Jm + 6 * gc * Jc + 2 * c / a * gp * Jp) / Jc   # :193
    else:
        out[I, jc, K] = 0.5 * (b / a * gm * Jm + gc * Jc + c / a * gp * Jp) / Jc                # :875


def _z_pass(scale, Gy, out, i0, i1, ny, nz):
    I, Jj = slice(i0, i1 + 1), slice(2, ny + 1)
    a, b, c = Gy[I, Jj, 1:nz], Gy[I, Jj, 2:nz + 1], Gy[I, Jj, 3:nz + 2]
    if scale == "h":
        out[I, Jj, 2:nz + 1] = 0.125 * (a + 6 * b + c)                      # Filter.cpp:227
    else:
        out[I, Jj, 2:nz + 1] = 0.25 * (a + 2 * b + c)                       # Filter.cpp:902


def _wrap_x(A, nx):
    """Periodic 3-plane exchange of level 3 on the single slab
    (Filter.cpp:447-466: GG[gend+1..gend+3] <- GG[3..5], GG[0..2] <- GG[gend-2..gend])."""
    g = nx + 2
    A[g + 1:g + 4] = A[3:6]
    A[0:3] = A[g - 2:g + 1]


def velocity_energy(scale: str, U: list[np.ndarray], J: np.ndarray, Yp: np.ndarray, nx: int, ny_cells: int,
                    nz_cells: int) -> np.ndarray:
    """E_s on the interior cells (NaN elsewhere), s = "h" or "2h"."""
    ny, nz = ny_cells + 1, nz_cells + 1
    g = nx + 2
    ranges = level_ranges(nx)
    fU = [None] * 4
    prev = [U[v] for v in range(4)]
    for lev in range(6):
        i0, i1 = ranges[lev]
        cur = []
        for v in range(4):
            Gx = U[v].copy()
            Gy = U[v].copy()
            L = U[v].copy()
            _x_pass(scale, prev[v], Gx, i0, i1, ny, nz)
            _y_pass(scale, Gx, Gy, J, Yp, i0, i1, ny, nz)
            _z_pass(scale, Gy, L, i0, i1, ny, nz)
            if lev == 2:
                _wrap_x(L, nx)
            cur.append(L)
            Li = L[3:g + 1, 2:ny + 1, 2:nz + 1]
            term = HIGH_PASS[lev] * Li if lev < 5 else Li
            if lev == 0:
                fU[v] = term
            elif lev < 5:
                fU[v] = fU[v] + term                                         # Filter.cpp:769, left to right
            else:
                fU[v] = fU[v] - term
        prev = cur
    E = np.full(U[0].shape, np.nan)
    I, Jj, K = slice(3, g + 1), slice(2, ny + 1), slice(2, nz + 1)
    u1 = U[0][I, Jj, K]
    Ue = U[1][I, Jj, K] / u1 - fU[1] / fU[0]                                # Filter.cpp:796-800
    Ve = U[2][I, Jj, K] / u1 - fU[2] / fU[0]
    We = U[3][I, Jj, K] / u1 - fU[3] / fU[0]
    E[I, Jj, K] = Ue * Ue + Ve * Ve + We * We
    return E


def fill_ghosts(E: np.ndarray, nx: int, ny_cells: int, nz_cells: int, x_ends: str | None = "periodic") -> None:
    """Filter.cpp:1521-1552 (y then z ghosts of the interior planes), plus
    the x-end planes 2 and gend+1 as described in the module docstring."""
    ny, nz = ny_cells + 1, nz_cells + 1
    g = nx + 2
    I = slice(3, g + 1)
    E[I, 1, 2:nz + 1] = E[I, 2, 2:nz + 1]
    E[I, ny + 1, 2:nz + 1] = E[I, ny, 2:nz + 1]
    E[I, 2:ny + 1, 1] = E[I, 2:ny + 1, 2]
    E[I, 2:ny + 1, nz + 1] = E[I, 2:ny + 1, nz]
    if x_ends == "periodic":
        E[2] = E[g]
        E[g + 1] = E[3]


def face_ratios(Eh: np.ndarray, E2h: np.ndarray, nx: int, ny_cells: int, nz_cells: int):
    """Emax of every face in the reference's EpX/EpY/EpZ index ranges
    (Filter.cpp:1564-1645); NaN outside them."""
    ny, nz = ny_cells + 1, nz_cells + 1
    g = nx + 2
    shape = Eh.shape
    RX, RY, RZ = (np.full(shape, np.nan) for _ in range(3))
    with np.errstate(divide="ignore", invalid="ignore"):
        I = slice(2, g + 1)                       # i = 2..gend
        a, b = np.s_[2:g + 1, 2:ny + 1, 2:nz + 1], np.s_[3:g + 2, 2:ny + 1, 2:nz + 1]
        RX[I, 1:ny, 1:nz] = (Eh[a] + Eh[b]) / (E2h[a] + E2h[b])
        I = slice(2, g)                           # i = 2..gend-1
        a, b = np.s_[3:g + 1, 1:ny + 1, 2:nz + 1], np.s_[3:g + 1, 2:ny + 2, 2:nz + 1]
        RY[I, 1:ny + 1, 1:nz] = (Eh[a] + Eh[b]) / (E2h[a] + E2h[b])
        a, b = np.s_[3:g + 1, 2:ny + 1, 1:nz + 1], np.s_[3:g + 1, 2:ny + 1, 2:nz + 2]
        RZ[I, 1:ny, 1:nz + 1] = (Eh[a] + Eh[b]) / (E2h[a] + E2h[b])
    return RX, RY, RZ


def face_masks(nx: int, ny_cells: int, nz_cells: int, shape, x_ends: str | None = "periodic"):
    """Boolean masks of the faces each Ep array defines; with x_ends=None the
    two EpX end faces that read unset planes are left out."""
    ny, nz = ny_cells + 1, nz_cells + 1
    g = nx + 2
    MX, MY, MZ = (np.zeros(shape, bool) for _ in range(3))
    MX[2:g + 1, 1:ny, 1:nz] = True
    if x_ends is None:
        MX[2] = False
        MX[g] = False
    MY[2:g, 1:ny + 1, 1:nz] = True
    MZ[2:g, 1:ny, 1:nz + 1] = True
    return MX, MY, MZ


def sensor(U: list[np.ndarray], J: np.ndarray, Yp: np.ndarray, nx: int, ny_cells: int, nz_cells: int,
           x_ends: str | None = "periodic"):
    """(RX, RY, RZ): the face ratios Emax whose comparison with Roe_criterion
    gives EpX/EpY/EpZ."""
    Eh = velocity_energy("h", U, J, Yp, nx, ny_cells, nz_cells)
    E2h = velocity_energy("2h", U, J, Yp, nx, ny_cells, nz_cells)
    fill_ghosts(Eh, nx, ny_cells, nz_cells, x_ends)
    fill_ghosts(E2h, nx, ny_cells, nz_cells, x_ends)
    return face_ratios(Eh, E2h, nx, ny_cells, nz_cells)


def filter_ep(U, J, Yp, nx, ny_cells, nz_cells, roe_criterion, e_high, e_low, x_ends="periodic"):
    """EpX, EpY, EpZ (Filter.cpp:1575-1640): E_high where the ratio is
    >= roe_criterion, E_low where it is not (NaN ratios compare false);
    faces outside the defined ranges are 0."""
    R = sensor(U, J, Yp, nx, ny_cells, nz_cells, x_ends)
    M = face_masks(nx, ny_cells, nz_cells, U[0].shape, x_ends)
    out = []
    for r, m in zip(R, M):
        ep = np.zeros(U[0].shape)
        with np.errstate(invalid="ignore"):
            ep[m] = np.where(r[m] >= roe_criterion, e_high, e_low)
        out.append(ep)
    return out, R, M
