"""Seeded turbulent-channel workloads: physical constants, grid spacings and the
initial field, in the array layout of the reference solver.

The reference hard-wires its case in compile-time headers (Resolution.h,
prm.h, Viscous_terms.h) and starts from a quiescent heated channel
(Initial_condition.cpp:64-97).  The workloads here are the periodic channel
at bulk Mach 0.2 and Re_b = 5600 (Re_b = rho0 * U_b * 2h / mu0, the
Kim-Moin-Moser convention), in the reference's dimensional SI units:

* domain 2*pi*h x 2h x pi*h, uniform in x and z, tanh wall clustering in y
  with the mapping of Jacobian.cpp:76-90 (stretching parameter 2.0);
* air: gamma 1.4, R 287, Cv 717.5, Sutherland viscosity written as in
  Viscous_terms.cpp:527 with mu0 = 1.85e-5 at 298.0592 K, Pr 0.72;
* isothermal walls at T0 on both sides (Y_boundary_condition.cpp:139,166
  with equal temperatures);
* initial field: laminar Poiseuille profile plus uniform-random velocity
  perturbations of +-10 % of U_b from a counter-based generator
  (splitmix64 of seed + 3*cell + component), each component's x-z plane
  mean removed; uniform density and temperature.  Q^n = Q^(n-1).

A workload is named by its cell counts; nothing here depends on a GPU.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, asdict

import numpy as np

GAMMA = 1.4
R_GAS = 287.0
CV = 717.5
T0 = 298.0592
P0 = 101300.0
MU0 = 1.85e-5
PR = 0.72
MACH_B = 0.2
RE_B = 5600.0
STRETCH = 2.0
# e of main.cpp:57, the low-Mach preconditioning floor beta >= e.  The
# reference uses 1e-4 for its near-incompressible heated cavity.  On the Mach
# 0.2 channel at CFL 1 the reference's own pseudo-time iteration diverges
# with 1e-4 (within the first step at 16x24x16), with 1e-3 at 256x192 cells
# and stalls with 1e-2 at 256 wall-normal cells; with 0.1 it converges on
# every workload (about a 1e-3 drop in 30 inner iterations at 256x192 and
# 384x256).  The viscous terms are explicit in pseudo-time
# (Dual_time_stepping.cpp:879-883 leaves the viscous spectral radius out), so
# the floor on the preconditioned sound speed is what keeps the near-wall
# cell Reynolds number of the pseudo-time iteration above one.
PRECOND_EPS = 0.1
SEED = 20261203


def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser (Steele, Lea, Flood 2014) on uint64 arrays."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)).astype(np.uint64)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


@dataclass
class Channel:
    """One channel workload: cell counts plus every derived constant the
    solver, the oracle and the reference build need."""
    nx: int
    ny: int
    nz: int
    cfl: float = 1.0
    seed: int = SEED
    # wavy lower wall yw(x) = wave * h * sin(4 pi x / Lx), blended linearly to
    # the flat upper wall (the curvilinear workload); False: the flat channel
    wavy: bool = False
    wave: float = 0.05
    # the reference's own configuration instead of the periodic channel: x
    # open with characteristic inflow / outflow ghost planes
    # (X_boundary_condition.cpp), sponge layers over the first nx_inlet and
    # the last nx_outlet cells (Dual_time_stepping.cpp:554-664), walls
    # isothermal only between them (Y_boundary_condition.cpp:114), and
    # optionally its buoyancy body force f = -(rho - 1.1842) 9.81
    # (Dual_time_stepping.cpp:831) in place of the controlled uniform force
    x_open: bool = False
    nx_inlet: int = 0
    nx_outlet: int = 0
    buoyancy: bool = False
    twall_lo: float = T0                  # lower / upper wall temperature (K)
    twall_hi: float = T0
    # a periodic sub-box of the channel: Lx and Lz scaled by these factors
    # (1: the full 2 pi h x 2h x pi h channel), e.g. a smaller domain with
    # the full channel's cell sizes for the learned guess's training data
    lx_scale: float = 1.0
    lz_scale: float = 1.0
    # derived (filled in __post_init__)
    rho0: float = field(init=False)
    c0: float = field(init=False)
    u_b: float = field(init=False)
    h: float = field(init=False)
    high: float = field(init=False)
    lx: float = field(init=False)
    lz: float = field(init=False)
    dxi: float = field(init=False)
    det: float = field(init=False)
    dzt: float = field(init=False)
    dt: float = field(init=False)
    force_lam: float = field(init=False)

    def __post_init__(self):
        self.rho0 = P0 / T0 / R_GAS                       # Initial_condition.cpp:75 order
        self.c0 = math.sqrt(GAMMA * R_GAS * T0)
        self.u_b = MACH_B * self.c0
        self.h = 0.5 * RE_B * MU0 / (self.rho0 * self.u_b)
        self.high = 2.0 * self.h                          # prm.h:16 (channel height)
        self.lx = 2.0 * math.pi * self.h * self.lx_scale
        self.lz = math.pi * self.h * self.lz_scale
        self.dxi = self.lx / self.nx                      # deltaXI, metres (xidx = 1)
        self.det = 1.0 / self.ny                          # deltaET, normalised eta
        self.dzt = self.lz / self.nz                      # deltaZT, metres (ztdz = 1)
        self.dt = self.cfl * self.dxi / self.u_b
        self.force_lam = 3.0 * MU0 * self.u_b / (self.h * self.h)

    @property
    def name(self) -> str:
        if self.x_open:
            return f"open_{self.nx}x{self.ny}x{self.nz}_{self.nx_inlet}_{self.nx_outlet}"
        box = "" if self.lx_scale == 1.0 and self.lz_scale == 1.0 else f"_box{self.lx_scale:g}x{self.lz_scale:g}"
        return f"{'wavy' if self.wavy else 'channel'}_{self.nx}x{self.ny}x{self.nz}{box}"

    @property
    def amplitude(self) -> float:
        """Wall-wave amplitude in metres (wave * h), 0 for the flat channel."""
        return self.wave * self.h if self.wavy else 0.0

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def shape(self) -> tuple[int, int, int]:
        """(X_np, Y_m, Z_m): the reference's per-array shape for one x-slab."""
        return (self.nx + 6, self.ny + 4, self.nz + 4)

    @property
    def target_flux(self) -> float:
        return self.rho0 * self.u_b

    def as_dict(self) -> dict:
        return asdict(self)

    # ------------------------------------------------------------------ IC
    def cell_y(self) -> np.ndarray:
        """Wall-normal cell-centre coordinates, the mapping of Jacobian.cpp:77
        evaluated at eta = (j - 1.5) * deltaET for interior j = 2..Ny+1."""
        j = np.arange(2, self.ny + 2, dtype=np.float64)
        g = STRETCH
        eta = (j - 1.5) * self.det
        return (0.5 * self.high) * (1 - 1. / math.tanh(g) * np.tanh(g * (1 - 2 * eta)))

    def y_point(self) -> np.ndarray:
        """Cell-centre y in the reference layout [X_np][Y_m][Z_m], the input
        of the filter's y pass: interior rows from cell_y(), wall ghost rows
        mirrored as Grid.cpp:86-90 writes them (j=1: -y(2); j=nyy:
        y(ny) + 2 y(2)) and z ghosts copied as Grid.cpp:104-111, on every
        x plane of the slab (Grid.cpp:82-83)."""
        X, Y, Z = self.shape
        ny, nz = self.ny + 1, self.nz + 1
        yp = np.zeros((X, Y, Z))
        yp[:, 2:ny + 1, 2:nz + 1] = self.cell_y()[None, :, None]
        yp[:, 1, 2:nz + 1] = -yp[:, 2, 2:nz + 1]
        yp[:, ny + 1, 2:nz + 1] = yp[:, ny, 2:nz + 1] + 2 * yp[:, 2, 2:nz + 1]
        yp[:, 1:ny + 2, 1] = yp[:, 1:ny + 2, 2]
        yp[:, 1:ny + 2, nz + 1] = yp[:, 1:ny + 2, nz]
        return yp

    def line_slope(self) -> np.ndarray:
        """dy/dx of the grid lines eta = const at the interior cell centres,
        shape (Nx, Ny): yw'(x) (1 - Y0(eta) / high) of the wavy-wall mapping
        (cgli_wavy_channel_metrics); zero for the flat channel."""
        if not self.wavy:
            return np.zeros((self.nx, self.ny))
        x = (np.arange(self.nx) + 0.5) * self.dxi
        kx = 4 * math.pi / (self.nx * self.dxi)
        ywp = self.amplitude * kx * np.cos(kx * x)
        y0 = self.cell_y()
        return ywp[:, None] * (1 - y0[None, :] / self.high)

    def initial_primitives(self) -> tuple[np.ndarray, ...]:
        """rho, u, v, w, p on the interior cells, shape (Nx, Ny, Nz)."""
        nx, ny, nz = self.nx, self.ny, self.nz
        y = self.cell_y()
        u_lam = 1.5 * self.u_b * (1.0 - (y / self.h - 1.0) ** 2)
        idx = np.arange(nx * ny * nz, dtype=np.uint64).reshape(nx, ny, nz)
        comps = []
        for c in range(3):
            ctr = np.uint64(self.seed) + np.uint64(3) * idx + np.uint64(c)
            r = (splitmix64(ctr) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
            pert = 0.1 * self.u_b * (2.0 * r - 1.0)
            pert -= pert.mean(axis=(0, 2), keepdims=True)
            comps.append(pert)
        u = u_lam[None, :, None] + comps[0]
        v = comps[1]
        w = comps[2]
        if self.wavy:
            # the laminar profile follows the grid lines eta = const (parallel
            # to the wavy wall next to it): v = u_lam * dy/dx along the line
            v = v + u_lam[None, :, None] * self.line_slope()[:, :, None]
        rho = np.full((nx, ny, nz), self.rho0)
        p = np.full((nx, ny, nz), P0)
        return rho, u, v, w, p

    def initial_conserved(self) -> np.ndarray:
        """(5, Nx, Ny, Nz) physical conserved variables rho, rho u, rho v,
        rho w, E (not divided by J) -- the content of one time level of the
        reference restart file (Initial_condition.cpp:136-221)."""
        rho, u, v, w, p = self.initial_primitives()
        vv = u * u + v * v + w * w
        return np.stack([rho, rho * u, rho * v, rho * w, p / (GAMMA - 1) + 0.5 * rho * vv])

    def write_restart(self, path: str, q_n: np.ndarray, q_nm1: np.ndarray, ranks: int = 3, rank: int = 1) -> None:
        """Writes the reference restart layout for a run presented as rank
        `rank` of `ranks` equal x-slabs: 10 fields [U1..U5 at n, U1..U5 at
        n-1], each of ranks*Nx x Ny x Nz doubles, this slab at x-offset
        rank*Nx."""
        nx, ny, nz = self.nx, self.ny, self.nz
        field = ranks * nx * ny * nz * 8
        with open(path, "wb") as fh:
            fh.truncate(10 * field)          # sparse: only this slab's part is written
            for f in range(10):
                q = q_n if f < 5 else q_nm1
                fh.seek(f * field + rank * nx * ny * nz * 8)
                fh.write(np.ascontiguousarray(q[f % 5], dtype=np.float64).tobytes())


def force_update(state: dict, bulk_flux: float, ch: Channel, kp: float = 0.5, ki: float = 0.05) -> float:
    """Mass-flux controller that holds the bulk flux at rho0*U_b.

    The reference only monitors the bulk flux (Driven_force.cpp:38-71) and
    applies buoyancy (Dual_time_stepping.cpp:831); the workloads replace that
    body force by a uniform x-force F that is updated once per physical step
    from the converged state:  e = Q_t - Q_b,  I += e,
    F = F_lam + (kp*e + ki*I) / dt,  F_lam = 3 mu0 U_b / h^2 (laminar wall
    shear).  `state` carries I between calls; returns the new F."""
    e = ch.target_flux - bulk_flux
    state["I"] = state.get("I", 0.0) + e
    return ch.force_lam + (kp * e + ki * state["I"]) / ch.dt


WORKLOADS = {
    "small": (8, 12, 8),
    "c1": (64, 64, 64),
    "c2": (256, 192, 192),
    "c3": (384, 256, 256),
    "c4": (256, 256, 128),     # with the wavy lower wall (WAVY)
    # profiling case: the channel at 160 x 128 x 128 cells (sweep data of one
    # pass ~0.4 GB, larger than L2; ~3 GB on the device)
    "p1": (160, 128, 128),
    # the reference's own open configuration at the 256 x 192 x 192 size
    # (OPEN): inflow / outflow, sponges, heated lower wall, buoyancy
    "o2": (256, 192, 192),
}
# open-configuration workloads: sponge layers (inlet, outlet cells) in the
# proportions of the reference's Resolution.h (100 and 150 of 650 planes)
OPEN = {"o2": (40, 60)}
# wall amplitude (fraction of h) of the wavy workloads: 0.01, not the 0.05 of
# its description, because the reference's scheme diverges within a few
# steps for amplitudes of 0.02 h and more on this mapping
WAVY = {"c4": 0.01}


def workload(name: str) -> "Channel":
    """The Channel of a named workload (c4 has the wavy lower wall, o2 is the
    open configuration with the reference's heated lower wall, 343.0592 K,
    and buoyancy)."""
    if name in WAVY:
        return Channel(*WORKLOADS[name], wavy=True, wave=WAVY[name])
    if name in OPEN:
        nin, nout = OPEN[name]
        return Channel(*WORKLOADS[name], x_open=True, nx_inlet=nin, nx_outlet=nout, buoyancy=True,
                       twall_lo=343.0592)
    return Channel(*WORKLOADS[name])
