"""Roofline bookkeeping of the dominant kernel (the wavefront sweep passes).

Algorithmic bytes of one sweep pass per cell, the per-unit figure of the
hot-path scope (compulsory traffic with each array touched once per pass):
the FP64 pass reads Q/J (5), J and nine metric terms (10) and MR or NL (5)
and writes NL or NR (5): 25 doubles = 200 B; with the sweep state, metrics
and MR/NL/NR in float (CGLI_MIXED) the same 25 words are 100 B.  The bound is
HBM bandwidth (no dense contraction); the peak is the measured copy bandwidth
of this GPU type (MEASURED_PEAKS.json, the burst figure, since the pass is
timed alone), else 6650 GB/s, an earlier measurement on the same hardware.
"""
from __future__ import annotations

import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PEAKS = os.path.join(os.path.dirname(HERE), "MEASURED_PEAKS.json")

SWEEP_BYTES_PER_CELL = {"fp64": 25 * 8, "mixed": 25 * 4}

# DRAM bytes (read + write) per cell of one sweep pass from an ncu capture of
# the current k_sweep (16 x 16-column FP64 tiles; dram__bytes_read.sum +
# dram__bytes_write.sum, forward 202 B and backward 250 B per cell, averaged)
# on the 160x128x128 channel; traffic grows with the cell count, so it is
# scaled to the benchmark grid.  The passes read each cell's 16-word record +
# MR slot (the backward pass also its forward result) and write 5 words.  See
# profiles/k_sweep_channel_160x128x128.md.
MEASURED_TRAFFIC_PER_CELL = {"fp64": (202.2 + 250.2) / 2, "mixed": None}


def hbm_peak() -> tuple[float, str]:
    try:
        with open(PEAKS) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def sweep_roofline(ch, pass_ms: float, precision: str) -> dict:
    """pass_ms: mean device time of one wavefront pass."""
    cells = ch.cells
    bpc = SWEEP_BYTES_PER_CELL[precision]
    dur_ms = pass_ms
    achieved = bpc * cells / (dur_ms / 1e3) / 1e9
    peak, kind = hbm_peak()
    tpc = MEASURED_TRAFFIC_PER_CELL.get(precision)
    return {"kernel": "k_sweep (LU-SGS wavefront pass, forward/backward mean)", "bound": "hbm",
            "achieved": round(achieved, 1), "peak": peak, "peak_kind": kind, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": None if tpc is None else int(tpc * cells),
            "algorithmic_bytes_per_launch": bpc * cells, "launch_ms": round(dur_ms, 4)}


# Algorithmic bytes of the residual side of one inner iteration per cell
# (halo and boundaries, the three flux sweeps, the viscous terms and the
# residual assembly together), the per-unit figure of the hot-path scope:
# Q at three time levels (15), J and nine cell metrics (10), three face sets
# of J_f and nine metrics (30), written MR (5): 60 doubles = 480 B.
RESIDUAL_BYTES_PER_CELL = 60 * 8
RESIDUAL_STAGES = ("halo_bc", "flux_x", "flux_y", "flux_z", "viscous", "residual")


# FP64 instructions per cell (thread level) of the residual side's kernels,
# from ncu (sm__inst_executed_pipe_fp64.sum x 32 / cells) on the
# 160x128x128 channel: fluxes 294 / 297 / 377 per face (x / y / z), k_vprim
# 27, viscous faces 279 (channel form), k_viscous_div 24, residual assembly
# 260.  With the FP64 pipe's measured rate on this GPU (a standalone FMA
# probe: 34 TFLOP/s = 17 T FP64 instructions/s) this is a lower bound on the
# side's time.  See profiles/k_flux_k_viscous_k_residual_fast_channel_160x128x128.md.
RESIDUAL_FP64_OPS_PER_CELL = 294 + 297 + 377 + 27 + 279 + 24 + 260
FP64_INST_PER_S = 17.0e12


def residual_roofline(ch, stage_ms: dict) -> dict:
    """stage_ms: device milliseconds per stage of one inner iteration."""
    dur_ms = sum(stage_ms[k] for k in RESIDUAL_STAGES)
    achieved = RESIDUAL_BYTES_PER_CELL * ch.cells / (dur_ms / 1e3) / 1e9
    fp64_ms = RESIDUAL_FP64_OPS_PER_CELL * ch.cells / FP64_INST_PER_S * 1e3
    peak, kind = hbm_peak()
    return {"kernels": "halo/boundaries, k_flux_x/y/z, k_vprim + k_viscous_faces + k_viscous_div, k_residual_fast",
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "peak_kind": kind, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "algorithmic_bytes_per_iteration": RESIDUAL_BYTES_PER_CELL * ch.cells,
            "ms_per_iteration": round(dur_ms, 4),
            "fp64_floor_ms": round(fp64_ms, 4), "fp64_frac": round(fp64_ms / dur_ms, 4)}

