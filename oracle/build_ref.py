"""Build recipe for the reference oracle library  oracle/_ref/<name>/libref.so.

Test infrastructure only.  It compiles the reference's own hot-path sources,
read from the reference tree, together with oracle/ref_harness.cpp and the
single-process MPI stub.  Nothing is copied into the repository: each source
is read, the recorded patch list is applied in memory, and the text is piped
to g++ on standard input; only objects and the shared library are written,
and only under oracle/_ref/.

The reference fixes its grid and physics at compile time, so one library is
built per workload from generated stand-ins for Resolution.h, prm.h,
Viscous_terms.h and MPI_prm.h (placed first on the include path; ijk.h and
Mpi_division.h are used as shipped).  The process is presented to the
reference as rank 1 of 3 equal x-slabs (X_out = 3*Nx, np = 3).

Patch list (each replacement must match the stated number of times):
  P4  Jacobian*.cpp:49-50  wall-clustering parameter 2.8 -> workload value
  P5  Y_boundary_condition.cpp:139,166  wall temperatures -> workload values
  P6  Dual_time_stepping.cpp:831  buoyancy -> uniform driving force read
      from the harness (mass-flux controller value)
  P9  Flux_Y.cpp:383-385, Flux_Z.cpp:339-341  the Roe pressure-jump term
      multiplies the never-initialised locals XIx, XIy, XIz; use the face
      unit normal of the routine's own direction (ETx.., ZTx..) instead
  P1-P3 (grid, channel height, viscosity, Pr) come from the generated headers;
  P10 (value-initialised arrays) is the harness's calloc.

Usage:  python oracle/build_ref.py --nx 8 --ny 12 --nz 8 [--name NAME]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF_SRC = os.environ.get("CGLI_REFERENCE_DIR", "/root/reference")

SOURCES = [
    "Jacobian.cpp", "Jacobian_u.cpp", "Jacobian_v.cpp", "Jacobian_w.cpp",
    "Initial_condition.cpp", "X_boundary_condition.cpp", "Y_boundary_condition.cpp",
    "Z_boundary_condition.cpp", "Flux_X.cpp", "Flux_Y.cpp", "Flux_Z.cpp",
    "Viscous_terms.cpp", "Dual_time_stepping.cpp", "Driven_force.cpp", "Hyperplane.cpp",
    "Filter.cpp", "DPLUSGS.cpp", "Statistic.cpp",
]

PATCHES = {
    "Jacobian.cpp": [("double gamma1 = 2.8;", "double gamma1 = CGLI_STRETCH;", 1)],
    "Jacobian_u.cpp": [("double gamma1 = 2.8;", "double gamma1 = CGLI_STRETCH;", 1)],
    "Jacobian_v.cpp": [("double gamma1 = 2.8;", "double gamma1 = CGLI_STRETCH;", 1)],
    "Jacobian_w.cpp": [("double gamma1 = 2.8;", "double gamma1 = CGLI_STRETCH;", 1)],
    "Y_boundary_condition.cpp": [("T = 343.0592;", "T = CGLI_TWALL_LO;", 1),
                                 ("T = 298.0592;", "T = CGLI_TWALL_HI;", 1)],
    "Dual_time_stepping.cpp": [("f = -(rho-1.1842)*9.81;", "f = cgli_ref_buoyancy ? -(rho-1.1842)*9.81 : cgli_ref_force;", 1),
                               ("void Dual_time_stepping",
                                "extern double cgli_ref_force;\nextern int cgli_ref_buoyancy;\nvoid Dual_time_stepping", 1)],
    # DPLUSGS.cpp reads the constant f of prm.h (included in its body); the
    # harness gives it the same driving force as Dual_time_stepping.  Its
    # relaxation loop never assigns j_ and k_ (ijk.h declares them, the
    # OpenMP clause makes them private and uninitialised), so the upper y / z
    # terms would read NL at indeterminate rows; the loop header sets them to
    # j+1 and k+1, the neighbours whose state the same terms use.
    "DPLUSGS.cpp": [("for (k = 2, _k = 1; k < nzz; k++, _k++) {",
                     "for (k = 2, _k = 1, j_ = j + 1, k_ = 3; k < nzz; k++, _k++, k_++) {", 2),("+f/J[i][j][k];", "+cgli_ref_force/J[i][j][k];", 1),
                    ("+f*u/J[i][j][k];", "+cgli_ref_force*u/J[i][j][k];", 1),
                    ("void DPLUSGS", "extern double cgli_ref_force;\nvoid DPLUSGS", 1)],
    "Flux_Y.cpp": [("deltaP*XIx;", "deltaP*ETx;", 1), ("deltaP*XIy;", "deltaP*ETy;", 1),
                   ("deltaP*XIz;", "deltaP*ETz;", 1)],
    "Flux_Z.cpp": [("deltaP*XIx;", "deltaP*ZTx;", 1), ("deltaP*XIy;", "deltaP*ZTy;", 1),
                   ("deltaP*XIz;", "deltaP*ZTz;", 1)],
}

CXXFLAGS = ["-O2", "-fopenmp", "-fPIC", "-w", "-std=gnu++14", "-ffp-contract=off"]
# The timing build ("perf"): the optimisation level of the reference's own
# Makefile (mpicxx -O3, Makefile:9,15) with OpenMP; the pinning build above
# keeps -O2 without contraction so that the C restatement matches it bit for
# bit.  Both compile the same patched sources.
CXXFLAGS_PERF = ["-O3", "-fopenmp", "-fPIC", "-w", "-std=gnu++14"]
FLAVORS = {"pin": CXXFLAGS, "perf": CXXFLAGS_PERF}


def r17(x: float) -> str:
    return repr(float(x))


def gen_headers(cfgdir: str, p: dict) -> None:
    """Periodic slab: rank 1 of 3 equal slabs (X_out = 3 Nx), every routine on
    its interior-rank path.  x_open: a single rank 0 of 1 (X_out = Nx), the
    reference's own inflow/outflow configuration with sponge layers."""
    open_ = bool(p.get("x_open", 0))
    nslab = 1 if open_ else 3
    nx3 = nslab * p["nx"]
    res = f"""/* generated stand-in for Resolution.h: rank {0 if open_ else 1} of {nslab} x-slabs */
#define nx_inlet  {p.get('nx_inlet', 0) if open_ else 0}
#define nx_outlet {p.get('nx_outlet', 0) if open_ else 0}
#define CGLI_NSLAB {nslab}
#define CGLI_MYID {0 if open_ else 1}
#define X_out {nx3}
#define Y_out {p['ny']}
#define Z_out {p['nz']}
#define X_m {nx3 + 4}
#define Y_m {p['ny'] + 4}
#define Z_m {p['nz'] + 4}
#define nx X_out+1
#define ny Y_out+1
#define nz Z_out+1
#define deltaXI {r17(p['dxi'])}
#define deltaET {r17(p['det'])}
#define deltaZT {r17(p['dzt'])}
#define nxx nx+1
#define nyy ny+1
#define nzz nz+1
#define nxxx nxx+1
#define nyyy nyy+1
#define nzzz nzz+1
#define CGLI_STRETCH {r17(p['stretch'])}
#define CGLI_TWALL_LO {r17(p['twall_lo'])}
#define CGLI_TWALL_HI {r17(p['twall_hi'])}
"""
    prm = f"""/* generated stand-in for prm.h */
#define K 1.4
#define R 287
#define minimum 0.0000001
double f = 0.5993;
double Q0 = 2.07;
double Qold = Q0;
double high = {r17(p['high'])};
double psi = 0.001;
"""
    vis = f"""/* generated stand-in for Viscous_terms.h */
#include "prm.h"
#define Cv 717.5
#define mu_L {r17(p['mu'])}
#define Pr_L {r17(p['pr'])}
#define R 287
double Cp = Cv*K;
double lambda_L = mu_L*Cv*K/Pr_L;
"""
    mpi = f"""/* generated stand-in for MPI_prm.h: {nslab} x-slab(s) */
#define np {nslab}
int nproc = np;
int istart, iend, icount, r_nbr, l_nbr, lastp, iroot;
int itag, isrc, idest, istart1, icount1,icount2, istart2, iend1, iend2;
int gstart0[np], gend0[np],gstart[np], gend[np], gcount[np];
double tstart,tend;
MPI_Request l_reqs1,l_reqs2,l_reqs3,l_reqs4,l_reqs5,
            r_reqs1,r_reqs2,r_reqs3,r_reqs4,r_reqs5;
MPI_Request r1,r2,r3,r4,r5,r6,r7,r8,r9,r10;
"""
    os.makedirs(cfgdir, exist_ok=True)
    for name, text in (("Resolution.h", res), ("prm.h", prm), ("Viscous_terms.h", vis), ("MPI_prm.h", mpi)):
        with open(os.path.join(cfgdir, name), "w") as fh:
            fh.write(text)


def patched_source(fname: str) -> str:
    with open(os.path.join(REF_SRC, fname)) as fh:
        text = fh.read()
    for old, new, count in PATCHES.get(fname, []):
        n = text.count(old)
        if n != count:
            raise RuntimeError(f"patch for {fname}: '{old}' found {n} times, expected {count}")
        text = text.replace(old, new)
    return text


def compile_one(fname: str, outdir: str, cfgdir: str, flags: list[str] = CXXFLAGS) -> str:
    obj = os.path.join(outdir, fname.replace(".cpp", ".o"))
    incs = ["-I", cfgdir, "-I", os.path.join(HERE, "mpi_stub"), "-I", REF_SRC]
    if fname == "ref_harness.cpp":
        cmd = ["g++", *flags, *incs, "-c", os.path.join(HERE, fname), "-o", obj]
        subprocess.run(cmd, check=True)
    else:
        cmd = ["g++", *flags, *incs, "-x", "c++", "-c", "-", "-o", obj]
        subprocess.run(cmd, input=patched_source(fname).encode(), check=True)
    return obj


def lib_path(name: str, flavor: str = "pin") -> str:
    """Where build() puts the library of workload `name` (the timing build
    in a directory of its own, <name>_O3)."""
    return os.path.join(HERE, "_ref", name if flavor == "pin" else f"{name}_O3", "libref.so")


def build(params: dict, name: str | None = None, jobs: int = 8, flavor: str = "pin") -> str:
    """Builds (if needed) and returns the path of libref.so for `params`
    (keys nx, ny, nz, dxi, det, dzt, high, mu, pr, stretch, twall_lo, twall_hi,
    and for the open configuration x_open, nx_inlet, nx_outlet).  flavor
    "pin" is the build the oracle is pinned to, "perf" the timing build with
    the reference Makefile's -O3."""
    if not os.path.isdir(REF_SRC):
        raise FileNotFoundError(f"reference sources not found at {REF_SRC}")
    name = name or f"channel_{params['nx']}x{params['ny']}x{params['nz']}"
    flags = FLAVORS[flavor]
    lib = lib_path(name, flavor)
    outdir = os.path.dirname(lib)
    stamp = os.path.join(outdir, "params.json")
    want = json.dumps(dict(params, cxxflags=flags) if flavor != "pin" else params, sort_keys=True)
    deps = [os.path.join(HERE, "ref_harness.cpp"), os.path.join(HERE, "mpi_stub", "mpi.h"),
            os.path.abspath(__file__)]
    if os.path.exists(lib) and os.path.exists(stamp):
        with open(stamp) as fh:
            same = fh.read() == want
        if same and all(os.path.getmtime(d) <= os.path.getmtime(lib) for d in deps):
            return lib
    cfgdir = os.path.join(outdir, "cfg")
    gen_headers(cfgdir, params)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda f: compile_one(f, outdir, cfgdir, flags), SOURCES + ["ref_harness.cpp"]))
    subprocess.run(["g++", "-shared", "-fopenmp", "-o", lib, *objs, "-Wl,--no-undefined", "-lm"], check=True)
    with open(stamp, "w") as fh:
        fh.write(want)
    return lib


def params_for(ch) -> dict:
    """Build parameters of the reference for a Channel workload (the open
    configuration adds its sponge layers; wall temperatures are patched in)."""
    sys.path.insert(0, REPO)
    from cgli_fu_flow_b200.channel import MU0, PR, STRETCH
    params = dict(nx=ch.nx, ny=ch.ny, nz=ch.nz, dxi=ch.dxi, det=ch.det, dzt=ch.dzt, high=ch.high,
                  mu=MU0, pr=PR, stretch=STRETCH, twall_lo=ch.twall_lo, twall_hi=ch.twall_hi)
    if ch.x_open:
        params.update(x_open=1, nx_inlet=ch.nx_inlet, nx_outlet=ch.nx_outlet)
    return params


def channel_params(nx: int, ny: int, nz: int) -> dict:
    sys.path.insert(0, REPO)
    from cgli_fu_flow_b200.channel import Channel
    return params_for(Channel(nx, ny, nz))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, required=True)
    ap.add_argument("--ny", type=int, required=True)
    ap.add_argument("--nz", type=int, required=True)
    ap.add_argument("--name", default=None)
    a = ap.parse_args()
    print(build(channel_params(a.nx, a.ny, a.nz), a.name))
