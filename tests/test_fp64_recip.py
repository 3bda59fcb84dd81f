"""The residual side's FP64 reciprocals and square roots are Newton-refined
hardware seeds (cgli_dev.cuh nr_rcp / nr_sqrt) rather than IEEE-rounded
division and sqrt.  This checks them on the GPU against CUDA's IEEE results:
at most one unit in the last place over 2^24 log-uniform operands in each
range the solver forms (state and sound-speed magnitudes, metric norms and
face Jacobians of the seeded grids, and a wide range around them)."""
import ctypes
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


@pytest.fixture(scope="module")
def check_lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("fp64") / "libfp64check.so"
    subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-shared",
                    "-Xcompiler", "-fPIC", "-I", os.path.join(REPO, "cgli_fu_flow_b200", "csrc"),
                    os.path.join(HERE, "csrc", "fp64_recip_check.cu"), "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    lib.fp64_recip_check.argtypes = [ctypes.c_longlong, ctypes.c_ulonglong, ctypes.c_double, ctypes.c_double,
                                     ctypes.POINTER(ctypes.c_longlong)]
    return lib


@pytest.mark.gpu
@pytest.mark.parametrize("lo,hi", [(1e-3, 1e3), (1e3, 1e7), (1e-12, 1e12), (1e-300, 1e300)])
def test_newton_reciprocal_and_sqrt_within_one_ulp(check_lib, lo, hi):
    worst = (ctypes.c_longlong * 2)()
    assert check_lib.fp64_recip_check(1 << 24, 12345, lo, hi, worst) == 0
    print(f"[{lo:.0e}, {hi:.0e}): reciprocal {worst[0]} ulp, sqrt {worst[1]} ulp")
    assert worst[0] <= 1 and worst[1] <= 1
