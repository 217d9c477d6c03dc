"""The correctly rounded exp/log/pow of gizmo_b200/csrc/crmath.cuh give the same
bits on the B200 as in the host build that tests/test_crmath.py checks against
exact decimal values.

Both builds start the shorter evaluation of log (and so of pow) from the
platform's own log, which differs between CUDA and the host C library; the
Newton step and the rounding test must still land on the same correctly
rounded double. A small CUDA program built here from the header (with the
flags of the FP64 units: no contraction) evaluates the functions on the
device; it is test scaffolding, not part of the library.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.abspath(os.path.join(HERE, "..", "gizmo_b200", "csrc", "crmath.cuh"))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

DEV_SRC = r"""
#include "%s"
#include <cuda_runtime.h>
__global__ void k_eval(int f, long n, const double *x, const double *y, double *o)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        o[i] = f == 0 ? gz::cr::exp(x[i]) : f == 1 ? gz::cr::log(x[i]) : gz::cr::pow(x[i], y[i]);
}
extern "C" int cr_eval_dev(int f, long n, const double *x, const double *y, double *out)
{
    double *dx = nullptr, *dy = nullptr, *dout = nullptr;
    const size_t b = sizeof(double) * (size_t)n;
    if (cudaMalloc(&dx, b) || cudaMalloc(&dy, b) || cudaMalloc(&dout, b)) return 1;
    cudaMemcpy(dx, x, b, cudaMemcpyHostToDevice);
    cudaMemcpy(dy, y, b, cudaMemcpyHostToDevice);
    k_eval<<<592, 256>>>(f, n, dx, dy, dout);
    cudaMemcpy(out, dout, b, cudaMemcpyDeviceToHost);
    const int err = (int)cudaGetLastError();
    cudaFree(dx); cudaFree(dy); cudaFree(dout);
    return err;
}
"""

HOST_SRC = r"""
#include "%s"
extern "C" void cr_eval_host(int f, long n, const double *x, const double *y, double *out) {
  for (long i = 0; i < n; i++)
    out[i] = f == 0 ? gz::cr::exp(x[i]) : f == 1 ? gz::cr::log(x[i]) : gz::cr::pow(x[i], y[i]);
}
"""


@pytest.fixture(scope="module")
def evals(tmp_path_factory):
    d = tmp_path_factory.mktemp("crmath_dev")
    (d / "dev.cu").write_text(DEV_SRC % HEADER)
    (d / "host.cc").write_text(HOST_SRC % HEADER)
    subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-fmad=false",
                    "-Xcompiler", "-fPIC", "-shared", str(d / "dev.cu"), "-o", str(d / "libdev.so")], check=True)
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-fPIC", "-shared", str(d / "host.cc"), "-o",
                    str(d / "libhost.so")], check=True)
    dev, host = C.CDLL(str(d / "libdev.so")), C.CDLL(str(d / "libhost.so"))
    D = C.POINTER(C.c_double)
    dev.cr_eval_dev.argtypes = [C.c_int, C.c_long, D, D, D]
    dev.cr_eval_dev.restype = C.c_int
    host.cr_eval_host.argtypes = [C.c_int, C.c_long, D, D, D]

    def run(f, x, y=None):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(x if y is None else y, dtype=np.float64)
        a, b = np.empty_like(x), np.empty_like(x)
        assert dev.cr_eval_dev(f, len(x), x.ctypes.data_as(D), y.ctypes.data_as(D), a.ctypes.data_as(D)) == 0
        host.cr_eval_host(f, len(x), x.ctypes.data_as(D), y.ctypes.data_as(D), b.ctypes.data_as(D))
        return a, b
    return run


def test_device_bits_equal_host_bits(evals):
    rng = np.random.default_rng(31)
    n = 200_000
    cases = [
        (0, rng.uniform(-708, 708, n), None),
        (0, rng.uniform(-4, 4, n), None),  # jump factors of the h-iteration
        (0, rng.uniform(-745, -670, n), None),  # results near and below the normal range
        (0, np.ldexp(rng.uniform(-1, 1, n), -rng.integers(0, 60, n)), None),
        (1, np.exp(rng.uniform(-700, 700, n)), None),
        (1, 1 + rng.uniform(-1e-2, 1e-2, n), None),  # count ratios near convergence
        (1, 1 + rng.uniform(-1e-8, 1e-8, n), None),
        (2, np.exp(rng.uniform(-60, 60, n)), np.full(n, 1.0 / 3.0)),
        (2, np.exp(rng.uniform(-30, 5, n)), np.full(n, 3.0)),
        (2, np.exp(rng.uniform(-30, 30, n)), rng.uniform(-8, 8, n)),
    ]
    for f, x, y in cases:
        a, b = evals(f, x, y)
        bad = np.flatnonzero(a.view(np.int64) != b.view(np.int64))
        assert bad.size == 0, (f, x[bad[:5]], a[bad[:5]], b[bad[:5]])
