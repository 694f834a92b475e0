"""The device side of csrc/zj_math.h on a B200: the reciprocal and square root
start from the hardware's approximate FP64 reciprocal / reciprocal square
root and take two Newton steps (the host side takes its integer seeds and
more steps); both within 2 ulp of numpy's correctly rounded 1/x and sqrt(x),
and x^0.7 within 2 ulp of numpy's x**0.7, on 2^20 log-uniform samples.  The
small harness is compiled here with nvcc for sm_100a."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = r'''
#include <cuda_runtime.h>
#include "zj_math.h"
__global__ void k(int f, const double* x, double* y, long n) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    y[i] = f == 0 ? zj::zj_rcp(x[i]) : f == 1 ? zj::zj_sqrt(x[i]) : zj::zj_pow07(x[i]);
}
extern "C" int run(int f, const double* x, double* y, long n) {
    double *dx = nullptr, *dy = nullptr;
    if (cudaMalloc(&dx, n * 8) != cudaSuccess || cudaMalloc(&dy, n * 8) != cudaSuccess) return 1;
    cudaMemcpy(dx, x, n * 8, cudaMemcpyHostToDevice);
    k<<<(unsigned)((n + 255) / 256), 256>>>(f, dx, dy, n);
    cudaError_t e = cudaMemcpy(y, dy, n * 8, cudaMemcpyDeviceToHost);
    cudaFree(dx); cudaFree(dy);
    return e == cudaSuccess ? 0 : 2;
}
'''


@pytest.fixture(scope="module")
def devmath(tmp_path_factory):
    d = tmp_path_factory.mktemp("zjmath_gpu")
    (d / "m.cu").write_text(SRC)
    so = d / "m.so"
    subprocess.run(["/usr/local/cuda/bin/nvcc", "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
                    "-gencode", "arch=compute_100a,code=sm_100a", "-I",
                    os.path.join(ROOT, "zhijian_b200", "csrc"), str(d / "m.cu"), "-o", str(so)],
                   check=True)
    lib = C.CDLL(str(so))
    lib.run.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_long]
    return lib


def dev(lib, f, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    assert lib.run(f, x.ctypes.data, y.ctypes.data, x.size) == 0
    return y


def ulps(a, b):
    return np.abs(a.view(np.int64) - b.view(np.int64))


def test_device_rcp_sqrt_pow07_within_2ulp(devmath):
    rng = np.random.default_rng(5)
    x = 10.0 ** rng.uniform(-300, 300, 1 << 20)
    x = np.concatenate([x, [1.0, 2.0, 0.5, 3.0, 1.4, 0.01, 100.0, 7.94, 1e-10]])
    assert ulps(dev(devmath, 0, x), 1.0 / x).max() <= 2
    assert ulps(dev(devmath, 1, x), np.sqrt(x)).max() <= 2
    assert ulps(dev(devmath, 2, x), x ** 0.7).max() <= 2
    sp = dev(devmath, 1, np.array([0.0, -1.0, np.inf]))
    assert sp[0] == 0.0 and np.isnan(sp[1]) and sp[2] == np.inf
