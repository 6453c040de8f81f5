// Self-check of the library's own device arithmetic: the reciprocal, inverse
// cube root and square root of fm_device.cuh (used by the element kernels
// in place of CUDA's division, rcbrt and sqrt) evaluated next
// to CUDA's own operations on the same inputs, so that a test can bound
// their difference in units in the last place.  No reference counterpart
// (the reference computes 1.0 / detJ, pow(6V, 1/3) and sqrt on the host,
// src/femVMSExplicitFluidSolver.cpp:64, 75, 585).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "fm_device.cuh"
#include "fm_internal.hpp"

using namespace fm;

// out[i * 8 + k]: rcp_nr(x), 1.0 / x, rcbrt_nr(x), rcbrt(x), sqrt_nr(x),
// sqrt(x), rcbrt_nr((float)x), rcbrtf((float)x).
__global__ void math_check_kernel(const double* x, int64_t n, double* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = x[i];
    const float f = (float)v;
    double* o = out + i * 8;
    o[0] = rcp_nr(v);
    o[1] = 1.0 / v;
    o[2] = rcbrt_nr(v);
    o[3] = rcbrt(v);
    o[4] = sqrt_nr(v);
    o[5] = sqrt(v);
    o[6] = (double)rcbrt_nr(f);
    o[7] = (double)rcbrtf(f);
  }
}

extern "C" int fm_math_check(const double* x, int64_t n, double* out) {
  if (!x || !out || n <= 0) return fail(FM_ERR_INVALID, "fm_math_check: null array or empty input");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FM_ERR_NODEVICE, "no CUDA device");
  double *dx = nullptr, *dout = nullptr;
  cudaError_t e = cudaMalloc(&dx, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&dout, n * 8 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    math_check_kernel<<<blocks, 256>>>(dx, n, dout);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, n * 8 * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(dout);
  if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("fm_math_check: ") + cudaGetErrorString(e));
  return FM_OK;
}
