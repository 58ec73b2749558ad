// FP64 throughput ceiling of the device: the rate at which the SMs retire
// independent double-precision adds, multiplies and fused multiply-adds.
// The step kernels are built without multiply-add contraction (their
// rounding must equal the reference's), so their FP64 work is issued as
// DADD/DMUL (plus the FMAs inside division and square root); the add and
// multiply rates are the ceiling they are measured against, next to the
// HBM roofline.
//
// Each thread runs NCHAIN independent dependency chains (enough to cover the
// pipeline latency at full occupancy) for `iters` iterations; the grid fills
// every SM.  Operands are loaded from memory and the result is stored, so
// nothing folds at compile time.
#include <cuda_runtime.h>
#include <stdio.h>

#include "../../include/harm_b200.h"

namespace {

constexpr int NCHAIN = 8;

template <int OP>
__global__ void __launch_bounds__(256) k_fp64_rate(const double* __restrict__ in, double* __restrict__ out, int iters)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double x[NCHAIN];
  const double b = in[0], c = in[1];
#pragma unroll
  for (int k = 0; k < NCHAIN; k++) x[k] = in[2 + k] + (double)t;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < NCHAIN; k++) {
      if (OP == 0) x[k] = __dadd_rn(x[k], b);
      else if (OP == 1) x[k] = __dmul_rn(x[k], c);
      else x[k] = __fma_rn(x[k], c, b);
    }
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < NCHAIN; k++) s = __dadd_rn(s, x[k]);
  out[t] = s;
}

}  // namespace

extern "C" int harm_measure_fp64_peak(double* out3)
{
  if (!out3) return HARM_EINVAL;
  int dev = 0;
  cudaDeviceProp prop;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return HARM_ENODEVICE;
  if (prop.major != 10) return HARM_ENODEVICE;
  const int threads = 256, blocks = prop.multiProcessorCount * 8, iters = 4096;
  const long long nthreads = (long long)threads * blocks;
  double *d_in = nullptr, *d_out = nullptr;
  if (cudaMalloc(&d_in, 16 * sizeof(double)) != cudaSuccess) return HARM_ENOMEM;
  if (cudaMalloc(&d_out, nthreads * sizeof(double)) != cudaSuccess) {
    cudaFree(d_in);
    return HARM_ENOMEM;
  }
  // b and c keep the chains finite and away from subnormals over the run
  const double h_in[16] = {1.0e-9, 0.999999999, 1, 2, 3, 4, 5, 6, 7, 8, 0, 0, 0, 0, 0, 0};
  cudaMemcpy(d_in, h_in, sizeof(h_in), cudaMemcpyHostToDevice);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = HARM_OK;
  for (int op = 0; op < 3; op++) {
    float best = 1e30f;
    for (int rep = 0; rep < 4; rep++) {  // the first launch warms up; the best of the rest counts
      cudaEventRecord(e0);
      if (op == 0) k_fp64_rate<0><<<blocks, threads>>>(d_in, d_out, iters);
      else if (op == 1) k_fp64_rate<1><<<blocks, threads>>>(d_in, d_out, iters);
      else k_fp64_rate<2><<<blocks, threads>>>(d_in, d_out, iters);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0 && ms < best) best = ms;
    }
    // instructions per second (one FP64 operation per thread per chain step)
    out3[op] = (double)nthreads * iters * NCHAIN / (best * 1e-3);
  }
  if (cudaGetLastError() != cudaSuccess) rc = HARM_ECUDA;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_in);
  cudaFree(d_out);
  return rc;
}
