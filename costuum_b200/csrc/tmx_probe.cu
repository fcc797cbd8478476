// FP64 throughput probes used as roofline denominators: the DFMA pipe
// (fma.rn.f64) and the FP64 tensor pipe (mma.sync m8n8k4 f64, DMMA).
// Each thread keeps independent accumulator chains so the pipe, not latency,
// bounds the loop. The result is stored so the work cannot be elided.
#include "tmx_common.cuh"
#include "tmx_kernels.h"

#define PROBE_CHAINS 8

__global__ void k_probe_dfma(double *out, int iters) {
  double a[PROBE_CHAINS];
  const double x = 1.0 + 1e-9 * threadIdx.x;
  const double y = 0.999999999;
#pragma unroll
  for (int c = 0; c < PROBE_CHAINS; ++c) {
    a[c] = 1e-3 * (c + 1);
  }
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < PROBE_CHAINS; ++c) {
      a[c] = fma(a[c], y, x);
    }
  }
  double s = 0.;
#pragma unroll
  for (int c = 0; c < PROBE_CHAINS; ++c) {
    s += a[c];
  }
  if (s == 12345.678) {
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
  }
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    out[0] = s;
  }
}

__global__ void k_probe_dmma(double *out, int iters) {
  double acc[PROBE_CHAINS][2];
  const double a = 1.0 + 1e-9 * threadIdx.x;
  const double b = 0.999999999;
#pragma unroll
  for (int c = 0; c < PROBE_CHAINS; ++c) {
    acc[c][0] = acc[c][1] = 1e-3 * (c + 1);
  }
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < PROBE_CHAINS; ++c) {
      asm volatile(
          "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, "
          "{%3}, {%0, %1};\n"
          : "+d"(acc[c][0]), "+d"(acc[c][1])
          : "d"(a), "d"(b));
    }
  }
  double s = 0.;
#pragma unroll
  for (int c = 0; c < PROBE_CHAINS; ++c) {
    s += acc[c][0] + acc[c][1];
  }
  if (s == 12345.678) {
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
  }
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    out[0] = s;
  }
}

void tmx_launch_probe_dfma(double *out, int iters, int blocks,
                           cudaStream_t stream) {
  k_probe_dfma<<<blocks, 256, 0, stream>>>(out, iters);
}

void tmx_launch_probe_dmma(double *out, int iters, int blocks,
                           cudaStream_t stream) {
  k_probe_dmma<<<blocks, 256, 0, stream>>>(out, iters);
}
