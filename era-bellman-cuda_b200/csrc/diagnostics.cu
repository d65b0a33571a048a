// Integer-multiply throughput probes: the roofline denominator of the bucket
// accumulation and reduction kernels (32-bit multiply instructions per
// second), measured on the device the library runs on.
#include "bellman-cuda-b200.h"
#include "bn254_curve.cuh"

#include <cuda_runtime.h>

namespace {

using namespace bn254;

// kind 0: sixteen independent mad.lo / mad.hi per iteration (no carries)
__global__ void __launch_bounds__(256) mad_peak_kernel(uint32_t seed, unsigned iters, uint32_t *sink) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t lo[8], hi[8];
  const uint32_t b = seed ^ (tid * 0x9e3779b9u), c = seed + tid;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    lo[j] = tid * (j + 3);
    hi[j] = tid ^ (j * 0x85ebca6bu);
  }
  for (unsigned i = 0; i < iters; i++) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
      asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(lo[j]) : "r"(b), "r"(c));
      asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(hi[j]) : "r"(b), "r"(c));
    }
  }
  uint32_t x = 0;
#pragma unroll
  for (int j = 0; j < 8; j++)
    x ^= lo[j] ^ hi[j];
  sink[tid] = x;
}

// kind 4: sixteen independent mad.lo per iteration
__global__ void __launch_bounds__(256) mad_lo_kernel(uint32_t seed, unsigned iters, uint32_t *sink) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t acc[16];
  const uint32_t b = seed ^ (tid * 0x9e3779b9u), c = seed + tid;
#pragma unroll
  for (int j = 0; j < 16; j++)
    acc[j] = tid * (j + 3);
  for (unsigned i = 0; i < iters; i++) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
      asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(acc[j]) : "r"(b), "r"(c));
    }
  }
  uint32_t x = 0;
#pragma unroll
  for (int j = 0; j < 16; j++)
    x ^= acc[j];
  sink[tid] = x;
}

// kind 1: one 16-instruction carry chain per iteration (madc.lo.cc / madc.hi.cc)
__global__ void __launch_bounds__(256) mad_chain_kernel(uint32_t seed, unsigned iters, uint32_t *sink) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t a[8], t[8];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    a[j] = seed * (j + 1) + tid;
    t[j] = tid ^ j;
  }
  const uint32_t b = seed ^ tid;
  for (unsigned i = 0; i < iters; i++) {
    t[0] = cc::mad_lo_cc(a[0], b, t[0]);
    t[1] = cc::madc_hi_cc(a[0], b, t[1]);
    t[2] = cc::madc_lo_cc(a[1], b, t[2]);
    t[3] = cc::madc_hi_cc(a[1], b, t[3]);
    t[4] = cc::madc_lo_cc(a[2], b, t[4]);
    t[5] = cc::madc_hi_cc(a[2], b, t[5]);
    t[6] = cc::madc_lo_cc(a[3], b, t[6]);
    t[7] = cc::madc_hi_cc(a[3], b, t[7]);
    t[0] = cc::madc_lo_cc(a[4], b, t[0]);
    t[1] = cc::madc_hi_cc(a[4], b, t[1]);
    t[2] = cc::madc_lo_cc(a[5], b, t[2]);
    t[3] = cc::madc_hi_cc(a[5], b, t[3]);
    t[4] = cc::madc_lo_cc(a[6], b, t[4]);
    t[5] = cc::madc_hi_cc(a[6], b, t[5]);
    t[6] = cc::madc_lo_cc(a[7], b, t[6]);
    t[7] = cc::madc_hi(a[7], b, t[7]);
  }
  uint32_t x = 0;
#pragma unroll
  for (int j = 0; j < 8; j++)
    x ^= t[j];
  sink[tid] = x;
}

// kind 2: two independent Montgomery products per iteration
__global__ void __launch_bounds__(128) montmul_kernel(uint32_t seed, unsigned iters, uint32_t *sink) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  fe x, y, z;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    x.l[j] = (seed * (j + 7)) ^ tid;
    y.l[j] = (seed + j) * 0x2545f491u;
    z.l[j] = tid * (j + 1);
  }
  x.l[7] &= 0x1fffffff;
  y.l[7] &= 0x1fffffff;
  z.l[7] &= 0x1fffffff;
  for (unsigned i = 0; i < iters; i++) {
    x = fq::mul(x, y);
    z = fq::mul(z, y);
  }
  sink[tid] = x.l[0] ^ z.l[1];
}

// kind 3: XYZZ += affine chain with add_affine_finite, the addition of the
// accumulation loop (never the doubling or cancelling branch: acc = k*G,
// k >= 2), at the accumulation kernel's 4 blocks of 128 threads per SM
__global__ void __launch_bounds__(128, 4) madd_kernel(unsigned iters, uint32_t *sink) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  fe one_std = fq::zero(), two_std = fq::zero();
  one_std.l[0] = 1;
  two_std.l[0] = 2;
  affine g;
  g.x = fq::to_mont(one_std);
  g.y = fq::to_mont(two_std);
  if (tid & 1)
    g.y = fq::neg(g.y);
  xyzz acc = curve::dbl_affine(g);
  bool inf = false;
  for (unsigned i = 0; i < iters; i++)
    acc = curve::add_affine_finite(acc, g, inf);
  sink[tid] = acc.x.l[0] ^ acc.zz.l[3] ^ (inf ? 1u : 0u);
}

} // namespace

extern "C" bc_error msm_b200_measure_mul_throughput(unsigned kind, double *mulops_per_second) {
  if (!mulops_per_second || kind > 4)
    return bc_error_invalid_value;
  int device = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess)
    return static_cast<bc_error>(e);
  const bool light = kind < 2 || kind == 4;
  const unsigned threads = light ? 256 : 128;
  const unsigned blocks = light ? sms * 8 : sms * 4;
  const unsigned iters = light ? 65536 : kind == 2 ? 4096 : 1024;
  const double per_iter = light ? 16.0 : kind == 2 ? 2.0 * 264 : 2392.0;
  uint32_t *sink = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t start = nullptr, stop = nullptr;
  float ms = 0;
  do {
    if ((e = cudaMalloc(&sink, (size_t)threads * blocks * 4)) != cudaSuccess)
      break;
    if ((e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)) != cudaSuccess)
      break;
    if ((e = cudaEventCreate(&start)) != cudaSuccess || (e = cudaEventCreate(&stop)) != cudaSuccess)
      break;
    for (int rep = 0; rep < 2 && e == cudaSuccess; rep++) {
      if ((e = cudaEventRecord(start, stream)) != cudaSuccess)
        break;
      switch (kind) {
      case 0: mad_peak_kernel<<<blocks, threads, 0, stream>>>(0x1234567u, iters, sink); break;
      case 1: mad_chain_kernel<<<blocks, threads, 0, stream>>>(0x1234567u, iters, sink); break;
      case 2: montmul_kernel<<<blocks, threads, 0, stream>>>(0x1234567u, iters, sink); break;
      case 4: mad_lo_kernel<<<blocks, threads, 0, stream>>>(0x1234567u, iters, sink); break;
      default: madd_kernel<<<blocks, threads, 0, stream>>>(iters, sink); break;
      }
      if ((e = cudaGetLastError()) != cudaSuccess)
        break;
      if ((e = cudaEventRecord(stop, stream)) != cudaSuccess)
        break;
      if ((e = cudaEventSynchronize(stop)) != cudaSuccess)
        break;
      e = cudaEventElapsedTime(&ms, start, stop);
    }
  } while (false);
  if (start)
    cudaEventDestroy(start);
  if (stop)
    cudaEventDestroy(stop);
  if (stream)
    cudaStreamDestroy(stream);
  if (sink)
    cudaFree(sink);
  if (e != cudaSuccess)
    return static_cast<bc_error>(e);
  *mulops_per_second = (double)threads * blocks * iters * per_iter / (ms * 1e-3);
  return bc_success;
}
