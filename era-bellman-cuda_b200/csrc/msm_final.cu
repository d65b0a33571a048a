// The caller-side final reduction of an MSM on the GPU: sum over i < 254 of
// 2^i R_i of the 254 per-bit Jacobian results, written as one canonical
// affine point (standard form, fully reduced, infinity flagged).  The
// reference leaves this Horner pass to its callers, on the host
// (src/bellman-cuda.h:496-505; tests/msm_test.cu:116-126).
//
// Whatever the order of the additions, the term 2^253 R_253 needs 253
// dependent doublings, so the sum is latency-bound on one thread.  A Horner
// pass also puts 253 additions on that chain; a pairwise tree over the bits
// puts 8: thread t starts from R_2t + 2 R_2t+1, and at level L = 1..7 the
// threads with t mod 2^L = 0 add their partner t + 2^(L-1), doubled 2^L
// times (its lowest bit is 2^L above theirs).  Critical path: 255 doublings
// and 8 additions, then one inversion by the binary extended Euclidean
// algorithm (far shorter than a Fermat inverse's 254 squarings).
#include "bellman-cuda-b200.h"
#include "msm_device.cuh"

#include <cuda_runtime.h>

namespace msm_b200 {

constexpr unsigned FINAL_THREADS = 128; // threads t < 127 start from results 2t, 2t + 1

__global__ void __launch_bounds__(FINAL_THREADS) final_sum_kernel(const jacobian *__restrict__ results, msm_b200_affine_point *point) {
  __shared__ xyzz partner[FINAL_THREADS];
  const unsigned t = threadIdx.x;
  xyzz q = curve::infinity();
  if (2 * t + 1 < RESULT_BITS) {
    const xyzz lo = curve::from_jacobian(results[2 * t]);
    const xyzz hi = curve::from_jacobian(results[2 * t + 1]);
    q = curve::add(lo, curve::dbl(hi));
  }
  for (unsigned level = 1; (1u << level) <= FINAL_THREADS; level++) {
    const unsigned half = 1u << (level - 1), mask = 2 * half - 1;
    if ((t & mask) == half)
      partner[t] = q;
    __syncthreads();
    if ((t & mask) == 0) {
      xyzz o = partner[t + half]; // t + half <= FINAL_THREADS - half
      for (unsigned k = 0; k < (1u << level); k++)
        o = curve::dbl(o);
      q = curve::add(q, o);
    }
    __syncthreads();
  }
  if (t == 0) {
    fe x, y;
    const bool infinity = curve::to_affine_standard(q, x, y);
    for (int i = 0; i < 8; i++) {
      point->x[i] = x.l[i];
      point->y[i] = y.l[i];
    }
    point->infinity = infinity ? 1u : 0u;
    for (int i = 0; i < 3; i++)
      point->reserved[i] = 0;
  }
}

// A pointer the kernel can dereference: device or managed memory as is,
// pinned host memory through its device alias; pageable memory is refused.
static cudaError_t device_view(const void *ptr, void **view) {
  cudaPointerAttributes attr{};
  const cudaError_t err = cudaPointerGetAttributes(&attr, ptr);
  if (err != cudaSuccess)
    return err;
  switch (attr.type) {
  case cudaMemoryTypeDevice:
  case cudaMemoryTypeManaged:
    *view = const_cast<void *>(ptr);
    return cudaSuccess;
  case cudaMemoryTypeHost:
    if (!attr.devicePointer)
      return cudaErrorInvalidValue;
    *view = attr.devicePointer;
    return cudaSuccess;
  default:
    return cudaErrorInvalidValue;
  }
}

cudaError_t final_sum(const void *results, msm_b200_affine_point *point, cudaStream_t stream) {
  if (!results || !point || reinterpret_cast<uintptr_t>(results) % 16 || reinterpret_cast<uintptr_t>(point) % 4)
    return cudaErrorInvalidValue;
  void *r = nullptr, *p = nullptr;
  cudaError_t err = device_view(results, &r);
  if (err == cudaSuccess)
    err = device_view(point, &p);
  if (err != cudaSuccess)
    return err;
  final_sum_kernel<<<1, FINAL_THREADS, 0, stream>>>(static_cast<const jacobian *>(r), static_cast<msm_b200_affine_point *>(p));
  return cudaGetLastError();
}

} // namespace msm_b200

extern "C" bc_error msm_b200_final_sum_async(const void *results, msm_b200_affine_point *point, bc_stream stream) {
  return static_cast<bc_error>(msm_b200::final_sum(results, point, static_cast<cudaStream_t>(stream.handle)));
}
