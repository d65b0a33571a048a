// The caller-side final reduction of an MSM on the GPU: sum over i < 254 of
// 2^i R_i of the 254 per-bit Jacobian results, written as one canonical
// affine point (standard form, fully reduced, infinity flagged).  The
// reference leaves this Horner pass to its callers, on the host
// (src/bellman-cuda.h:496-505; tests/msm_test.cu:116-126).
//
// Whatever the order of the additions, the term 2^253 R_253 needs 253
// dependent doublings, so the sum is latency-bound.  A Horner pass also puts
// 253 additions on that chain; a pairwise tree over the bits puts 8: thread t
// starts from R_2t + 2 R_2t+1, and at level L = 1..7 the sum starting at bit
// 2t (t mod 2^L = 0) takes its partner's (t + 2^(L-1)), doubled 2^L times.
// From level 2 on (252 of the 255 doublings on the critical path) each
// doubling is shared by four lanes (dbl_group4).  Then one inversion by the
// binary extended Euclidean algorithm (far shorter than a Fermat inverse's
// 254 squarings).
#include "bellman-cuda-b200.h"
#include "msm_device.cuh"
#include "msm_group4.cuh"
#include "pointer_access.h"

#include <cuda_runtime.h>

namespace msm_b200 {

constexpr unsigned FINAL_THREADS = 128; // threads t < 127 start from results 2t, 2t + 1

__global__ void __launch_bounds__(FINAL_THREADS) final_sum_kernel(const jacobian *__restrict__ results, msm_b200_affine_point *point) {
  __shared__ xyzz part[FINAL_THREADS]; // part[t]: the sum of the bits starting at 2t (weights relative to 2^2t)
  const unsigned t = threadIdx.x;
  // level 0, one thread per pair of results
  xyzz q = curve::infinity();
  if (2 * t + 1 < RESULT_BITS) {
    const xyzz lo = curve::from_jacobian(results[2 * t]);
    const xyzz hi = curve::from_jacobian(results[2 * t + 1]);
    q = curve::add(lo, curve::dbl(hi));
  }
  part[t] = q;
  __syncthreads();
  // level 1, one thread per pair of level-0 sums (reads odd entries, writes even ones)
  if ((t & 1) == 0)
    part[t] = curve::add(part[t], curve::dbl(curve::dbl(part[t + 1])));
  __syncthreads();
  // levels 2..7: group g of four lanes adds part[g 2^L + 2^(L-1)], doubled
  // 2^L times, into part[g 2^L]; groups past the last pair (and whole warps
  // without an active group) double a copy of part[0] and write nothing
  for (unsigned level = 2; (1u << level) <= FINAL_THREADS; level++) {
    const unsigned pairs = FINAL_THREADS >> level, group = t >> 2;
    const unsigned target = group << level, partner = target + (1u << (level - 1));
    if (((t & ~31u) >> 2) < pairs) { // warp-uniform: the warp's first group is active
      const bool active = group < pairs;
      xyzz o = part[active ? partner : 0];
      // the double of infinity is infinity: a warp whose active partners are
      // all infinity skips the chain (the batched path's results are
      // infinity above bit c - 1, so most of its chains are skipped)
      if (!__all_sync(0xffffffffu, !active || curve::is_inf(o)))
        for (unsigned k = 0; k < (1u << level); k++)
          o = dbl_group4(o);
      if (active && (t & 3) == 0)
        part[target] = curve::add(part[target], o);
    }
    __syncthreads();
  }
  if (t == 0) {
    fe x, y;
    const bool infinity = curve::to_affine_standard(part[0], x, y);
    for (int i = 0; i < 8; i++) {
      point->x[i] = x.l[i];
      point->y[i] = y.l[i];
    }
    point->infinity = infinity ? 1u : 0u;
    for (int i = 0; i < 3; i++)
      point->reserved[i] = 0;
  }
}

// A pointer the kernel can dereference (pointer_access.h): device memory of
// the current device or of a peer it has access to, managed memory, or pinned
// host memory through its device alias; anything else is refused.
static cudaError_t device_view(const void *ptr, void **view) {
  int device = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess)
    return err;
  cudaPointerAttributes attr{};
  if ((err = cudaPointerGetAttributes(&attr, ptr)) != cudaSuccess)
    return err;
  const bool peer = attr.type == cudaMemoryTypeDevice && attr.device != device && peer_access_recorded(device, attr.device);
  return kernel_view(ptr, attr, device, peer, host_memory::device_alias, view);
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
