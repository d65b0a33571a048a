// bc_* runtime wrappers, ff_set_up / ff_tear_down, and the generator-multiple
// kernel of the extension ABI.
//
// The bc_* functions are thin casts over the CUDA runtime, exactly the
// reference's contract (src/bellman-cuda.cu:9-102, src/bc.cu:7-21): each
// returns the CUDA error code of the call it wraps.
#include "bellman-cuda-b200.h"
#include "bellman-cuda.h"
#include "bn254_curve.cuh"
#include "pointer_access.h"

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <utility>
#include <vector>

namespace {

inline bc_error to_bc(cudaError_t e) { return static_cast<bc_error>(e); }
inline cudaStream_t S(bc_stream s) { return static_cast<cudaStream_t>(s.handle); }
inline cudaEvent_t E(bc_event e) { return static_cast<cudaEvent_t>(e.handle); }
inline cudaMemPool_t P(bc_mem_pool p) { return static_cast<cudaMemPool_t>(p.handle); }

// (current device, peer) pairs with peer access enabled through
// bc_device_enable_peer_access and not disabled since.
std::mutex peer_lock;
std::vector<std::pair<int, int>> peer_pairs;

void record_peer_access(int peer, bool enabled) {
  int current = 0;
  if (cudaGetDevice(&current) != cudaSuccess)
    return;
  std::lock_guard<std::mutex> guard(peer_lock);
  const auto pair = std::make_pair(current, peer);
  const auto it = std::find(peer_pairs.begin(), peer_pairs.end(), pair);
  if (enabled && it == peer_pairs.end())
    peer_pairs.push_back(pair);
  if (!enabled && it != peer_pairs.end())
    peer_pairs.erase(it);
}

} // namespace

bool msm_b200::peer_access_recorded(int from, int peer) {
  std::lock_guard<std::mutex> guard(peer_lock);
  return std::find(peer_pairs.begin(), peer_pairs.end(), std::make_pair(from, peer)) != peer_pairs.end();
}

extern "C" {

bc_error bc_get_device_count(int *count) { return to_bc(cudaGetDeviceCount(count)); }
bc_error bc_get_device(int *device_id) { return to_bc(cudaGetDevice(device_id)); }
bc_error bc_set_device(int device_id) { return to_bc(cudaSetDevice(device_id)); }

bc_error bc_stream_create(bc_stream *stream, bool blocking_sync) {
  if (!stream)
    return bc_error_invalid_value;
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreate(&s);
  if (e != cudaSuccess)
    return to_bc(e);
  stream->handle = s;
  if (!blocking_sync)
    return bc_success;
  cudaStreamAttrValue policy{};
  policy.syncPolicy = cudaSyncPolicyBlockingSync;
  return to_bc(cudaStreamSetAttribute(s, cudaStreamAttributeSynchronizationPolicy, &policy));
}

bc_error bc_stream_wait_event(bc_stream stream, bc_event event) { return to_bc(cudaStreamWaitEvent(S(stream), E(event), 0)); }
bc_error bc_stream_synchronize(bc_stream stream) { return to_bc(cudaStreamSynchronize(S(stream))); }
bc_error bc_stream_query(bc_stream stream) { return to_bc(cudaStreamQuery(S(stream))); }
bc_error bc_stream_destroy(bc_stream stream) { return to_bc(cudaStreamDestroy(S(stream))); }
bc_error bc_launch_host_fn(bc_stream stream, bc_host_fn fn, void *user_data) { return to_bc(cudaLaunchHostFunc(S(stream), fn, user_data)); }

bc_error bc_event_create(bc_event *event, bool blocking_sync, bool disable_timing) {
  if (!event)
    return bc_error_invalid_value;
  const unsigned flags = (blocking_sync ? cudaEventBlockingSync : 0u) | (disable_timing ? cudaEventDisableTiming : 0u);
  cudaEvent_t ev = nullptr;
  cudaError_t e = cudaEventCreateWithFlags(&ev, flags);
  if (e == cudaSuccess)
    event->handle = ev;
  return to_bc(e);
}

bc_error bc_event_record(bc_event event, bc_stream stream) { return to_bc(cudaEventRecord(E(event), S(stream))); }
bc_error bc_event_synchronize(bc_event event) { return to_bc(cudaEventSynchronize(E(event))); }
bc_error bc_event_query(bc_event event) { return to_bc(cudaEventQuery(E(event))); }
bc_error bc_event_destroy(bc_event event) { return to_bc(cudaEventDestroy(E(event))); }
bc_error bc_event_elapsed_time(float *ms, bc_event start, bc_event end) { return to_bc(cudaEventElapsedTime(ms, E(start), E(end))); }

bc_error bc_mem_get_info(size_t *free, size_t *total) { return to_bc(cudaMemGetInfo(free, total)); }
bc_error bc_malloc(void **ptr, size_t size) { return to_bc(cudaMalloc(ptr, size)); }
bc_error bc_malloc_host(void **ptr, size_t size) { return to_bc(cudaMallocHost(ptr, size)); }
bc_error bc_free(void *ptr) { return to_bc(cudaFree(ptr)); }
bc_error bc_free_host(void *ptr) { return to_bc(cudaFreeHost(ptr)); }
bc_error bc_host_register(void *ptr, size_t size) { return to_bc(cudaHostRegister(ptr, size, cudaHostRegisterDefault)); }
bc_error bc_host_unregister(void *ptr) { return to_bc(cudaHostUnregister(ptr)); }
// The peer-access wrappers also keep the record that the kernels' pointer
// checks consult (pointer_access.h): memory of another device is accepted only
// while the current device has peer access to it.
bc_error bc_device_disable_peer_access(int device_id) {
  const cudaError_t e = cudaDeviceDisablePeerAccess(device_id);
  if (e == cudaSuccess || e == cudaErrorPeerAccessNotEnabled)
    record_peer_access(device_id, false);
  return to_bc(e);
}
bc_error bc_device_enable_peer_access(int device_id) {
  const cudaError_t e = cudaDeviceEnablePeerAccess(device_id, 0);
  if (e == cudaSuccess || e == cudaErrorPeerAccessAlreadyEnabled)
    record_peer_access(device_id, true);
  return to_bc(e);
}
bc_error bc_memcpy(void *dst, const void *src, size_t count) { return to_bc(cudaMemcpy(dst, src, count, cudaMemcpyDefault)); }
bc_error bc_memcpy_async(void *dst, const void *src, size_t count, bc_stream stream) {
  return to_bc(cudaMemcpyAsync(dst, src, count, cudaMemcpyDefault, S(stream)));
}
bc_error bc_memset(void *ptr, int value, size_t count) { return to_bc(cudaMemset(ptr, value, count)); }
bc_error bc_memset_async(void *ptr, int value, size_t count, bc_stream stream) { return to_bc(cudaMemsetAsync(ptr, value, count, S(stream))); }

bc_error bc_mem_pool_create(bc_mem_pool *pool, int device_id) {
  if (!pool)
    return bc_error_invalid_value;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device_id;
  cudaMemPool_t p = nullptr;
  cudaError_t e = cudaMemPoolCreate(&p, &props);
  if (e != cudaSuccess)
    return to_bc(e);
  pool->handle = p;
  uint64_t threshold = UINT64_MAX; // keep freed memory for reuse by later calls
  return to_bc(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &threshold));
}

bc_error bc_mem_pool_destroy(bc_mem_pool pool) { return to_bc(cudaMemPoolDestroy(P(pool))); }

bc_error bc_mem_pool_disable_peer_access(bc_mem_pool pool, int device_id) {
  cudaMemAccessDesc desc{};
  desc.location.type = cudaMemLocationTypeDevice;
  desc.location.id = device_id;
  desc.flags = cudaMemAccessFlagsProtNone;
  return to_bc(cudaMemPoolSetAccess(P(pool), &desc, 1));
}

bc_error bc_mem_pool_enable_peer_access(bc_mem_pool pool, int device_id) {
  cudaMemAccessDesc desc{};
  desc.location.type = cudaMemLocationTypeDevice;
  desc.location.id = device_id;
  desc.flags = cudaMemAccessFlagsProtReadWrite;
  return to_bc(cudaMemPoolSetAccess(P(pool), &desc, 1));
}

bc_error bc_malloc_from_pool_async(void **ptr, size_t size, bc_mem_pool pool, bc_stream stream) {
  return to_bc(cudaMallocFromPoolAsync(ptr, size, P(pool), S(stream)));
}

bc_error bc_free_async(void *ptr, bc_stream stream) { return to_bc(cudaFreeAsync(ptr, S(stream))); }

// The reference precomputes twiddle tables here (src/ff.cu:12-17); a coarse
// log count above the field's 2-adicity (28) cannot be served there either.
bc_error ff_set_up(unsigned powers_of_w_coarse_log_count, unsigned powers_of_g_coarse_log_count) {
  if (powers_of_w_coarse_log_count > 28 || powers_of_g_coarse_log_count > 28)
    return bc_error_invalid_value;
  return to_bc(cudaFree(nullptr)); // establishes the context, as the reference's allocations do
}

bc_error ff_tear_down() { return bc_success; }

} // extern "C"

// ---------------------------------------------------------------------------
// Generator multiples k * G (extension; synthetic base tables).
// Fixed-base comb with 4-bit digits: table[j][v-1] = v * 16^j * G (affine,
// Montgomery form) for j < 64, v < 16, built once per device; k * G is then
// at most 64 mixed additions, followed by one Fermat inversion to go affine.
// ---------------------------------------------------------------------------
namespace {

using namespace bn254;

constexpr unsigned COMB_DIGITS = 64, COMB_VALUES = 15;
__device__ affine g_comb_table[COMB_DIGITS * COMB_VALUES];


__global__ void comb_table_kernel() {
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= COMB_DIGITS * COMB_VALUES)
    return;
  const unsigned j = t / COMB_VALUES, v = t % COMB_VALUES + 1;
  fe one_std = fq::zero(), two_std = fq::zero();
  one_std.l[0] = 1;
  two_std.l[0] = 2;
  affine g;
  g.x = fq::to_mont(one_std);
  g.y = fq::to_mont(two_std);
  xyzz base = curve::from_affine(g);
  for (unsigned k = 0; k < 4 * j; k++)
    base = curve::dbl(base);
  xyzz acc = base;
  for (unsigned k = 1; k < v; k++)
    acc = curve::add(acc, base);
  g_comb_table[t] = curve::to_affine(acc);
}

__global__ void generator_multiples_kernel(const fe *__restrict__ k, affine *__restrict__ out, unsigned count) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count)
    return;
  const fe s = k[i];
  xyzz acc = curve::infinity();
  for (unsigned j = 0; j < COMB_DIGITS; j++) {
    const unsigned v = (s.l[j >> 3] >> ((j & 7) * 4)) & 15;
    if (v)
      acc = curve::add_affine(acc, g_comb_table[j * COMB_VALUES + v - 1]);
  }
  if (curve::is_inf(acc)) {
    out[i].x = fq::zero();
    out[i].y = fq::zero();
    return;
  }
  out[i] = curve::to_affine(acc);
}

std::mutex comb_lock;
bool comb_ready[64];

cudaError_t ensure_comb_table(cudaStream_t stream) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess)
    return e;
  if (device < 0 || device >= 64)
    return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> guard(comb_lock);
  if (comb_ready[device])
    return cudaSuccess;
  comb_table_kernel<<<(COMB_DIGITS * COMB_VALUES + 63) / 64, 64, 0, stream>>>();
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return e;
  e = cudaStreamSynchronize(stream);
  if (e == cudaSuccess)
    comb_ready[device] = true;
  return e;
}

} // namespace

extern "C" bc_error msm_b200_generator_multiples_async(const void *k, void *bases, unsigned count, bc_stream stream) {
  if (!k || !bases)
    return bc_error_invalid_value;
  if (count == 0)
    return bc_success;
  cudaStream_t s = static_cast<cudaStream_t>(stream.handle);
  cudaError_t e = ensure_comb_table(s);
  if (e != cudaSuccess)
    return static_cast<bc_error>(e);
  generator_multiples_kernel<<<(count + 127) / 128, 128, 0, s>>>(static_cast<const fe *>(k), static_cast<affine *>(bases), count);
  return static_cast<bc_error>(cudaGetLastError());
}
