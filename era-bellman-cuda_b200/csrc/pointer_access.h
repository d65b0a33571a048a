// Host-side rules for the memory this library's kernels dereference, and the
// per-context cache of values that belong to one CUDA context.  Header-only and
// free of CUDA calls, so that the CPU tests compile it against the CUDA headers
// alone (tests/native/pointer_check.cpp) and feed it fabricated attributes.
#pragma once

#include <cuda_runtime_api.h>

#include <cstddef>
#include <mutex>
#include <utility>
#include <vector>

namespace msm_b200 {

// What a kernel may do with pinned host memory: refuse it (the entry point
// takes device memory only) or use its device alias in place.
enum class host_memory { refuse, device_alias };

// Whether memory described by `attr` (from cudaPointerGetAttributes on `ptr`)
// can be handed to a kernel running on `current_device`, and the address the
// kernel then uses (*view):
//   * device memory of the current device: as is;
//   * device memory of another device: only when the current device has peer
//     access to it (`peer_enabled`); without it the kernel's first access would
//     fault, so the call is refused before anything is enqueued;
//   * managed memory: as is;
//   * pinned host memory: its device alias when `host` allows it;
//   * pageable (unregistered) memory: refused.
// Refusals return cudaErrorInvalidValue.
inline cudaError_t kernel_view(const void *ptr, const cudaPointerAttributes &attr, int current_device, bool peer_enabled, host_memory host,
                               void **view) {
  switch (attr.type) {
  case cudaMemoryTypeDevice:
    if (attr.device != current_device && !peer_enabled)
      return cudaErrorInvalidValue;
    *view = const_cast<void *>(ptr);
    return cudaSuccess;
  case cudaMemoryTypeManaged:
    *view = const_cast<void *>(ptr);
    return cudaSuccess;
  case cudaMemoryTypeHost:
    if (host != host_memory::device_alias || !attr.devicePointer)
      return cudaErrorInvalidValue;
    *view = attr.devicePointer;
    return cudaSuccess;
  default:
    return cudaErrorInvalidValue;
  }
}

// Peer access the library has seen enabled through bc_device_enable_peer_access
// (and not disabled since): from the device that was current to `peer`.
// Defined in bc_runtime.cu.
bool peer_access_recorded(int from, int peer);

// Values looked up once per CUDA context, keyed by the context's unique id
// (cuCtxGetId: ids are never reused within a process).  A context that is
// destroyed and created again -- cudaDeviceReset, or a caller's own
// driver-API context on the same device -- has a new id and therefore gets a
// fresh lookup instead of a value that belonged to the old context.  The
// cache keeps the most recent MAX_ENTRIES contexts.
template <class V> class context_cache {
public:
  static constexpr std::size_t MAX_ENTRIES = 64;

  // *out = the value for context `id`, calling lookup(V &) the first time.
  template <class F> cudaError_t get(unsigned long long id, V *out, F lookup) {
    std::lock_guard<std::mutex> guard(lock_);
    for (const auto &e : entries_)
      if (e.first == id) {
        *out = e.second;
        return cudaSuccess;
      }
    V value{};
    const cudaError_t err = lookup(value);
    if (err != cudaSuccess)
      return err;
    if (entries_.size() == MAX_ENTRIES)
      entries_.erase(entries_.begin());
    entries_.emplace_back(id, value);
    *out = value;
    return cudaSuccess;
  }

  std::size_t size() {
    std::lock_guard<std::mutex> guard(lock_);
    return entries_.size();
  }

private:
  std::mutex lock_;
  std::vector<std::pair<unsigned long long, V>> entries_;
};

} // namespace msm_b200
