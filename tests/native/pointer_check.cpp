// Host build of the pointer-access rule and the per-context cache
// (era-bellman-cuda_b200/csrc/pointer_access.h) for tests/test_pointer_access.py:
// fabricated cudaPointerAttributes in, the decision out.  No CUDA call is made.
#include "pointer_access.h"

#include <cstdint>

using namespace msm_b200;

extern "C" {

// type: cudaMemoryType value; returns the cudaError_t; *view the kernel's address
int pc_kernel_view(int type, int device, int current, int peer_enabled, int allow_host, uintptr_t ptr, uintptr_t device_ptr, uintptr_t *view) {
  cudaPointerAttributes attr{};
  attr.type = static_cast<cudaMemoryType>(type);
  attr.device = device;
  attr.devicePointer = reinterpret_cast<void *>(device_ptr);
  attr.hostPointer = reinterpret_cast<void *>(ptr);
  void *out = nullptr;
  const cudaError_t err = kernel_view(reinterpret_cast<const void *>(ptr), attr, current, peer_enabled != 0,
                                      allow_host ? host_memory::device_alias : host_memory::refuse, &out);
  *view = reinterpret_cast<uintptr_t>(out);
  return static_cast<int>(err);
}

// One cache; lookups count how often the value had to be looked up.
static context_cache<uintptr_t> g_cache;
static unsigned g_lookups = 0;

// value for context `id`: looked up as id * 0x1000 + lookups so far (a fresh
// lookup is visible in the value); fail != 0 makes the lookup fail.
int pc_cache_get(unsigned long long id, int fail, uintptr_t *value) {
  return static_cast<int>(g_cache.get(id, value, [&](uintptr_t &v) {
    if (fail)
      return cudaErrorInvalidValue;
    v = static_cast<uintptr_t>(id * 0x1000 + g_lookups++);
    return cudaSuccess;
  }));
}
unsigned pc_cache_lookups() { return g_lookups; }
unsigned long long pc_cache_size() { return g_cache.size(); }
unsigned long long pc_cache_max() { return context_cache<uintptr_t>::MAX_ENTRIES; }
}
