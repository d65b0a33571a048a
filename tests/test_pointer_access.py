"""The host-side pointer rule shared by the MSM entry points and the final sum,
and the per-context cache of the no-allocation scratch address
(era-bellman-cuda_b200/csrc/pointer_access.h), built for the host and driven
with fabricated pointer attributes: no GPU, no CUDA call."""
import ctypes
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "era-bellman-cuda_b200", "csrc")
CUDA_INCLUDE = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")

UNREGISTERED, HOST, DEVICE, MANAGED = 0, 1, 2, 3  # cudaMemoryType
SUCCESS, INVALID_VALUE = 0, 1


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(os.path.join(CUDA_INCLUDE, "cuda_runtime_api.h")):
        pytest.skip("CUDA headers absent")
    out = os.path.join(HERE, "native", "_build")
    os.makedirs(out, exist_ok=True)
    so = os.path.join(out, "libpointer_check.so")
    src = os.path.join(HERE, "native", "pointer_check.cpp")
    hdr = os.path.join(CSRC, "pointer_access.h")
    if not os.path.exists(so) or max(os.path.getmtime(src), os.path.getmtime(hdr)) > os.path.getmtime(so):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I" + CSRC, "-I" + CUDA_INCLUDE, "-o", so, src], check=True)
    lib = ctypes.CDLL(so)
    lib.pc_kernel_view.argtypes = [ctypes.c_int] * 5 + [ctypes.c_size_t, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    lib.pc_cache_get.argtypes = [ctypes.c_ulonglong, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]
    lib.pc_cache_size.restype = ctypes.c_ulonglong
    lib.pc_cache_max.restype = ctypes.c_ulonglong
    return lib


def view(lib, mem_type, device, current=0, peer=False, allow_host=False, ptr=0x7000, device_ptr=0x9000):
    out = ctypes.c_size_t(0)
    rc = lib.pc_kernel_view(mem_type, device, current, int(peer), int(allow_host), ptr, device_ptr, ctypes.byref(out))
    return rc, out.value


def test_device_memory_of_the_current_device(lib):
    assert view(lib, DEVICE, 0) == (SUCCESS, 0x7000)
    assert view(lib, DEVICE, 3, current=3) == (SUCCESS, 0x7000)


def test_device_memory_of_another_device_needs_peer_access(lib):
    """Another GPU's memory without peer access would fault in the kernel:
    refused before anything is enqueued; with peer access it is used as is."""
    assert view(lib, DEVICE, 1, current=0)[0] == INVALID_VALUE
    assert view(lib, DEVICE, 1, current=0, peer=True) == (SUCCESS, 0x7000)


def test_host_memory(lib):
    assert view(lib, HOST, 0)[0] == INVALID_VALUE  # device-memory-only entry points
    assert view(lib, HOST, 0, allow_host=True) == (SUCCESS, 0x9000)  # pinned: its device alias
    assert view(lib, HOST, 0, allow_host=True, device_ptr=0)[0] == INVALID_VALUE
    assert view(lib, UNREGISTERED, 0, allow_host=True)[0] == INVALID_VALUE  # pageable


def test_managed_memory(lib):
    assert view(lib, MANAGED, 1, current=0) == (SUCCESS, 0x7000)


def test_context_cache_is_keyed_by_context_id(lib):
    """One lookup per context id; a new id (a context destroyed and created
    again, e.g. after cudaDeviceReset) gets its own lookup, never the old
    context's value; a failed lookup is not cached."""
    v = ctypes.c_size_t()
    assert lib.pc_cache_get(11, 0, ctypes.byref(v)) == SUCCESS
    first = v.value
    assert lib.pc_cache_get(11, 0, ctypes.byref(v)) == SUCCESS and v.value == first
    assert lib.pc_cache_lookups() == 1
    assert lib.pc_cache_get(12, 0, ctypes.byref(v)) == SUCCESS and v.value != first and v.value >> 12 == 12
    assert lib.pc_cache_lookups() == 2
    assert lib.pc_cache_get(13, 1, ctypes.byref(v)) == INVALID_VALUE
    assert lib.pc_cache_get(13, 0, ctypes.byref(v)) == SUCCESS and v.value >> 12 == 13
    assert lib.pc_cache_lookups() == 3
    # bounded: the oldest contexts are dropped
    for cid in range(100, 100 + 2 * lib.pc_cache_max()):
        assert lib.pc_cache_get(cid, 0, ctypes.byref(v)) == SUCCESS
    assert lib.pc_cache_size() == lib.pc_cache_max()
    before = lib.pc_cache_lookups()
    assert lib.pc_cache_get(11, 0, ctypes.byref(v)) == SUCCESS and v.value != first
    assert lib.pc_cache_lookups() == before + 1
