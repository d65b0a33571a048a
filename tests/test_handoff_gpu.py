"""The producer -> MSM hand-off on one stream (reference tests/bc_test.cu:69-124,
`ntt_into_msm` / `ntt_into_four_msms_in_series`): a kernel earlier on the
caller's stream writes the Montgomery-form scalars into pool memory allocated
on that stream, and msm_execute_async calls follow on the same stream with no
host synchronisation in between; the buffer is released with bc_free_async
after them.  The producer here is a device gather (torch, on the caller's
stream through torch.cuda.ExternalStream), delayed by a spin of the GPU clock
so that an MSM that did not wait for it would read the buffer before it is
written.  Every result is checked against the oracle's checksum of the
produced scalars."""
import ctypes

import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu


class _DeviceArray:
    """A raw device buffer seen by torch without a copy (__cuda_array_interface__)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (ptr, False), "version": 3,
                                         "strides": None, "stream": None}


def test_producer_then_four_msms_in_series(oracle):
    torch = pytest.importorskip("torch")
    import bellman_cuda as bcm
    bc = bcm.BellmanCuda()
    bc.set_device(0)
    bc.msm_set_up()
    pool = bc.mem_pool_create(0)
    stream = bc.stream_create(True)
    log_n, msms = 12, 4
    n = 1 << log_n
    total = msms * n
    # inputs of the producer: a permutation of the scalars the MSMs must see
    scalars, k = synth.workload("uniform", total, 401)
    perm = np.random.Generator(np.random.PCG64(402)).permutation(total)
    staged = np.empty_like(scalars)
    staged[perm] = scalars  # the producer computes values[i] = staged[perm[i]] = scalars[i]
    kd = bc.to_device(k)
    bd = bc.malloc(total * 64)
    bc.generator_multiples(kd, bd, total, stream)
    bc.stream_synchronize(stream)
    bc.free(kd)
    staged_t = torch.from_numpy(staged.view(np.int64)).cuda()
    perm_t = torch.from_numpy(perm.astype(np.int64)).cuda()
    torch.cuda.synchronize()
    results = [np.zeros((254, 24), np.uint32) for _ in range(msms)]
    # --- everything below is enqueued on one stream, no host synchronisation ---
    values = ctypes.c_void_p()
    bc.check(bc.lib.bc_malloc_from_pool_async(ctypes.byref(values), total * 32, pool, stream), "bc_malloc_from_pool_async")
    values_t = torch.as_tensor(_DeviceArray(values.value, (total, 4), "<i8"), device="cuda")
    producer = torch.cuda.ExternalStream(stream.handle)
    with torch.cuda.stream(producer):
        torch.cuda._sleep(20_000_000)  # ~10 ms of GPU clock before the producer writes
        torch.index_select(staged_t, 0, perm_t, out=values_t)
    for i in range(msms):
        bc.msm(pool, stream, bd + i * n * 64, values.value + i * n * 32, results[i], log_n)
    bc.check(bc.lib.bc_free_async(values, stream), "bc_free_async")
    bc.stream_synchronize(stream)
    # ---------------------------------------------------------------------------
    for i in range(msms):
        sl = slice(i * n, (i + 1) * n)
        assert oracle.horner(results[i]) == oracle.msm_checksum(np.ascontiguousarray(k[sl]), np.ascontiguousarray(scalars[sl])), i
    bc.free(bd)
    bc.stream_destroy(stream)
    bc.mem_pool_destroy(pool)
