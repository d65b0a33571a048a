"""msm_b200_execute_no_alloc_async: the MSM entry point that allocates nothing.

Some callers cannot allocate device memory when they call the MSM: code in a
host callback or a driver layer where cudaMalloc is not allowed, or a prover
whose device memory is all handed out by its own allocator up front.  This
entry point runs the same pipeline with its scratch in a fixed 64 MiB block
that is part of the library image, so the caller passes only its inputs and
outputs.  Here it is called through the C ABI and checked against the
pool-allocating entry point (msm_b200_execute_async) on the same inputs,
bit-exact on the normalised affine point, for two calls in a row: the second
call is smaller than the first, so it runs over the block the first call left
behind.

This file sorts last so that a run stopping at the first failure has already
run every other test; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import bellman_cuda as bcm
    bc = bcm.BellmanCuda()
    bc.set_device(0)
    bc.msm_set_up()
    pool = bc.mem_pool_create(0)
    stream = bc.stream_create(True)
    yield bc, pool, stream
    bc.stream_destroy(stream)
    bc.mem_pool_destroy(pool)


def generated_bases(bc, stream, k):
    kd = bc.to_device(k)
    bd = bc.malloc(len(k) * 64)
    bc.generator_multiples(kd, bd, len(k), stream)
    bc.stream_synchronize(stream)
    bc.free(kd)
    return bd


def test_no_alloc_matches_pool_entry_point_twice(lib, oracle):
    import bellman_cuda as bcm
    bc, pool, stream = lib
    results_a = bc.malloc(254 * 96)
    results_b = bc.malloc(254 * 96)
    # first call at the maximum size (uniform scalars), second smaller (skewed)
    for n, dist, seed in ((bcm.NO_ALLOC_MAX_COUNT, "uniform", 301), (3001, "skewed", 302)):
        scalars, k = synth.workload(dist, n, seed)
        bd = generated_bases(bc, stream, k)
        sd = bc.to_device(scalars)
        assert bc.msm_no_alloc(stream, bd, sd, results_a, n) == bcm.BC_SUCCESS
        assert bc.msm_any(pool, stream, bd, sd, results_b, n) == bcm.BC_SUCCESS
        bc.stream_synchronize(stream)
        got = oracle.horner(bc.from_device(results_a, (254, 24)))
        want = oracle.horner(bc.from_device(results_b, (254, 24)))
        bc.free(bd)
        bc.free(sd)
        assert got == want
        assert got == oracle.msm_checksum(k, scalars)
    bc.free(results_a)
    bc.free(results_b)


def test_no_alloc_rejects_what_it_cannot_run(lib):
    """Checked on the host before anything is enqueued."""
    import bellman_cuda as bcm
    bc, _, stream = lib
    n = 1024
    bd, sd, rd = bc.malloc(n * 64), bc.malloc(n * 32), bc.malloc(254 * 96)
    host_results = np.zeros((254, 24), np.uint32)
    assert bc.msm_no_alloc(stream, bd, sd, rd, 0) == bcm.BC_ERROR_INVALID_VALUE
    assert bc.msm_no_alloc(stream, bd, sd, rd, bcm.NO_ALLOC_MAX_COUNT + 1) == bcm.BC_ERROR_INVALID_VALUE
    assert bc.msm_no_alloc(stream, bd, sd, host_results, n) == bcm.BC_ERROR_INVALID_VALUE
    assert bc.msm_no_alloc(stream, None, sd, rd, n) == bcm.BC_ERROR_INVALID_VALUE
    bc.stream_synchronize(stream)
    for p in (bd, sd, rd):
        bc.free(p)
