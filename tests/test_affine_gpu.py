"""GPU parity of the affine pairing levels (csrc/msm_affine.cuh) against the
oracle, with the level count forced through msm_b200_set_affine_levels at
sizes where the default runs none: repeated bases (doublings inside a level),
a point and its negation in one bucket (infinity markers carried through later
levels and skipped by the XYZZ pass), every window width, skewed scalars, and
the work counts of the profile."""
import numpy as np
import pytest

import msm_helpers as H
import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bc():
    import bellman_cuda as bcm
    b = bcm.BellmanCuda()
    b.set_device(0)
    b.msm_set_up()
    b.pool_handle = b.mem_pool_create(0)
    b.stream_handle = b.stream_create(True)
    yield b
    b.set_affine_levels(-1)


def run(bc, bases, scalars, window_bits=0, bases_dev=None, profile=False):
    n = len(scalars)
    bd = bases_dev if bases_dev is not None else bc.to_device(np.ascontiguousarray(bases))
    sd = bc.to_device(np.ascontiguousarray(scalars))
    rd = bc.malloc(254 * 96)
    prof = None
    if profile:
        prof = bc.msm_profiled(bc.pool_handle, bc.stream_handle, bd, sd, rd, n, window_bits)
    else:
        assert bc.msm_any(bc.pool_handle, bc.stream_handle, bd, sd, rd, n, window_bits) == 0
        bc.stream_synchronize(bc.stream_handle)
    res = bc.from_device(rd, (254, 24))
    for p in ([sd, rd] if bases_dev is not None else [bd, sd, rd]):
        bc.free(p)
    return (res, prof) if profile else res


@pytest.mark.parametrize("levels", [1, 2, 3, 4])
@pytest.mark.parametrize("log_n", [0, 1, 2, 3, 5, 8, 10, 12, 14])
def test_levels_table_bases(bc, oracle, levels, log_n):
    """Bases from the 256-point table (repeats: doublings and equal x), the
    default width of each size."""
    bc.set_affine_levels(levels)
    try:
        bases, scalars, k = H.table_workload(1 << log_n, 900 + log_n)
        assert oracle.horner(run(bc, bases, scalars)) == oracle.msm_checksum(k, scalars)
    finally:
        bc.set_affine_levels(-1)


@pytest.mark.parametrize("levels", [1, 3])
def test_levels_cancellation_and_doublings(bc, oracle, levels):
    """One base with scalars s and r - s (each bucket holds P and -P: the
    level's sums are infinity markers) and with equal scalars (every pair a
    doubling), each also with a few other points mixed in."""
    table = H.load_g_bases()
    bc.set_affine_levels(levels)
    try:
        for vals in ([7] * 128 + [H.R - 7] * 128, [5] * 256, [3, H.R - 3] * 128, [11] * 200 + list(range(1, 57))):
            n = len(vals)
            idx = [3] * n
            if len(set(vals)) > 2:
                idx = [3] * 200 + [i % 256 for i in range(56)]
            bases = H.mont_point_array([table[i] for i in idx])
            k = np.zeros((n, 8), np.uint32)
            k[:, 0] = np.array(idx) + 1
            scalars = H.mont_scalar_array(vals)
            assert oracle.horner(run(bc, bases, scalars)) == oracle.msm_checksum(k, scalars)
    finally:
        bc.set_affine_levels(-1)


@pytest.mark.parametrize("window_bits", [2, 4, 7, 11, 13, 16, 17, 20])
def test_levels_any_window(bc, oracle, window_bits):
    bc.set_affine_levels(3)
    try:
        bases, scalars, k = H.table_workload(3001, 77)
        assert oracle.horner(run(bc, bases, scalars, window_bits)) == oracle.msm_checksum(k, scalars)
    finally:
        bc.set_affine_levels(-1)


@pytest.mark.parametrize("dist", ["uniform", "skewed"])
@pytest.mark.parametrize("levels", [0, 1, 2, 4])
def test_levels_generated_bases(bc, oracle, dist, levels):
    """2^17 + 5 points over k_i G, the work counts of the profile: the levels
    remove elements (affine additions), and what the XYZZ pass adds is the
    rest."""
    n = (1 << 17) + 5
    scalars, k = synth.workload(dist, n, 950 + levels)
    kd = bc.to_device(k)
    bd = bc.malloc(n * 64)
    bc.generator_multiples(kd, bd, n, bc.stream_handle)
    bc.stream_synchronize(bc.stream_handle)
    bc.free(kd)
    bc.set_affine_levels(levels)
    try:
        res, prof = run(bc, None, scalars, bases_dev=bd, profile=True)
    finally:
        bc.set_affine_levels(-1)
        bc.free(bd)
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)
    assert prof.affine_levels == levels
    assert prof.sort_wait_timeouts == 0
    if levels == 0:
        assert prof.affine_additions == 0
    else:
        assert 0 < prof.affine_additions < prof.nonzero_entries
        if dist == "uniform":
            # about 8 entries per bucket: a level halves every bucket run (odd
            # ends aside), so the first level alone removes over 40 %
            assert prof.affine_additions > prof.nonzero_entries * 0.4
    assert prof.madds >= 0


def test_levels_default_by_size(bc):
    """The default runs no levels (measured slower than the XYZZ pass on a
    B200 at every size); a forced count applies to every size."""
    for forced, n, want in ((-1, 1 << 12, 0), (-1, 1 << 18, 0), (2, 1 << 18, 2)):
        bc.set_affine_levels(forced)
        scalars, k = synth.workload("uniform", n, 990)
        kd = bc.to_device(k)
        bd = bc.malloc(n * 64)
        bc.generator_multiples(kd, bd, n, bc.stream_handle)
        bc.stream_synchronize(bc.stream_handle)
        bc.free(kd)
        _, prof = run(bc, None, scalars, bases_dev=bd, profile=True)
        bc.free(bd)
        bc.set_affine_levels(-1)
        assert prof.affine_levels == want


def test_levels_invalid_count(bc):
    import bellman_cuda as bcm
    assert bc.lib.msm_b200_set_affine_levels(5) == bcm.BC_ERROR_INVALID_VALUE


def test_levels_chunked_host_scalars(bc, oracle):
    """Host-resident (pageable) scalars are processed in chunks, each running
    its own levels over its own sorted entries into the chunk's buckets."""
    n = 1 << 20
    scalars, k = synth.workload("uniform", n, 977)
    kd = bc.to_device(k)
    bd = bc.malloc(n * 64)
    bc.generator_multiples(kd, bd, n, bc.stream_handle)
    bc.stream_synchronize(bc.stream_handle)
    bc.free(kd)
    res = np.zeros((254, 24), np.uint32)
    bc.set_affine_levels(2)
    try:
        assert bc.msm_execute_async(bc.pool_handle, bc.stream_handle, bd, np.ascontiguousarray(scalars), res, 20) == 0
        bc.stream_synchronize(bc.stream_handle)
    finally:
        bc.set_affine_levels(-1)
        bc.free(bd)
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)
