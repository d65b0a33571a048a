"""GPU parity of msm_b200_final_sum_async, the caller-side final reduction
(sum over i of 2^i R_i, src/bellman-cuda.h:496-505) run on the device with a
canonical affine output, against the oracle's host Horner pass
(tests/msm_test.cu:116-126 style): on MSM results of this library and of the
reference's sm_100a build, and on crafted result arrays that reach the
infinity, equal-point and opposite-point branches at every tree level."""
import ctypes

import numpy as np
import pytest

import msm_helpers as H
import synth
from test_msm_gpu import REF_GPU, Runner

pytestmark = pytest.mark.gpu

P = H.P
MONT = H.MONT


@pytest.fixture(scope="module")
def gpu():
    return Runner()


def final_sum(gpu, results, out_mem="device"):
    """Runs the extension on `results` (254 x 24 words, uploaded to the device)
    and returns (infinity, x, y)."""
    import bellman_cuda as bcm
    bc = gpu.bc
    rd = gpu.upload(np.ascontiguousarray(results, dtype=np.uint32))
    if out_mem == "device":
        pd = bc.malloc(ctypes.sizeof(bcm.AffinePoint))
        assert bc.final_sum_async(rd, pd, gpu.stream) == 0
        bc.stream_synchronize(gpu.stream)
        out = bc.from_device(pd, (20,))
        bc.free(pd)
    else:
        view, ptr = bc.pinned_array((20,))
        view[...] = 0xFFFFFFFF
        assert bc.final_sum_async(rd, ptr, gpu.stream) == 0
        bc.stream_synchronize(gpu.stream)
        out = view.copy()
        bc.free_host(ptr)
    bc.free(rd)
    point = bcm.AffinePoint.from_buffer_copy(out.tobytes())
    assert not any(point.reserved)
    return point.as_tuple()


def jacobian(pt, z=1):
    """Montgomery-form Jacobian words of an affine point (None = infinity, the
    reference's (0, 1, 0))."""
    if pt is None:
        return np.concatenate([H.limbs(0), H.limbs(MONT % P), H.limbs(0)])
    x, y = pt
    return np.concatenate([H.limbs(x * z * z % P * MONT % P), H.limbs(y * z ** 3 % P * MONT % P), H.limbs(z * MONT % P)])


def neg(pt):
    return (pt[0], (P - pt[1]) % P)


def results_of(points, zs=None):
    out = np.zeros((254, 24), np.uint32)
    for i in range(254):
        out[i] = jacobian(points.get(i), 1 if zs is None else zs[i])
    return out


def test_msm_results(gpu, oracle):
    """This library's own 254 results (uniform and skewed inputs)."""
    for dist, log_n, seed in (("uniform", 12, 0), ("skewed", 14, 2), ("uniform", 16, 5)):
        scalars, k = synth.workload(dist, 1 << log_n, seed)
        bases = oracle.gen_bases(k)
        res = gpu.msm(bases, scalars)
        assert final_sum(gpu, res) == oracle.horner(res) == oracle.msm_checksum(k, scalars)


def test_reference_results(oracle):
    """The reference build's results (its own window split) reduce to the same point."""
    import os
    if not os.path.exists(REF_GPU):
        pytest.skip("reference sm_100a build absent (make -C oracle ref)")
    ref = Runner(REF_GPU)
    ours = Runner()
    bases, scalars, k = H.table_workload(1 << 12, 21)
    res = ref.msm(bases, scalars)
    assert final_sum(ours, res) == oracle.horner(res) == oracle.msm_checksum(k, scalars)


def test_crafted_branches(gpu, oracle):
    table = H.load_g_bases()  # (i + 1) * G
    G, G2, G4 = table[0], table[1], table[3]
    inf, *g128 = oracle.affine_mul(G[0], G[1], 1 << 128)
    assert not inf
    g128 = tuple(g128)
    cases = {
        "all infinity": {},
        "R0 = G": {0: G},
        "R253 = G": {253: G},
        "R252, R253": {252: G2, 253: table[6]},
        "every bit G": {i: G for i in range(254)},
        "level 0 cancels": {0: G2, 1: neg(G)},           # 2G + 2(-G)
        "level 0 equal": {0: G2, 1: G},                   # 2G + 2G: doubling branch
        "level 1 cancels": {0: neg(G4), 2: G},           # -4G + 4G
        "level 1 equal": {0: G4, 2: G},                   # 4G + 4G
        "level 7 cancels": {0: neg(g128), 128: G},       # -2^128 G + 2^128 G
        "level 7 equal": {0: g128, 128: G},               # 2^128 G + 2^128 G
        "top cancels": {126: neg(G2), 127: G, 253: G},
    }
    for name, pts in cases.items():
        res = results_of(pts)
        assert final_sum(gpu, res) == oracle.horner(res), name
    assert final_sum(gpu, results_of({}))[0]
    assert final_sum(gpu, results_of({0: G})) == (False, *G)
    assert final_sum(gpu, results_of({0: G2, 1: neg(G)}))[0]
    assert final_sum(gpu, results_of({0: neg(G4), 2: G}))[0]
    assert final_sum(gpu, results_of({0: neg(g128), 128: G}))[0]
    assert final_sum(gpu, results_of({0: g128, 128: G})) == oracle.affine_mul(G[0], G[1], 1 << 129)


def test_random_projective_inputs(gpu, oracle):
    """Random multiples with random Z (non-normalised Jacobian), some infinity."""
    table = H.load_g_bases()
    rng = np.random.Generator(np.random.PCG64(31))
    for trial in range(3):
        pts = {i: table[int(rng.integers(0, 256))] for i in range(254) if rng.random() < 0.8}
        for i in list(pts)[::5]:
            pts[i] = neg(pts[i])
        zs = [int.from_bytes(rng.bytes(32), "little") % P or 1 for _ in range(254)]
        res = results_of(pts, zs)
        assert final_sum(gpu, res, "pinned" if trial == 1 else "device") == oracle.horner(res)


def test_invalid_arguments(gpu):
    """Null, pageable or misaligned pointers are refused before any launch."""
    import bellman_cuda as bcm
    bc = gpu.bc
    rd = bc.malloc(254 * 96)
    pd = bc.malloc(ctypes.sizeof(bcm.AffinePoint))
    host = np.zeros(254 * 24, np.uint32)
    assert bc.final_sum_async(None, pd, gpu.stream) == bcm.BC_ERROR_INVALID_VALUE
    assert bc.final_sum_async(rd, None, gpu.stream) == bcm.BC_ERROR_INVALID_VALUE
    assert bc.final_sum_async(host, pd, gpu.stream) == bcm.BC_ERROR_INVALID_VALUE
    assert bc.final_sum_async(rd + 8, pd, gpu.stream) == bcm.BC_ERROR_INVALID_VALUE
    bc.stream_synchronize(gpu.stream)
    bc.free(rd)
    bc.free(pd)


def test_pinned_results_input(gpu, oracle):
    """Results in pinned host memory (msm_execute_async writes them there when
    the caller passes host results) are read in place through their device alias."""
    import bellman_cuda as bcm
    bc = gpu.bc
    bases, scalars, k = H.table_workload(1 << 11, 41)
    res = gpu.msm(bases, scalars)
    view, ptr = bc.pinned_array((254, 24))
    view[...] = res
    pd = bc.malloc(ctypes.sizeof(bcm.AffinePoint))
    assert bc.final_sum_async(ptr, pd, gpu.stream) == 0
    bc.stream_synchronize(gpu.stream)
    point = bcm.AffinePoint.from_buffer_copy(bc.from_device(pd, (20,)).tobytes()).as_tuple()
    bc.free(pd)
    bc.free_host(ptr)
    assert point == oracle.msm_checksum(k, scalars)


def test_batched_results(gpu, oracle):
    """The 254 results of batched instances (one window's partial sums per bit
    position, precomputed multiples) reduce to each instance's MSM."""
    bc = gpu.bc
    n = 5000
    k = synth.base_multipliers(47, n)
    kd = gpu.upload(k)
    bd = bc.malloc(n * 64)
    bc.generator_multiples(kd, bd, n, gpu.stream)
    bc.stream_synchronize(gpu.stream)
    table = bc.base_table_create(bd, n, gpu.stream)
    bc.stream_synchronize(gpu.stream)
    lengths = [n, 1, 777]
    work = [synth.uniform_scalars(700 + j, m) for j, m in enumerate(lengths)]
    batch = bc.batch_create(table, lengths)
    sd = [gpu.upload(s) for s in work]
    rd = [bc.malloc(254 * 96) for _ in lengths]
    bc.batch_execute(batch, sd, rd, gpu.stream)
    bc.stream_synchronize(gpu.stream)
    for m, s, r in zip(lengths, work, rd):
        res = bc.from_device(r, (254, 24))
        assert final_sum(gpu, res) == oracle.msm_checksum(k[:m], s) == oracle.horner(res)
    bc.batch_destroy(batch)
    bc.base_table_destroy(table)
    for p in sd + rd + [kd, bd]:
        bc.free(p)
