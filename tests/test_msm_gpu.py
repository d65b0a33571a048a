"""GPU parity of msm_execute_async (and the any-length extension) against the
oracle, the golden fixtures and, when built, the reference's own sm_100a
library on identical inputs.  Every comparison is bit-exact on the normalised
affine point (standard form, fully reduced, infinity flagged), after the
caller-side Horner reduction of the 254 results."""
import ctypes
import os

import numpy as np
import pytest

import msm_helpers as H
import synth

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_GPU = os.path.join(REPO, "oracle", "_ref", "libbellman-cuda-ref.so")


class Runner:
    """One library (ours or the reference) driven through the bellman-cuda ABI."""

    def __init__(self, path=None):
        import bellman_cuda as bcm
        self.bc = bcm.BellmanCuda(path) if path else bcm.BellmanCuda()
        self.bc.set_device(0)
        self.bc.ff_set_up(25, 14)
        self.bc.msm_set_up()
        self.pool = self.bc.mem_pool_create(0)
        self.stream = self.bc.stream_create(True)

    def upload(self, a):
        return self.bc.to_device(np.ascontiguousarray(a))

    def msm(self, bases, scalars, log_n=None, scalars_mem="device", results_mem="device", bases_dev=None):
        bc = self.bc
        n = len(scalars)
        if log_n is None:
            log_n = max(0, (n - 1).bit_length())
        full = 1 << log_n
        if full != n:  # pad with zero scalars: zero digits contribute nothing
            scalars = np.concatenate([scalars, np.zeros((full - n, 8), np.uint32)])
            bases = np.concatenate([bases, np.repeat(bases[:1], full - n, axis=0)])
        owned = []
        if bases_dev is None:
            bases_dev = self.upload(bases)
            owned.append(bases_dev)
        pinned = []
        if scalars_mem == "device":
            s = self.upload(scalars)
            owned.append(s)
        elif scalars_mem == "pinned":
            s, ptr = bc.pinned_array(scalars.shape)
            s[...] = scalars
            pinned.append(ptr)
        else:
            s = np.ascontiguousarray(scalars)
        results = np.zeros((254, 24), np.uint32)
        if results_mem == "device":
            r = bc.malloc(results.nbytes)
            owned.append(r)
        elif results_mem == "pinned":
            r, ptr = bc.pinned_array((254, 24))
            pinned.append(ptr)
        else:
            r = results
        bc.msm(self.pool, self.stream, bases_dev, s, r, log_n)
        bc.stream_synchronize(self.stream)
        if results_mem == "device":
            bc.memcpy(results, r, results.nbytes)
        elif results_mem == "pinned":
            results[...] = r
        for p in owned:
            bc.free(p)
        for p in pinned:
            bc.free_host(p)
        return results


@pytest.fixture(scope="module")
def gpu():
    return Runner()


@pytest.fixture(scope="module")
def ref_gpu():
    if not os.path.exists(REF_GPU):
        pytest.skip("reference sm_100a build absent (make -C oracle ref)")
    return Runner(REF_GPU)


def generated_bases(gpu, k):
    """k_i * G on the device (extension kernel); returns (device pointer, host copy)."""
    bc = gpu.bc
    kd = gpu.upload(k)
    bd = bc.malloc(len(k) * 64)
    bc.generator_multiples(kd, bd, len(k), gpu.stream)
    bc.stream_synchronize(gpu.stream)
    bc.free(kd)
    return bd, bc.from_device(bd, (len(k), 16))


# ---------------------------------------------------------------------------
@pytest.mark.parametrize("case", H.load_json("msm_small.json")["cases"], ids=lambda c: c["name"])
def test_small_golden(gpu, oracle, case):
    table = H.load_g_bases()
    bases = H.mont_point_array([table[i] for i in case["bases"]])
    scalars = H.mont_scalar_array([int(s, 16) for s in case["scalars"]])
    assert oracle.horner(gpu.msm(bases, scalars)) == H.expected_point(case)


def test_config0_golden(gpu, oracle):
    """N = 2^12, seed 0, bases k_i*G: the committed reference result."""
    cfg = H.load_json("config0.json")
    scalars, k = synth.workload("uniform", cfg["n"], cfg["seed"])
    bases = oracle.gen_bases(k)
    assert oracle.horner(gpu.msm(bases, scalars)) == H.expected_point(cfg)


@pytest.mark.parametrize("log_n", [0, 1, 2, 3, 4, 5, 7, 8, 10, 11, 13, 14, 16])
def test_sizes_table_bases(gpu, oracle, log_n):
    """Reference-test style (tests/msm_test.cu:155-170): bases from the 256-point
    table, so repeated bases exercise the doubling branches."""
    bases, scalars, k = H.table_workload(1 << log_n, 10 + log_n)
    assert oracle.horner(gpu.msm(bases, scalars)) == oracle.msm_checksum(k, scalars)


@pytest.mark.parametrize("dist", ["uniform", "skewed"])
@pytest.mark.parametrize("log_n", [12, 16, 18])
def test_generated_bases(gpu, oracle, dist, log_n):
    n = 1 << log_n
    scalars, k = synth.workload(dist, n, 100 + log_n)
    bd, _ = generated_bases(gpu, k)
    res = gpu.msm(None, scalars, bases_dev=bd)
    gpu.bc.free(bd)
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)


def test_generator_multiples_match_oracle(gpu, oracle):
    k = synth.base_multipliers(77, 1024)
    k[0] = 0
    k[0, 0] = 1  # 1 * G
    k[1] = H.limbs(H.R - 1)  # -G
    _, host = generated_bases(gpu, k)
    assert (host == oracle.gen_bases(k)).all()


def test_edge_scalars(gpu, oracle):
    table = H.load_g_bases()
    n = 64
    bases = H.mont_point_array([table[i % 256] for i in range(n)])
    k = np.zeros((n, 8), np.uint32)
    k[:, 0] = (np.arange(n) % 256) + 1
    for values in ([0] * n, [1] * n, [H.R - 1] * n, [(H.R - 1) // 2] * n, [(H.R + 1) // 2] * n, [1 << 253] * n,
                   [(1 << 16) + i for i in range(n)]):
        scalars = H.mont_scalar_array(values)
        assert oracle.horner(gpu.msm(bases, scalars)) == oracle.msm_checksum(k, scalars)


def test_cancellation_and_repeats(gpu, oracle):
    """s*P + (r-s)*P = 0 and many copies of one base in one bucket."""
    table = H.load_g_bases()
    bases = H.mont_point_array([table[3]] * 256)
    vals = [7] * 128 + [H.R - 7] * 128
    scalars = H.mont_scalar_array(vals)
    assert oracle.horner(gpu.msm(bases, scalars))[0]
    scalars = H.mont_scalar_array([5] * 256)
    assert oracle.horner(gpu.msm(bases, scalars)) == oracle.affine_mul(1, 2, 4 * 5 * 256)


@pytest.mark.parametrize("smem,rmem", [("device", "device"), ("pinned", "pinned"), ("pageable", "pageable"),
                                        ("pinned", "device"), ("device", "pageable")])
def test_memory_residence(gpu, oracle, smem, rmem):
    """Scalars and results in device, pinned or pageable memory (msm_test.cu:172-260)."""
    bases, scalars, k = H.table_workload(1 << 12, 3)
    assert oracle.horner(gpu.msm(bases, scalars, scalars_mem=smem, results_mem=rmem)) == oracle.msm_checksum(k, scalars)


def test_host_bases(gpu, oracle):
    """Bases in pageable host memory are copied in, like the reference (src/msm.cu:175-182)."""
    import bellman_cuda as bcm
    bases, scalars, k = H.table_workload(1 << 10, 4)
    res = np.zeros((254, 24), np.uint32)
    gpu.bc.msm(gpu.pool, gpu.stream, np.ascontiguousarray(bases), np.ascontiguousarray(scalars), res, 10)
    gpu.bc.stream_synchronize(gpu.stream)
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)
    del bcm


def test_events_and_callbacks(gpu, oracle):
    """h2d / d2h events are recorded and callbacks fire when copies happen."""
    import bellman_cuda as bcm
    bc = gpu.bc
    bases, scalars, k = H.table_workload(1 << 11, 5)
    bd = gpu.upload(bases)
    fired = []
    cb = bcm.HOST_FN(lambda data: fired.append(data))
    e1, e2 = bc.event_create(), bc.event_create()
    res = np.zeros((254, 24), np.uint32)
    bc.msm(gpu.pool, gpu.stream, bd, np.ascontiguousarray(scalars), res, 11, h2d_event=e1, h2d_callback=cb, h2d_data=1,
           d2h_event=e2, d2h_callback=cb, d2h_data=2)
    bc.stream_synchronize(gpu.stream)
    bc.event_synchronize(e1)
    bc.event_synchronize(e2)
    assert sorted(fired) == [1, 2]
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)
    bc.event_destroy(e1)
    bc.event_destroy(e2)
    bc.free(bd)


@pytest.mark.parametrize("log_n,smem,bases_on_host", [(20, "pageable", False), (21, "pinned", True), (22, "pinned", False),
                                                     (23, "pinned", False)])
def test_chunked_host_inputs(gpu, oracle, log_n, smem, bases_on_host):
    """Host-resident inputs of 2^20 points and more are processed in 2 chunks (3 from
    2^23) whose copies overlap the previous chunk's work; every chunk after the
    first is folded into the MSM's buckets.  Skewed scalars put the heavy buckets
    in every chunk."""
    n = 1 << log_n
    scalars, k = synth.workload("skewed" if log_n % 2 else "uniform", n, 200 + log_n)
    bd, bases = generated_bases(gpu, k)
    if bases_on_host:  # pageable bases and pinned scalars, both copied chunk by chunk
        bc = gpu.bc
        bc.free(bd)
        hs, hs_ptr = bc.pinned_array(scalars.shape)
        hs[...] = scalars
        res = np.zeros((254, 24), np.uint32)
        bc.msm(gpu.pool, gpu.stream, np.ascontiguousarray(bases), hs_ptr, res, log_n)
        bc.stream_synchronize(gpu.stream)
        bc.free_host(hs_ptr)
    else:
        res = gpu.msm(None, scalars, scalars_mem=smem, bases_dev=bd)
        gpu.bc.free(bd)
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)


def test_chunked_events_and_callbacks(gpu, oracle):
    """The h2d event and callback fire after the last chunk's copy, d2h after the results."""
    import bellman_cuda as bcm
    bc = gpu.bc
    n = 1 << 20
    scalars, k = synth.workload("uniform", n, 211)
    bd, _ = generated_bases(gpu, k)
    hs, hs_ptr = bc.pinned_array(scalars.shape)
    hs[...] = scalars
    fired = []
    cb = bcm.HOST_FN(lambda data: fired.append(data))
    e1, e2 = bc.event_create(), bc.event_create()
    res = np.zeros((254, 24), np.uint32)
    bc.msm(gpu.pool, gpu.stream, bd, hs_ptr, res, 20, h2d_event=e1, h2d_callback=cb, h2d_data=1,
           d2h_event=e2, d2h_callback=cb, d2h_data=2)
    bc.stream_synchronize(gpu.stream)
    bc.event_synchronize(e1)
    bc.event_synchronize(e2)
    assert sorted(fired) == [1, 2]
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)
    for ev in (e1, e2):
        bc.event_destroy(ev)
    bc.free(bd)
    bc.free_host(hs_ptr)


def test_concurrent_streams_and_threads(gpu, oracle):
    """msm_execute_async is re-entrant: MSMs on different streams, enqueued from
    different host threads, overlap on the device and all come out right
    (the reference's tests/bc_test.cu:126-170 does the same with its MSM)."""
    import threading
    bc = gpu.bc
    jobs = []
    for j, log_n in enumerate((12, 16, 18, 20)):
        bases, scalars, k = H.table_workload(1 << log_n, 40 + j)
        jobs.append((log_n, gpu.upload(bases), gpu.upload(scalars), bc.malloc(254 * 96), k, scalars, bc.stream_create(True)))
    errors = []

    def run(job):
        log_n, bd, sd, rd, _, _, st = job
        try:
            for _ in range(3):
                bc.msm(gpu.pool, st, bd, sd, rd, log_n)
            bc.stream_synchronize(st)
        except Exception as e:  # reported below, on the main thread
            errors.append(e)

    threads = [threading.Thread(target=run, args=(job,)) for job in jobs]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for log_n, bd, sd, rd, k, scalars, st in jobs:
        assert oracle.horner(bc.from_device(rd, (254, 24))) == oracle.msm_checksum(k, scalars), f"2^{log_n}"
        for p in (bd, sd, rd):
            bc.free(p)
        bc.stream_destroy(st)


def test_invalid_arguments(gpu):
    bc = gpu.bc
    res = np.zeros((254, 24), np.uint32)
    assert bc.msm_execute_async(gpu.pool, gpu.stream, None, None, res, 4) == 1
    assert bc.msm_execute_async(gpu.pool, gpu.stream, 16, 16, res, 40) == 1
    assert bc.lib.ff_set_up(29, 14) == 1


@pytest.mark.parametrize("window_bits", [2, 3, 5, 8, 11, 13, 16, 17, 20])
def test_any_window_and_length(gpu, oracle, window_bits):
    """The extension entry point: any length, forced window widths."""
    n = 3001
    bases, scalars, k = H.table_workload(n, 6)
    bd, sd = gpu.upload(bases), gpu.upload(scalars)
    rd = gpu.bc.malloc(254 * 96)
    assert gpu.bc.msm_any(gpu.pool, gpu.stream, bd, sd, rd, n, window_bits) == 0
    gpu.bc.stream_synchronize(gpu.stream)
    res = gpu.bc.from_device(rd, (254, 24))
    for p in (bd, sd, rd):
        gpu.bc.free(p)
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)


@pytest.mark.parametrize("n,window_bits", [(4097, 13), (8191, 15), (12289, 16), (65537, 17), (200003, 17), (131071, 9)])
def test_sort_tile_edges(gpu, oracle, n, window_bits):
    """Lengths just past and short of whole sort tiles (4096 keys), skewed
    scalars (many zero digits, one heavy bucket): the first pass's partial last
    tile and the later passes over windows whose nonzero entries start
    mid-tile; 9-bit windows take one radix pass, the others two.  Below 128
    sort tiles these run the histogram + scan + scatter passes; the look-back
    passes over such windows are covered by test_lookback_ranking_paths and
    the tests from 2^19 points up."""
    scalars, k = synth.workload("skewed", n, 500 + n % 97)
    bd, _ = generated_bases(gpu, k)
    sd = gpu.upload(scalars)
    rd = gpu.bc.malloc(254 * 96)
    assert gpu.bc.msm_any(gpu.pool, gpu.stream, bd, sd, rd, n, window_bits) == 0
    gpu.bc.stream_synchronize(gpu.stream)
    res = gpu.bc.from_device(rd, (254, 24))
    for p in (bd, sd, rd):
        gpu.bc.free(p)
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)


def crafted_window_scalars(n: int, seed: int):
    """Scalars with chosen 16-bit signed digits, one sort-key pattern per
    window (window w of width 16 holds bits [16 w, 16 w + 16); every digit
    lies in [0, 2^15], so the recoding takes it as is, and the top digit
    stays below 2^11, so s < r / 2 and the fold keeps s).  Windows cycle
    through four patterns of the key |d| - 1: uniform; low byte 5 or 12;
    low byte 5 or 13; 95 % zero digits and uniform otherwise.  Returns
    (Montgomery scalars, the (16, n) digit matrix)."""
    g = np.random.Generator(np.random.PCG64(np.random.SeedSequence([seed, 9])))
    digits = np.zeros((16, n), np.int64)
    for w in range(16):
        mode = w % 4
        if mode == 0:
            d = g.integers(1, (1 << 15) + 1, n)
        elif mode in (1, 2):
            low = np.where(g.integers(0, 2, n) == 0, 5, 12 if mode == 1 else 13)
            d = ((g.integers(0, 1 << 7, n) << 8) | low) + 1
        else:
            d = np.where(g.random(n) < 0.95, 0, g.integers(1, (1 << 15) + 1, n))
        if w == 15:
            d = np.minimum(d, 1 << 11)
        digits[w] = d
    limbs = np.zeros((n, 8), np.uint64)
    for w in range(16):
        limbs[:, w // 2] |= digits[w].astype(np.uint64) << np.uint64(16 * (w % 2))
    mont = np.empty((n, 8), np.uint32)
    for i in range(n):
        v = int.from_bytes(limbs[i].astype(np.uint32).tobytes(), "little")
        assert 2 * v < synth.R
        mont[i] = np.frombuffer(((v * synth.MONT_R) % synth.R).to_bytes(32, "little"), np.uint32)
    return mont, digits


def test_lookback_ranking_paths(gpu, oracle):
    """The second radix pass ranks a tile with shared atomics when its keys'
    low bytes span fewer than eight values and with ballots otherwise.  At
    n = 2^19 + 4099 and 16-bit windows (two passes, look-back tiles of 4096
    keys over each window's nonzero entries, sorted by the low byte by the
    first pass) the crafted windows give tiles spanning 1-3 values (uniform
    keys), exactly 7 (low bytes 5 and 12: the atomic path's last counter
    row), exactly 8 (5 and 13: ballots) and dozens (sparse windows: ballots).
    The spans are checked on the host first; the MSM must equal the checksum
    oracle."""
    n = (1 << 19) + 4099
    scalars, digits = crafted_window_scalars(n, 41)
    spans = set()
    for w in range(16):
        keys = np.sort((digits[w][digits[w] > 0] - 1) & 0xFF, kind="stable")
        for t in range(0, len(keys), 4096):
            tile = keys[t:t + 4096]
            spans.add(int(tile[-1] - tile[0]))
    assert {0, 7, 8}.issubset(spans) and max(spans) > 8
    k = synth.base_multipliers(41, n)
    bd, _ = generated_bases(gpu, k)
    sd = gpu.upload(scalars)
    rd = gpu.bc.malloc(254 * 96)
    assert gpu.bc.msm_any(gpu.pool, gpu.stream, bd, sd, rd, n, 16) == 0
    gpu.bc.stream_synchronize(gpu.stream)
    res = gpu.bc.from_device(rd, (254, 24))
    for p in (bd, sd, rd):
        gpu.bc.free(p)
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)


@pytest.mark.parametrize("dist", ["uniform", "skewed"])
def test_full_size_2_22(gpu, oracle, dist):
    """Configs 1 and 2 (N = 2^22, seeds 1 and 2) against the checksum oracle."""
    seed = 1 if dist == "uniform" else 2
    n = 1 << 22
    scalars, k = synth.workload(dist, n, seed)
    bd, _ = generated_bases(gpu, k)
    res = gpu.msm(None, scalars, bases_dev=bd)
    gpu.bc.free(bd)
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)


# ---- the reference's own sm_100a build on identical inputs ----------------------
@pytest.mark.parametrize("log_n", [0, 8, 12])
def test_reference_parity_small(gpu, ref_gpu, oracle, log_n):
    bases, scalars, k = H.table_workload(1 << log_n, 20 + log_n)
    ours = oracle.horner(gpu.msm(bases, scalars))
    theirs = oracle.horner(ref_gpu.msm(bases, scalars))
    assert ours == theirs == oracle.msm_checksum(k, scalars)


@pytest.mark.parametrize("dist", ["uniform", "skewed"])
def test_reference_parity_2_22(gpu, ref_gpu, oracle, dist):
    seed = 1 if dist == "uniform" else 2
    n = 1 << 22
    scalars, k = synth.workload(dist, n, seed)
    bd, bases = generated_bases(gpu, k)
    ours = oracle.horner(gpu.msm(None, scalars, bases_dev=bd))
    gpu.bc.free(bd)
    theirs = oracle.horner(ref_gpu.msm(bases, scalars))
    assert ours == theirs


# ---- memory fit (reference src/msm.cu:431-459) and large device-resident sizes ----
def limited_pool(device: int, max_bytes: int):
    """A memory pool that can hold at most max_bytes (cudaMemPoolProps.maxSize),
    made through cuda-python; returns (bc_mem_pool handle, destroy function)."""
    rt = pytest.importorskip("cuda.bindings.runtime")
    import bellman_cuda as bcm
    props = rt.cudaMemPoolProps()
    props.allocType = rt.cudaMemAllocationType.cudaMemAllocationTypePinned
    props.location.type = rt.cudaMemLocationType.cudaMemLocationTypeDevice
    props.location.id = device
    props.maxSize = max_bytes
    err, pool = rt.cudaMemPoolCreate(props)
    assert err == rt.cudaError_t.cudaSuccess, err
    handle = bcm.Handle()
    handle.handle = int(pool)
    return handle, lambda: rt.cudaMemPoolDestroy(pool)


@pytest.mark.parametrize("scalars_mem", ["device", "pinned"])
def test_memory_fit_in_a_small_pool(gpu, oracle, scalars_mem):
    """A pool that cannot hold the whole-size scratch of a 2^22 MSM (half of it):
    the call runs in smaller chunks instead of failing, device-resident or
    host-resident scalars alike, bit-exact; a pool too small for even the
    smallest chunk gives bc_error_memory_allocation (nothing enqueued)."""
    import bellman_cuda as bcm
    bc = gpu.bc
    n = 1 << 22
    full = bc.scratch_bytes(n)
    scalars, k = synth.workload("skewed" if scalars_mem == "device" else "uniform", n, 231)
    bd, _ = generated_bases(gpu, k)
    rd = bc.malloc(254 * 96)
    owned, pinned = [], []
    if scalars_mem == "device":
        sd = gpu.upload(scalars)
        owned.append(sd)
    else:
        hs, sd = bc.pinned_array(scalars.shape)
        hs[...] = scalars
        pinned.append(sd)
    pool, destroy = limited_pool(0, full // 2)
    try:
        assert bc.msm_execute_async(pool, gpu.stream, bd, sd, rd, 22) == bcm.BC_SUCCESS
        bc.stream_synchronize(gpu.stream)
        assert oracle.horner(bc.from_device(rd, (254, 24))) == oracle.msm_checksum(k, scalars)
    finally:
        destroy()
    tiny, destroy_tiny = limited_pool(0, 32 << 20)
    try:
        assert bc.msm_execute_async(tiny, gpu.stream, bd, sd, rd, 22) == bcm.BC_ERROR_MEMORY_ALLOCATION
        bc.stream_synchronize(gpu.stream)
    finally:
        destroy_tiny()
    for p in owned + [bd, rd]:
        bc.free(p)
    for p in pinned:
        bc.free_host(p)


@pytest.mark.parametrize("log_n", [24, 26])
def test_device_resident_large(gpu, oracle, log_n):
    """Device-resident MSMs past 2^22 (the reference tests and benchmarks up to
    2^26, tests/msm_test.cu:253-260): every window stride and entry index past
    2^31 entries, against the checksum oracle."""
    n = 1 << log_n
    scalars, k = synth.workload("skewed" if log_n == 24 else "uniform", n, 240 + log_n)
    kd = gpu.upload(k)
    bd = gpu.bc.malloc(n * 64)
    gpu.bc.generator_multiples(kd, bd, n, gpu.stream)
    gpu.bc.stream_synchronize(gpu.stream)
    gpu.bc.free(kd)
    res = gpu.msm(None, scalars, bases_dev=bd)
    gpu.bc.free(bd)
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)


def test_reference_parity_2_24(gpu, ref_gpu, oracle):
    n = 1 << 24
    scalars, k = synth.workload("uniform", n, 265)
    bd, bases = generated_bases(gpu, k)
    ours = oracle.horner(gpu.msm(None, scalars, bases_dev=bd))
    gpu.bc.free(bd)
    theirs = oracle.horner(ref_gpu.msm(bases, scalars))
    assert ours == theirs == oracle.msm_checksum(k, scalars)


@pytest.mark.parametrize("dist", ["uniform", "skewed"])
def test_profiled_counts(gpu, oracle, dist):
    """msm_b200_execute_profiled: the work counts match the digits of the
    scalars (nonzero entries = W n - zero digits, counted here on the host with
    the oracle's digit rule), no radix-pass look-back wait gave up, and the
    result is right."""
    n = 1 << 16
    scalars, k = synth.workload(dist, n, 700 + (dist == "skewed"))
    bd, _ = generated_bases(gpu, k)
    sd = gpu.upload(scalars)
    rd = gpu.bc.malloc(254 * 96)
    prof = gpu.bc.msm_profiled(gpu.pool, gpu.stream, bd, sd, rd, n)
    res = gpu.bc.from_device(rd, (254, 24))
    for p in (bd, sd, rd):
        gpu.bc.free(p)
    assert prof.sort_wait_timeouts == 0
    c, windows = prof.window_bits, prof.windows
    assert windows == (254 + c - 1) // c
    # signed digits of min(s, r - s) (the fold of the digit kernel), zero digits counted
    R = H.R
    unmont = pow(H.MONT, -1, R)
    zeros = 0
    for row in scalars:
        s = H.to_int(row) * unmont % R
        s = min(s, R - s)
        carry = 0
        for w in range(windows):
            raw = ((s >> (w * c)) & ((1 << c) - 1)) + carry
            carry = int(raw > (1 << (c - 1)))
            zeros += int(raw in (0, 1 << c))
    assert prof.nonzero_entries == windows * n - zeros
    assert 0 < prof.nonempty_buckets <= windows << (c - 1)
    assert prof.madds == prof.nonzero_entries - prof.nonempty_buckets - prof.heads
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)


@pytest.mark.parametrize("smem", ["pinned", "pageable"])
def test_chunked_host_inputs_ragged(gpu, oracle, smem):
    """Host-resident scalars of a length that is neither a power of two nor a
    multiple of the sort tile (3,000,017 points) through the any-length entry
    point: chunk boundaries fall mid-tile, the last chunk is ragged."""
    n = 3_000_017
    scalars, k = synth.workload("uniform", n, 611)
    bd, _ = generated_bases(gpu, k)
    rd = gpu.bc.malloc(254 * 96)
    pinned = None
    if smem == "pinned":
        hs, pinned = gpu.bc.pinned_array(scalars.shape)
        hs[...] = scalars
        src = pinned
    else:
        src = np.ascontiguousarray(scalars)
    assert gpu.bc.msm_any(gpu.pool, gpu.stream, bd, src, rd, n, 0) == 0
    gpu.bc.stream_synchronize(gpu.stream)
    res = gpu.bc.from_device(rd, (254, 24))
    for p in (bd, rd):
        gpu.bc.free(p)
    if pinned is not None:
        gpu.bc.free_host(pinned)
    assert oracle.horner(res) == oracle.msm_checksum(k, scalars)
