"""The MSM request server (msm_b200_server_*), through the C ABI: continuous
batching over one resident table.  Every request's normalised point is the
same alone and in the mix (bit-exact, and equal to the oracle's checksum MSM),
with device, pinned and pageable inputs and outputs; the scheduler really
groups requests and overlaps groups on the device; admission respects the
scratch budget and fails requests that can never fit; Poisson arrivals from
another thread all complete with ordered timestamps."""
import threading
import time

import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu


class Env:
    def __init__(self, n_table):
        import bellman_cuda as bcm
        self.bcm = bcm
        bc = self.bc = bcm.BellmanCuda()
        bc.set_device(0)
        bc.msm_set_up()
        self.stream = bc.stream_create(True)
        self.k = synth.base_multipliers(51, n_table)
        kd = bc.to_device(self.k)
        self.bases = bc.malloc(n_table * 64)
        bc.generator_multiples(kd, self.bases, n_table, self.stream)
        bc.stream_synchronize(self.stream)
        bc.free(kd)
        self.table = bc.base_table_create(self.bases, n_table, self.stream)


@pytest.fixture(scope="module")
def env():
    e = Env(1 << 18)
    yield e
    e.bc.base_table_destroy(e.table)
    e.bc.free(e.bases)


def make_requests(count, seed, lo=8, hi=18):
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = np.rint(np.exp2(rng.uniform(lo, hi, count))).astype(int)
    reqs = []
    for j, n in enumerate(sizes):
        s = synth.skewed_scalars(seed * 100 + j, int(n)) if j % 2 else synth.uniform_scalars(seed * 100 + j, int(n))
        reqs.append(s)
    return reqs


class Buffers:
    """Scalars and results of one request, in the memory kind chosen by j."""

    def __init__(self, bc, scalars, j):
        self.bc = bc
        self.kind = ("device", "pinned", "pageable")[j % 3]
        self.owned, self.pinned = [], []
        if self.kind == "device":
            self.s = bc.to_device(scalars)
            self.r = bc.malloc(254 * 96)
            self.owned += [self.s, self.r]
        elif self.kind == "pinned":
            arr, ptr = bc.pinned_array(scalars.shape)
            arr[...] = scalars
            self.s = ptr
            self.r_arr, self.r = bc.pinned_array((254, 24))
            self.pinned += [ptr, self.r]
        else:
            self.s = np.ascontiguousarray(scalars)
            self.r_arr = np.zeros((254, 24), np.uint32)
            self.r = self.r_arr

    def results(self):
        if self.kind == "device":
            return self.bc.from_device(self.r, (254, 24))
        return np.array(self.r_arr)

    def free(self):
        for p in self.owned:
            self.bc.free(p)
        for p in self.pinned:
            self.bc.free_host(p)


def run_all(env, server, reqs):
    bufs = [Buffers(env.bc, s, j) for j, s in enumerate(reqs)]
    tickets = [env.bc.server_submit(server, b.s, len(s), b.r) for b, s in zip(bufs, reqs)]
    out = []
    for t, b in zip(tickets, bufs):
        rc, times = env.bc.server_wait(server, t)
        assert rc == 0
        assert times.submit_us <= times.start_us <= times.done_us
        out.append(b.results())
        b.free()
    return out


def test_server_same_alone_and_in_mix(env, oracle):
    bc = env.bc
    reqs = make_requests(36, 3)
    server = bc.server_create(env.table, 2 << 30, streams=4, max_group=8)
    mixed = run_all(env, server, reqs)
    stats = bc.server_stats(server)
    assert stats.requests == len(reqs)
    assert stats.groups < len(reqs), "requests were never grouped"
    assert stats.max_inflight_groups >= 2, "groups never overlapped on the device"
    bc.server_destroy(server)
    alone_server = bc.server_create(env.table, 2 << 30, streams=1, max_group=1)
    for j, (s, res) in enumerate(zip(reqs, mixed)):
        alone = run_all(env, alone_server, [s])[0]
        got = oracle.horner(res)
        assert got == oracle.horner(alone), f"request {j} differs between the mix and alone"
        assert got == oracle.msm_checksum(env.k[: len(s)], s), f"request {j}"
    bc.server_destroy(alone_server)


def test_server_admission_budget(env, oracle):
    """A 48 MiB arena admits small requests a few at a time; a 2^18-point request
    (larger than the whole arena) fails with bc_error_memory_allocation."""
    bc = env.bc
    server = bc.server_create(env.table, 48 << 20, streams=4, max_group=16)
    small = make_requests(12, 5, lo=8, hi=12)
    big = synth.uniform_scalars(77, 1 << 18)
    bufs = [Buffers(bc, s, 0) for s in small]
    big_buf = Buffers(bc, big, 0)
    tickets = [bc.server_submit(server, b.s, len(s), b.r) for b, s in zip(bufs, small)]
    big_ticket = bc.server_submit(server, big_buf.s, len(big), big_buf.r)
    for t, b, s in zip(tickets, bufs, small):
        rc, _ = bc.server_wait(server, t)
        assert rc == 0
        assert oracle.horner(b.results()) == oracle.msm_checksum(env.k[: len(s)], s)
        b.free()
    rc, _ = bc.server_wait(server, big_ticket)
    assert rc == env.bcm.BC_ERROR_MEMORY_ALLOCATION
    big_buf.free()
    assert bc.server_stats(server).arena_used == 0
    bc.server_destroy(server)


def test_server_poisson_arrivals(env, oracle):
    """Requests arrive from another thread at Poisson times while earlier ones run."""
    bc = env.bc
    reqs = make_requests(24, 9, lo=10, hi=17)
    bufs = [Buffers(bc, s, j) for j, s in enumerate(reqs)]
    server = bc.server_create(env.table, 1 << 30, streams=3, max_group=8)
    rng = np.random.Generator(np.random.PCG64(4))
    gaps = rng.exponential(0.0004, len(reqs))
    tickets = [None] * len(reqs)

    def producer():
        t = time.perf_counter()
        for j, (b, s) in enumerate(zip(bufs, reqs)):
            t += gaps[j]
            while time.perf_counter() < t:
                pass
            tickets[j] = bc.server_submit(server, b.s, len(s), b.r)

    th = threading.Thread(target=producer)
    th.start()
    th.join()
    last_submit = 0.0
    for j, (t, b, s) in enumerate(zip(tickets, bufs, reqs)):
        rc, times = bc.server_wait(server, t)
        assert rc == 0
        assert times.submit_us >= last_submit
        last_submit = times.submit_us
        assert oracle.horner(b.results()) == oracle.msm_checksum(env.k[: len(s)], s), f"request {j}"
        b.free()
    bc.server_destroy(server)
