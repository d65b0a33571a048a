"""Batched MSMs over one resident base table (msm_b200_base_table_* /
msm_b200_batch_*), through the C ABI: every instance's Horner-reduced,
normalised point equals the oracle's checksum MSM and the plain entry point's
result on the same inputs (bit-exact), for tuned and forced window widths,
re-executions with new scalar/result buffers, a table saved and loaded back,
and the full 64-instance batch of lengths log-uniform in [2^10, 2^22] (seed 3)."""
import pytest

import synth

pytestmark = pytest.mark.gpu


class Lib:
    def __init__(self):
        import bellman_cuda as bcm
        self.bcm = bcm
        self.bc = bcm.BellmanCuda()
        self.bc.set_device(0)
        self.bc.msm_set_up()
        self.pool = self.bc.mem_pool_create(0)
        self.stream = self.bc.stream_create(True)

    def generated_bases(self, k):
        bc = self.bc
        kd = bc.to_device(k)
        bd = bc.malloc(len(k) * 64)
        bc.generator_multiples(kd, bd, len(k), self.stream)
        bc.stream_synchronize(self.stream)
        bc.free(kd)
        return bd

    def run_batch(self, table, scalars_list, window_bits=None):
        """One execution; returns the (254, 24) results of every instance."""
        bc = self.bc
        counts = [len(s) for s in scalars_list]
        batch = bc.batch_create(table, counts, window_bits)
        sd = [bc.to_device(s) for s in scalars_list]
        rd = [bc.malloc(254 * 96) for _ in counts]
        bc.batch_execute(batch, sd, rd, self.stream)
        bc.stream_synchronize(self.stream)
        out = [bc.from_device(r, (254, 24)) for r in rd]
        for p in sd + rd:
            bc.free(p)
        bc.batch_destroy(batch)
        return out

    def plain(self, bases_dev, scalars):
        bc = self.bc
        sd, rd = bc.to_device(scalars), bc.malloc(254 * 96)
        assert bc.msm_any(self.pool, self.stream, bases_dev, sd, rd, len(scalars)) == 0
        bc.stream_synchronize(self.stream)
        res = bc.from_device(rd, (254, 24))
        bc.free(sd)
        bc.free(rd)
        return res


@pytest.fixture(scope="module")
def lib():
    return Lib()


@pytest.fixture(scope="module")
def table16(lib):
    """2^16 generated bases k_i G and a table with the tuned widths."""
    n = 1 << 16
    k = synth.base_multipliers(41, n)
    bd = lib.generated_bases(k)
    table = lib.bc.base_table_create(bd, n, lib.stream)
    yield k, bd, table
    lib.bc.base_table_destroy(table)
    lib.bc.free(bd)


SMALL_LENGTHS = [1, 2, 3, 17, 100, 1000, 4096, 5000, 30000, 65536, 65535, 12345]


def test_batch_tuned_widths(lib, oracle, table16):
    k, bd, table = table16
    work = [synth.skewed_scalars(500 + j, n) if j % 2 else synth.uniform_scalars(500 + j, n) for j, n in enumerate(SMALL_LENGTHS)]
    results = lib.run_batch(table, work)
    for j, (n, s, res) in enumerate(zip(SMALL_LENGTHS, work, results)):
        got = oracle.horner(res)
        assert got == oracle.msm_checksum(k[:n], s), f"instance {j} (n={n})"
        assert got == oracle.horner(lib.plain(bd, s)), f"instance {j} (n={n}) vs the plain entry point"


@pytest.mark.parametrize("widths", [[2, 5, 9], [13, 16, 17], [11, 20]])
def test_batch_forced_widths(lib, oracle, widths):
    """Instances of one batch with different forced widths (separate reduction groups)."""
    n = 20000
    kk = synth.base_multipliers(43, n)
    bd = lib.generated_bases(kk)
    table = lib.bc.base_table_create(bd, n, lib.stream, window_bits=widths)
    lengths = [n, 777, 1, 19999, 4096, 3][: 2 * len(widths)]
    wb = [widths[j % len(widths)] for j in range(len(lengths))]
    work = [synth.skewed_scalars(600 + j, m) if j % 2 else synth.uniform_scalars(600 + j, m) for j, m in enumerate(lengths)]
    results = lib.run_batch(table, work, wb)
    for j, (m, s, res) in enumerate(zip(lengths, work, results)):
        assert oracle.horner(res) == oracle.msm_checksum(kk[:m], s), f"instance {j} (n={m}, c={wb[j]})"
    lib.bc.base_table_destroy(table)
    lib.bc.free(bd)


def test_batch_reexecution_new_buffers(lib, oracle, table16):
    """The captured graph replays with new scalar and result pointers."""
    k, _, table = table16
    bc = lib.bc
    lengths = [3000, 65536, 70, 40000]
    batch = bc.batch_create(table, lengths)
    for rep in range(3):
        work = [synth.uniform_scalars(700 + 10 * rep + j, n) for j, n in enumerate(lengths)]
        sd = [bc.to_device(s) for s in work]
        rd = [bc.malloc(254 * 96) for _ in lengths]
        bc.batch_execute(batch, sd, rd, lib.stream)
        bc.stream_synchronize(lib.stream)
        for j, (n, s, r) in enumerate(zip(lengths, work, rd)):
            assert oracle.horner(bc.from_device(r, (254, 24))) == oracle.msm_checksum(k[:n], s), f"rep {rep} instance {j}"
        for p in sd + rd:
            bc.free(p)
    bc.batch_destroy(batch)


def test_batch_invalid_arguments(lib, table16):
    _, _, table = table16
    bc = lib.bc
    assert bc.batch_create_raw(table, [])[0] == 1
    assert bc.batch_create_raw(table, [0])[0] == 1
    assert bc.batch_create_raw(table, [(1 << 16) + 1])[0] == 1  # longer than the table
    assert bc.batch_create_raw(table, [10], window_bits=[23])[0] == 1  # width not in the table
    assert bc.batch_create_raw(table, [10] * 257)[0] == 1


def test_table_export_import(lib, oracle, table16):
    """A table saved and loaded again (no recomputation) gives the same results;
    truncated or corrupted images are rejected."""
    k, _, table = table16
    bc = lib.bc
    img = bc.base_table_export(table)
    rc, copy = bc.base_table_import_raw(img, lib.stream)
    assert rc == 0
    assert bc.base_table_bytes(copy) == bc.base_table_bytes(table)
    assert (bc.base_table_export(copy) == img).all()
    lengths = [65536, 999, 4]
    work = [synth.uniform_scalars(800 + j, n) for j, n in enumerate(lengths)]
    for a, b, n, s in zip(lib.run_batch(table, work), lib.run_batch(copy, work), lengths, work):
        assert oracle.horner(a) == oracle.horner(b) == oracle.msm_checksum(k[:n], s)
    bc.base_table_destroy(copy)
    assert bc.base_table_import_raw(img[: len(img) - 64], lib.stream)[0] == 1
    bad = img.copy()
    bad[0] ^= 1
    assert bc.base_table_import_raw(bad, lib.stream)[0] == 1


def test_batch_config3_full(lib, oracle):
    """64 instances, lengths log-uniform in [2^10, 2^22] (seed 3), prefixes of one
    2^22-point table, even instances uniform and odd ones skewed."""
    lengths = synth.batch_lengths(3, 64)
    n_table = 1 << 22
    k = synth.base_multipliers(3, n_table)
    bd = lib.generated_bases(k)
    table = lib.bc.base_table_create(bd, n_table, lib.stream)
    work = synth.batch_workload(3, lengths)
    results = lib.run_batch(table, [s for _, s in work])
    for j, (n, (dist, s), res) in enumerate(zip(lengths, work, results)):
        assert oracle.horner(res) == oracle.msm_checksum(k[:n], s), f"instance {j} (n={n}, {dist})"
    lib.bc.base_table_destroy(table)
    lib.bc.free(bd)


def test_batch_many_instances_edge_scalars(lib, oracle, table16):
    """The batch's limit of 256 instances: a 2^16-point instance beside 255
    small ones (so the look-back passes' interleaved ticket order ends with
    one segment alone), instances of all-zero scalars (no nonzero entry: every
    later-pass tile of the segment returns at once), all ones (one heavy
    bucket), r - 1, 2^253 and (r + 1) / 2."""
    import numpy as np
    import msm_helpers as H
    k, _, table = table16
    rng = np.random.Generator(np.random.PCG64(77))
    lengths = [1 << 16] + [int(x) for x in rng.integers(1, 3000, size=255)]
    fixed = {1: 0, 2: 1, 3: H.R - 1, 4: 1 << 253, 5: (H.R + 1) // 2}
    work = []
    for j, n in enumerate(lengths):
        if j in fixed:
            work.append(H.mont_scalar_array([fixed[j]] * n))
        elif j % 2:
            work.append(synth.skewed_scalars(900 + j, n))
        else:
            work.append(synth.uniform_scalars(900 + j, n))
    results = lib.run_batch(table, work)
    for j, (n, s, res) in enumerate(zip(lengths, work, results)):
        assert oracle.horner(res) == oracle.msm_checksum(k[:n], s), f"instance {j} (n={n})"
