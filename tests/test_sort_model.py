"""Integer model of the plain pipeline's radix sort (era-bellman-cuda_b200/csrc/
msm_kernels.cu: digits_histogram_kernel, sort_scan_kernel,
sort_scatter_first_kernel, lookback_stable_kernel; tile code in
msm_device.cuh): per-pass digit counts per tile from the digit kernel (the
first pass's per tile, later passes' summed into digit totals), one scan
giving the first pass's tile offsets and totals, the first pass (drops zero
digits, any order among equal digits), then one kernel per later 8-bit pass
in which each tile finds, digit by digit, the positions of its runs by
decoupled look-back over packed words (status in the top two bits, count
below): it publishes its count as an aggregate, reads the earlier tiles' words
of its digit eight at a time, newest first, adding counts until an inclusive
one (waiting while a word is still empty), and publishes its inclusive count.
A later-pass tile whose entries span at most eight values of the lower key
bits ranks equal digits in any order within each value (the kernels' atomic
ranking), others stably.  The model gives the later passes a tile size of
their own (the kernels may use one).  Tickets go to windows in turn and tiles and digits finish in a
random order.  Checked: the window segments come out grouped exactly by key
(a stable sort of the first pass's output), at [w S + zeros_w, w S + n)."""
import random

import pytest

RADIX_BITS, RADIX, TILE = 8, 256, 64  # the model's tiles are small so that windows span many tiles
LOOKBACK_TILE = 96  # the later passes' tiles
AGG, INCL, COUNT = 1 << 30, 2 << 30, (1 << 30) - 1  # look-back word: status bits over the count
BATCH = 8
SEGMENTS = 8  # lower-bit values a later-pass tile may span and still rank with atomics
ZERO_KEY = 0xFFFFFFFF


def digit(key, shift):
    return (key >> shift) & (RADIX - 1)


def model_sort(keys, vals, n, windows, stride, passes, rng):
    tiles = (n + TILE - 1) // TILE
    # digit kernel: per (pass, window, tile) counts of the nonzero keys; zeros per window
    zeros = [0] * windows
    hist = [[[[0] * RADIX for _ in range(tiles)] for _ in range(windows)] for _ in range(passes)]
    for w in range(windows):
        for i in range(n):
            k = keys[w * stride + i]
            if k == ZERO_KEY:
                zeros[w] += 1
                continue
            for p in range(passes):
                hist[p][w][i // TILE][digit(k, p * RADIX_BITS)] += 1
    # totals kernel; pass 0's counts are published aggregates, later passes' are cleared
    totals = [[[sum(hist[p][w][t][d] for t in range(tiles)) for d in range(RADIX)] for w in range(windows)] for p in range(passes)]
    # the scan: pass 0's exclusive prefix over tiles; later passes use look-back
    scan0 = [[[sum(hist[0][w][u][d] for u in range(t)) for d in range(RADIX)] for t in range(tiles)] for w in range(windows)]
    cur_k, cur_v = list(keys), list(vals)
    for p in range(passes):
        shift = p * RADIX_BITS
        size = TILE if p == 0 else LOOKBACK_TILE
        ptiles = (n + size - 1) // size
        words = [[[0] * RADIX for _ in range(ptiles)] for _ in range(windows)]  # cleared before the pass
        out_k, out_v = [None] * len(keys), [None] * len(vals)
        # every (window, tile) is one block; tickets go to windows in turn
        # (ticket = tile * windows + w) and blocks progress in a random order;
        # a block's look-back only ever waits for earlier tiles of its window,
        # and each digit's look-back goes on by itself
        pending = [(w, t) for t in range(ptiles) for w in range(windows)]
        rng.shuffle(pending)
        state = {}
        while pending:
            progressed = False
            for item in list(pending):
                w, t = item
                live = n if p == 0 else n - zeros[w]
                base = t * size
                if base >= live:
                    pending.remove(item)
                    progressed = True
                    continue
                seg_in = w * stride if p == 0 else w * stride + zeros[w]
                seg_out = w * stride + zeros[w]
                items = [(cur_k[seg_in + base + i], cur_v[seg_in + base + i]) for i in range(min(size, live - base))]
                if p == 0:
                    items = [it for it in items if it[0] != ZERO_KEY]
                    rng.shuffle(items)  # the first pass ranks equal digits in any order
                else:
                    # a tile whose lower bits span few values ranks with atomics per
                    # (value, digit): runs ordered by the lower bits, equal keys in any order
                    lower = (1 << shift) - 1
                    if ((items[-1][0] & lower) - (items[0][0] & lower)) < SEGMENTS:
                        rng.shuffle(items)
                        items.sort(key=lambda it: it[0] & lower)
                count = [0] * RADIX
                for k, _ in items:
                    count[digit(k, shift)] += 1
                if p == 0:
                    prefix = scan0[w][t]
                else:
                    if item not in state:  # ranked: every digit publishes its count
                        for d in range(RADIX):
                            words[w][t][d] = (INCL if t == 0 else AGG) | count[d]
                        state[item] = {"prefix": [0] * RADIX, "next": [t - 1] * RADIX, "done": [t == 0] * RADIX}
                        progressed = True
                    st = state[item]
                    for d in rng.sample(range(RADIX), RADIX):  # digits in any order, one or two steps each
                        for _ in range(rng.randint(1, 2)):
                            if st["done"][d]:
                                break
                            j = st["next"][d]
                            batch = [words[w][j - k][d] if j - k >= 0 else INCL for k in range(BATCH)]
                            for v in batch:
                                if v < AGG:
                                    break  # empty: that tile has not ranked yet, poll again
                                progressed = True
                                st["prefix"][d] += v & COUNT
                                st["next"][d] -= 1
                                if v >= INCL:
                                    st["done"][d] = True
                                    words[w][t][d] = INCL | (st["prefix"][d] + count[d])
                                    break
                    if not all(st["done"]):
                        continue
                    prefix = st["prefix"]
                dbase = [0] * RADIX
                for d in range(1, RADIX):
                    dbase[d] = dbase[d - 1] + totals[p][w][d - 1]
                rank = [0] * RADIX
                for k, v in items:
                    d = digit(k, shift)
                    pos = seg_out + dbase[d] + prefix[d] + rank[d]
                    rank[d] += 1
                    assert out_k[pos] is None
                    out_k[pos], out_v[pos] = k, v
                pending.remove(item)
                progressed = True
            assert progressed, "look-back deadlock"
        cur_k, cur_v = out_k, out_v
    return cur_k, cur_v, zeros


@pytest.mark.parametrize("trial", range(10))
def test_onesweep_model_sorts_each_window(trial):
    rng = random.Random(1000 + trial)
    key_bits = rng.choice([7, 8, 12, 16]) if trial < 6 else rng.choice([12, 16, 20])
    passes = (key_bits + RADIX_BITS - 1) // RADIX_BITS
    windows = rng.randint(1, 4)
    n = rng.randint(1, 700)
    stride = (n + 31) // 32 * 32
    keys, vals = [ZERO_KEY] * (windows * stride), [0] * (windows * stride)
    zero_share = rng.choice([0.0, 0.3, 0.9, 1.0])
    for w in range(windows):
        hot = rng.randrange(1 << key_bits)
        for i in range(n):
            r = rng.random()
            k = ZERO_KEY if r < zero_share else (hot if r < zero_share + 0.2 else rng.randrange(1 << key_bits))
            if trial >= 6 and k != ZERO_KEY:  # few distinct low bytes: later-pass tiles span few values
                k = (k & ~0xFF) | rng.choice([3, 4, 9, 30])
            keys[w * stride + i] = k
            vals[w * stride + i] = i | (rng.randrange(2) << 31)
    out_k, out_v, zeros = model_sort(keys, vals, n, windows, stride, passes, rng)
    for w in range(windows):
        nonzero = [(keys[w * stride + i], vals[w * stride + i]) for i in range(n) if keys[w * stride + i] != ZERO_KEY]
        assert zeros[w] == n - len(nonzero)
        got = list(zip(out_k[w * stride + zeros[w]: w * stride + n], out_v[w * stride + zeros[w]: w * stride + n]))
        # grouped exactly by key; after a stable later pass, the order of
        # equal full keys is whatever the first pass left (any order)
        assert [k for k, _ in got] == sorted(k for k, _ in nonzero)
        assert sorted(got) == sorted(nonzero)


def batch_ticket_order(tiles):
    """The batched look-back passes' ticket order (msm_batch.cu,
    descriptor_image): instance k's local tile j is global tile base[k] + j,
    and every instance's local tile j comes before any instance's tile j + 1."""
    base, acc = [], 0
    for t in tiles:
        base.append(acc)
        acc += t
    order = []
    for j in range(max(tiles, default=0)):
        for k, t in enumerate(tiles):
            if j < t:
                order.append(base[k] + j)
    return order, base


@pytest.mark.parametrize("tiles", [[1], [5, 1, 3], [2000, 7, 0 + 1, 1300, 64], [3] * 64, [13312, 11000, 40, 1]])
def test_batch_ticket_order(tiles):
    """Every tile gets exactly one ticket, and a tile's predecessors in its
    own segment (the only tiles its look-back waits for) hold earlier tickets,
    so they are resident or finished whenever it waits."""
    order, base = batch_ticket_order(tiles)
    assert sorted(order) == list(range(sum(tiles)))
    ticket = {t: q for q, t in enumerate(order)}
    for k, n in enumerate(tiles):
        for j in range(1, n):
            assert ticket[base[k] + j - 1] < ticket[base[k] + j]
