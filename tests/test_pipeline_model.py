"""Integer model of the GPU pipeline's decomposition (a point is its discrete
log mod r): signed digits of min(s, r - s), stable per-window sort, equal
ranges with head partial sums, warp-segmented head merging, grouped running sums and
the binary decomposition that places every partial sum at its bit of the
254-entry result.  Checks sum_i 2^i R_i == sum_i k_i s_i, and that no partial
sum lands above bit 253.  Mirrors era-bellman-cuda_b200/csrc/msm_kernels.cu."""
import random

import pytest

R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
ZERO_KEY = 0xFFFFFFFF  # sort key of a zero digit (|d| - 1 wrapped)


def key_slot(key, B):
    return (key + 1) & (B - 1)


MERGE_SMALL_LEVEL = 64  # the model's level size at which the merge takes 8 heads per warp (the kernels': 32 per SM)


def merge_heads_level(hb, hp, heads, buckets, per_warp=32):
    """One merge_heads_kernel launch (per_warp = 32, one head per lane) or
    merge_heads_group4_kernel launch (per_warp = 8, one head per group of
    four lanes): warp w takes heads [per_warp w, per_warp (w + 1)), a
    segmented Kogge-Stone inclusive scan leaves each segment's sum in its
    last slot; the segment holding slot 0 is a continuation when the head
    before the warp has its bucket (-> the warp's output head), every other
    segment is added into its bucket."""
    P = per_warp
    out = (heads + P - 1) // P
    hb2, hp2 = [None] * out, [0] * out
    updated = set()
    for w in range(out):
        b = [hb[P * w + l] if P * w + l < heads else None for l in range(P)]
        acc = [hp[P * w + l] if b[l] is not None else 0 for l in range(P)]
        d = 1
        while d < P:
            old = list(acc)  # every lane shuffles before any adds
            for l in range(P):
                if l >= d and b[l - d] == b[l] and b[l] is not None:
                    acc[l] = (old[l - d] + old[l]) % R
            d <<= 1
        joins = [l > 0 and b[l - 1] == b[l] for l in range(P)]
        before = hb[P * w - 1] if w > 0 else None
        continued = b[0] is not None and before == b[0]
        for l in range(P):
            if b[l] is None or (l < P - 1 and b[l + 1] == b[l]):
                continue
            first = max(f for f in range(l + 1) if not joins[f])
            if first == 0 and continued:
                hb2[w], hp2[w] = b[l], acc[l]
            else:
                assert b[l] not in updated, "two segments of one launch update one bucket"
                updated.add(b[l])
                buckets[b[l]] = (buckets[b[l]] + acc[l]) % R
    return hb2, hp2


def model_msm(scal, kl, c, T, log_m_max=3):
    n = len(scal)
    W = (254 + c - 1) // c
    log_b = c - 1
    B = 1 << log_b
    keys = [[0] * n for _ in range(W)]
    vals = [[None] * n for _ in range(W)]
    for i, s in enumerate(scal):
        neg = R - s
        flip = neg < s
        if flip:
            s = neg
        assert s < (1 << 253)
        carry = 0
        for w in range(W):
            raw = ((s >> (w * c)) & ((1 << c) - 1)) + carry
            negd = 0
            if raw > B:
                raw, negd, carry = (1 << c) - raw, 1, 1
            else:
                carry = 0
            keys[w][i], vals[w][i] = (raw - 1) & 0xFFFFFFFF, (i, negd ^ flip)
        assert carry == 0
    # the first sort pass drops zero digits; the nonzero entries of a window
    # end up sorted at the end of its segment (the prefix is never read)
    for w in range(W):
        order = sorted(range(n), key=lambda i: (keys[w][i] != ZERO_KEY, keys[w][i]))
        keys[w] = [keys[w][i] for i in order]
        vals[w] = [vals[w][i] for i in order]
    zeros = [sum(1 for k in keys[w] if k == ZERO_KEY) for w in range(W)]
    pre = [0]
    for w in range(W):
        pre.append(pre[-1] + n - zeros[w])
    M = pre[-1]

    def entry(v):
        w = next(x for x in range(W) if pre[x] <= v < pre[x + 1])
        return w, zeros[w] + v - pre[w]

    def point(w, idx):
        i, sg = vals[w][idx]
        return (-kl[i] if sg else kl[i]) % R

    buckets, hb, hp = {}, [None] * T, [0] * T
    active = min(M, T)
    for t in range(active):
        beg, end = M * t // active, M * (t + 1) // active
        assert beg < end
        w, idx = entry(beg)
        key = keys[w][idx]
        cont = idx > zeros[w] and keys[w][idx - 1] == key
        cur, acc, first = (w << log_b) | key_slot(key, B), point(w, idx), True
        for v in range(beg + 1, end):
            w, idx = entry(v)
            b = (w << log_b) | key_slot(keys[w][idx], B)
            if b != cur:
                if first and cont:
                    hb[t], hp[t] = cur, acc
                else:
                    assert cur not in buckets
                    buckets[cur] = acc
                first, cur, acc = False, b, point(w, idx)
            else:
                acc = (acc + point(w, idx)) % R
        if first and cont:
            hb[t], hp[t] = cur, acc
        else:
            assert cur not in buckets
            buckets[cur] = acc
    heads = T
    while heads > 1:
        # the heads of one bucket must be contiguous: one merge launch may not
        # update a bucket from two threads
        valid = [k for k in range(heads) if hb[k] is not None]
        for a, b in zip(valid, valid[1:]):
            if hb[a] == hb[b]:
                assert b == a + 1, "heads of one bucket are not contiguous"
        hb2, hp2 = merge_heads_level(hb, hp, heads, buckets, 8 if heads <= MERGE_SMALL_LEVEL else 32)
        out = len(hb2)
        hb, hp, heads = hb2, hp2, out
    log_m = min(log_m_max, log_b)
    log_g = log_b - log_m
    G, m = 1 << log_g, 1 << log_m
    res = [0] * 254
    for w in range(W):
        run, accs = [0] * G, [0] * G
        for g in range(G):
            r_, a_ = 0, 0
            for i in range(m - 1, 0, -1):
                r_ = (r_ + buckets.get((w << log_b) + g * m + i, 0)) % R
                a_ = (a_ + r_) % R
            if g > 0:
                r_ = (r_ + buckets.get((w << log_b) + g * m, 0)) % R
            run[g], accs[g] = r_, a_
        # reduce_level_kernel: at each level every live stream takes one
        # pairwise step and the tree's odd entries start a new stream, so all
        # streams shrink together to one sum each
        streams, t0 = [accs], run
        for level in range(log_g):
            assert all(len(st) == G >> level for st in streams)
            streams = [[(st[2 * i] + st[2 * i + 1]) % R for i in range(len(st) // 2)] for st in streams]
            streams.append(t0[1::2])
            t0 = [(t0[2 * i] + t0[2 * i + 1]) % R for i in range(len(t0) // 2)]
        assert all(len(st) == 1 for st in streams)
        sums = [st[0] for st in streams]
        for o in range(c):
            val = 0
            if o == 0:
                val = sums[0]
            elif o == c - 1:
                val = buckets.get(w << log_b, 0)
            elif log_m <= o < log_m + log_g:
                val = sums[o - log_m + 1]
            if c * w + o >= 254:
                assert val == 0
            else:
                res[c * w + o] = val
    return sum(res[i] * pow(2, i, R) for i in range(254)) % R


@pytest.mark.parametrize("trial", range(40))
def test_model_matches_sum(trial):
    rng = random.Random(trial)
    n = rng.choice([1, 2, 3, 5, 16, 33, 100, 257])
    c = rng.choice([2, 3, 4, 5, 6, 8, 10, 12, 16])
    T = rng.choice([1, 2, 3, 7, 16, 64, 200])
    mode = rng.choice(["uniform", "small", "skewed"])
    if mode == "uniform":
        scal = [rng.randrange(R) for _ in range(n)]
    elif mode == "small":
        scal = [rng.choice([0, 1, 2, R - 1, R - 2, rng.randrange(1 << 16)]) for _ in range(n)]
    else:
        scal = [rng.choice([0, 0, 1, 1, rng.randrange(1 << 16), rng.randrange(R)]) for _ in range(n)]
    kl = [rng.randrange(1, R) for _ in range(n)]
    assert model_msm(scal, kl, c, T) == sum(s * k for s, k in zip(scal, kl)) % R


def model_final_sum(values, threads=128, result_bits=254):
    """The index arithmetic of final_sum_kernel (msm_final.cu) with points as
    integers mod R (doubling = 2x, addition = x + y): level 0 per thread
    (R_2t + 2 R_2t+1), level 1 per even thread (partner doubled twice),
    levels 2..7 per group of four lanes, group g adding part[g 2^L + 2^(L-1)]
    doubled 2^L times into part[g 2^L].  Every partner index must stay in
    the block and be read before anyone writes it at that level."""
    part = [0] * threads
    for t in range(threads):
        if 2 * t + 1 < result_bits:
            part[t] = (values[2 * t] + 2 * values[2 * t + 1]) % R
    for t in range(0, threads, 2):
        part[t] = (part[t] + 4 * part[t + 1]) % R
    level = 2
    while (1 << level) <= threads:
        pairs = threads >> level
        targets, partners = set(), set()
        for group in range(threads // 4):
            if group < pairs:
                target, partner = group << level, (group << level) + (1 << (level - 1))
                assert partner < threads
                targets.add(target)
                partners.add(partner)
                part[target] = (part[target] + pow(2, 1 << level, R) * part[partner]) % R
        assert not targets & partners  # no group reads a slot another group writes
        level += 1
    return part[0]


@pytest.mark.parametrize("trial", range(6))
def test_final_sum_tree(trial):
    rng = random.Random(2000 + trial)
    values = [rng.randrange(R) if rng.random() < 0.8 else 0 for _ in range(254)]
    assert model_final_sum(values) == sum(v * pow(2, i, R) for i, v in enumerate(values)) % R


@pytest.mark.parametrize("n,c,T,mode", [(2000, 4, 1500, "one"), (700, 2, 3000, "uniform"), (1200, 3, 1100, "skewed"),
                                        (64, 2, 5000, "uniform")])
def test_model_many_heads(n, c, T, mode):
    """Many heads per bucket: a bucket's heads span several warps of the merge
    and several merge levels (all scalars 1 puts every entry in one bucket)."""
    rng = random.Random(n * 31 + T)
    if mode == "one":
        scal = [1] * n
    elif mode == "uniform":
        scal = [rng.randrange(R) for _ in range(n)]
    else:
        scal = [rng.choice([0, 1, 1, 2, rng.randrange(R)]) for _ in range(n)]
    kl = [rng.randrange(1, R) for _ in range(n)]
    assert model_msm(scal, kl, c, T) == sum(s * k for s, k in zip(scal, kl)) % R
