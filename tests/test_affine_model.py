"""Integer model of the affine pairing levels (era-bellman-cuda_b200/csrc/
msm_affine.cuh: affine_forward, affine_apply; msm_kernels.cu:
affine_invert_kernel; the list bound of msm_host.cu: level_output_bound).

Points are elements v of the additive group Z_q (q prime), with "x" the class
{v, -v} (so equal x means equal or opposite points, as on the curve) and a
marker for infinity.  One level runs exactly as the kernels arrange it: warp g
owns pairs [P g / W, P (g + 1) / W), lane l the pairs first + 32 k + l; the
forward pass walks each lane's pairs from the last round to the first storing
the prefix product of the slope denominators (random nonzero residues mod a
second prime stand in for x1 - x0 and 2 y0), the warps' and the block's
products of the other chains are formed as the kernels form them, and the
apply pass walks the rounds forward computing each inverse from the stored
prefix.  Checked, for random sorted bucket lists and every kind of pair:
every addition's inverse times its denominator is 1, the output list keeps
the input order (sorted by bucket, each bucket's sum unchanged), and the
output count never exceeds the bound the host sizes the lists with."""
import random

import pytest

Q = 1_000_003          # the model group Z_q
M = (1 << 61) - 1      # the model field of the slope denominators
MARKER = None

LONE, SPLIT, KEEP0, KEEP1, INF, ADD, DOUBLE = range(7)


def cls(v):
    return min(v, (Q - v) % Q)


def classify(lst, i):
    """pair_kind of pair i (classify_pair)."""
    j = 2 * i
    if j + 1 >= len(lst):
        return LONE
    (b0, v0), (b1, v1) = lst[j], lst[j + 1]
    if b0 != b1:
        return SPLIT
    m0, m1 = v0 is MARKER, v1 is MARKER
    if m0 or m1:
        return INF if m0 and m1 else KEEP1 if m0 else KEEP0
    if cls(v0) != cls(v1):
        return ADD
    if v0 == v1 and v0 != 0:
        return DOUBLE
    return INF


def outputs(kind):
    return 2 if kind == SPLIT else 1


def warp_products(vals):
    """others[l] = product of the other lanes' values, total (warp_products)."""
    n = len(vals)
    pre, suf = list(vals), list(vals)
    d = 1
    while d < n:
        pre = [pre[l] * pre[l - d] % M if l >= d else pre[l] for l in range(n)]
        suf = [suf[l] * suf[l + d] % M if l + d < n else suf[l] for l in range(n)]
        d <<= 1
    ep = [1] + pre[:-1]
    es = suf[1:] + [1]
    return [ep[l] * es[l] % M for l in range(n)], pre[-1]


def run_level(lst, warps, rng):
    m = len(lst)
    pairs = (m + 1) // 2
    denom = {}  # pair -> its slope denominator (nonzero)
    pre = {}
    lane_acc, warp_outputs = {}, []
    # forward
    for g in range(warps):
        beg, end = pairs * g // warps, pairs * (g + 1) // warps
        rounds = (end - beg + 31) // 32
        accs, outs = [], 0
        for lane in range(32):
            acc = 1
            for k in reversed(range(rounds)):
                i = beg + 32 * k + lane
                if i < end:
                    kind = classify(lst, i)
                    outs += outputs(kind)
                    if kind >= ADD:
                        d = denom.setdefault(i, rng.randrange(1, M))
                        pre[i] = acc
                        acc = acc * d % M
            accs.append(acc)
        others, total = warp_products(accs)
        lane_acc[g] = (others, total)
        warp_outputs.append(outs)
    # invert: the inverse of every warp total and the warps' output offsets
    # (one thread per warp here: the block arrangement is a product of the same factors)
    winv = [pow(lane_acc[g][1], M - 2, M) for g in range(warps)]
    wbase, acc = [], 0
    for c in warp_outputs:
        wbase.append(acc)
        acc += c
    count = acc
    # apply
    out = [None] * count
    for g in range(warps):
        beg, end = pairs * g // warps, pairs * (g + 1) // warps
        rounds = (end - beg + 31) // 32
        others, _ = lane_acc[g]
        inv = [winv[g] * others[lane] % M for lane in range(32)]
        pos = wbase[g]
        for k in range(rounds):
            n_out = []
            kinds = []
            for lane in range(32):
                i = beg + 32 * k + lane
                kind = classify(lst, i) if i < end else None
                kinds.append(kind)
                n_out.append(0 if kind is None else outputs(kind))
            for lane in range(32):
                kind = kinds[lane]
                at = pos + sum(n_out[:lane])  # popc of the lower lanes' ballots
                if kind is None:
                    continue
                i = beg + 32 * k + lane
                (b0, v0) = lst[2 * i]
                if kind >= ADD:
                    dinv = inv[lane] * pre[i] % M
                    assert dinv * denom[i] % M == 1
                    inv[lane] = inv[lane] * denom[i] % M
                    s = (v0 + lst[2 * i + 1][1]) % Q
                    out[at] = (b0, MARKER if s == 0 else s)
                elif kind == SPLIT:
                    out[at], out[at + 1] = lst[2 * i], lst[2 * i + 1]
                elif kind == KEEP1:
                    out[at] = lst[2 * i + 1]
                elif kind == INF:
                    out[at] = (b0, MARKER)
                else:
                    out[at] = lst[2 * i]
            pos += sum(n_out)
        assert pos == wbase[g] + warp_outputs[g]
    return out


def bound(m, slots):
    return min(m, (m + 1) // 2 + slots)


def bucket_sums(lst):
    sums = {}
    for b, v in lst:
        sums[b] = (sums.get(b, 0) + (0 if v is MARKER else v)) % Q
    return sums


def runs_contiguous(lst):
    seen, prev = set(), None
    for b, _ in lst:
        if b != prev:
            if b in seen:
                return False
            seen.add(b)
            prev = b
    return True


def run_order(lst):
    order = []
    for b, _ in lst:
        if not order or order[-1] != b:
            order.append(b)
    return order


def random_list(rng, length, slots, style):
    """A bucket-sorted list in the window order of the pipeline (slot 0 last)."""
    bucket_of = [rng.randrange(slots) for _ in range(length)]
    order = sorted(range(length), key=lambda i: ((bucket_of[i] - 1) % slots, i))
    lst = []
    base = [rng.randrange(1, Q) for _ in range(8)]
    for i in order:
        if style == "uniform":
            v = rng.randrange(1, Q)
        elif style == "repeats":  # few distinct points: doublings and cancellations
            v = rng.choice(base + [Q - x for x in base])
        else:  # markers already present (later levels)
            v = MARKER if rng.random() < 0.2 else rng.choice(base + [Q - x for x in base])
        lst.append((bucket_of[i], v))
    return lst


@pytest.mark.parametrize("style", ["uniform", "repeats", "markers"])
@pytest.mark.parametrize("length,slots,warps", [(0, 4, 1), (1, 4, 1), (2, 1, 1), (3, 2, 2), (37, 3, 1), (300, 5, 3), (2000, 40, 7),
                                                (2000, 3000, 4), (5000, 1, 9)])
def test_levels_keep_sums_and_order(style, length, slots, warps):
    rng = random.Random(length * 7919 + slots * 31 + warps + len(style))
    lst = random_list(rng, length, slots, style)
    want = bucket_sums(lst)
    cap = length
    for level in range(4):
        out = run_level(lst, warps, rng)
        cap = bound(cap, slots)
        assert len(out) <= bound(len(lst), slots) <= cap
        assert runs_contiguous(out)
        assert run_order(out) == run_order(lst)  # the input order of the buckets, none lost
        assert bucket_sums(out) == want
        lst = out
    # each full level at least halves every run of one bucket (rounded up)
    if style == "uniform" and length >= 2000 and slots <= 40:
        assert len(lst) <= length // 8 + 2 * 4 * slots


def test_bound_is_tight_for_alternating_buckets():
    # every pair split: outputs = elements, the min() side of the bound
    lst = [(i % 2, i + 1) for i in range(64)]
    lst.sort(key=lambda e: (e[0] - 1) % 2)
    rng = random.Random(1)
    out = run_level(lst, 2, rng)
    assert len(out) <= bound(len(lst), 2)
    alt = [(i, i + 1) for i in range(64)]  # 64 buckets of one element each
    out = run_level(alt, 2, rng)
    assert len(out) == 64 == bound(64, 64)
