"""Seeded synthetic MSM workloads (the shapes of the reference's benchmark configs).

Generator: numpy's PCG64 bit generator seeded through SeedSequence([seed, stream])
(both documented as stable across numpy versions); only raw 64-bit outputs are
used.  Stream 0 = scalars, 1 = base multipliers k, 2 = category shuffle.

A field element is 8 x u32 little-endian limbs (uint32 array of shape (n, 8)).
Scalars are produced directly in Montgomery form, which is what
msm_execute_async takes: for uniform scalars a uniform Montgomery
representative is a uniform scalar (x -> x * 2^256 mod r is a bijection);
special values (0, 1, small integers) are mapped through their exact
Montgomery images.
"""
from __future__ import annotations

import numpy as np

P = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
MONT_R = (1 << 256) % R

_R_WORDS = np.array([(R >> (64 * i)) & ((1 << 64) - 1) for i in range(4)], dtype=np.uint64)


def _bitgen(seed: int, stream: int) -> np.random.PCG64:
    return np.random.PCG64(np.random.SeedSequence([int(seed), int(stream)]))


def _less_than_r(w: np.ndarray) -> np.ndarray:
    """w: (m, 4) uint64 little-endian words -> bool mask of w < r."""
    lt = np.zeros(len(w), dtype=bool)
    eq = np.ones(len(w), dtype=bool)
    for i in (3, 2, 1, 0):
        lt |= eq & (w[:, i] < _R_WORDS[i])
        eq &= w[:, i] == _R_WORDS[i]
    return lt


def uniform_below_r(seed: int, stream: int, n: int, nonzero: bool = False) -> np.ndarray:
    """n values uniform in [0, r) (or [1, r)) by rejection on 254-bit draws; (n, 8) uint32."""
    g = _bitgen(seed, stream)
    out = np.empty((0, 4), dtype=np.uint64)
    while len(out) < n:
        need = n - len(out)
        draw = g.random_raw(4 * (need + need // 3 + 16)).astype(np.uint64).reshape(-1, 4)
        draw[:, 3] &= np.uint64((1 << 62) - 1)
        ok = _less_than_r(draw)
        if nonzero:
            ok &= (draw != 0).any(axis=1)
        out = np.concatenate([out, draw[ok]])
    return np.ascontiguousarray(out[:n]).view(np.uint32).reshape(n, 8)


def int_to_limbs(x: int) -> np.ndarray:
    return np.array([(x >> (32 * i)) & 0xFFFFFFFF for i in range(8)], dtype=np.uint32)


def limbs_to_int(a) -> int:
    return sum(int(a[i]) << (32 * i) for i in range(8))


def to_mont_small(values: np.ndarray) -> np.ndarray:
    """Montgomery images v * 2^256 mod r of small non-negative integers (< 2^16 distinct table)."""
    values = np.asarray(values, dtype=np.int64)
    uniq, inv = np.unique(values, return_inverse=True)
    table = np.stack([int_to_limbs((int(v) * MONT_R) % R) for v in uniq]) if len(uniq) else np.zeros((0, 8), np.uint32)
    return np.ascontiguousarray(table[inv].reshape(len(values), 8))


def uniform_scalars(seed: int, n: int) -> np.ndarray:
    """Uniform scalars in [0, r), Montgomery form (configs 0, 1)."""
    return uniform_below_r(seed, 0, n)


def skewed_scalars(seed: int, n: int) -> np.ndarray:
    """Witness-like mix (config 2): 40% zero, 20% one, 20% uniform in [0, 2^16),
    20% uniform in [0, r), shuffled.  Montgomery form."""
    n0 = (4 * n) // 10
    n1 = (2 * n) // 10
    n2 = (2 * n) // 10
    n3 = n - n0 - n1 - n2
    g = _bitgen(seed, 0)
    small = (g.random_raw(max(n2, 1)).astype(np.uint64) & np.uint64(0xFFFF)).astype(np.int64)[:n2]
    out = np.empty((n, 8), dtype=np.uint32)
    cat = np.concatenate([np.zeros(n0, np.int8), np.ones(n1, np.int8), np.full(n2, 2, np.int8), np.full(n3, 3, np.int8)])
    order = np.argsort(_bitgen(seed, 2).random_raw(n).astype(np.uint64), kind="stable")
    cat = cat[order]
    out[cat == 0] = 0
    out[cat == 1] = int_to_limbs(MONT_R)
    idx2 = np.nonzero(cat == 2)[0]
    out[idx2] = to_mont_small(small)
    idx3 = np.nonzero(cat == 3)[0]
    out[idx3] = uniform_below_r(seed, 3, len(idx3))
    return out


def base_multipliers(seed: int, n: int) -> np.ndarray:
    """k_i uniform in [1, r), standard form: base i is k_i * G."""
    return uniform_below_r(seed, 1, n, nonzero=True)


def workload(name: str, n: int, seed: int):
    """(scalars_mont, k_std) for a named scalar distribution."""
    if name == "uniform":
        s = uniform_scalars(seed, n)
    elif name == "skewed":
        s = skewed_scalars(seed, n)
    else:
        raise ValueError(name)
    return s, base_multipliers(seed, n)


def batch_lengths(seed: int, instances: int, lo_log: int = 10, hi_log: int = 22) -> np.ndarray:
    """Instance lengths log-uniform in [2^lo_log, 2^hi_log], rounded to integers
    (config 3: 64 instances in [2^10, 2^22], seed 3).  Stream 4."""
    u = (_bitgen(seed, 4).random_raw(instances).astype(np.uint64) >> np.uint64(11)).astype(np.float64) / float(1 << 53)
    return np.rint(np.exp2(lo_log + (hi_log - lo_log) * u)).astype(np.int64)


def batch_workload(seed: int, lengths) -> list:
    """Per instance k: (distribution, Montgomery scalars); even k uniform, odd k
    skewed (the config-2 mix), instance k drawn from seed * 1000 + k.  All
    instances use prefixes of one base table (base_multipliers of the table)."""
    out = []
    for k, n in enumerate(lengths):
        dist = "uniform" if k % 2 == 0 else "skewed"
        sub = seed * 1000 + k
        out.append((dist, uniform_scalars(sub, int(n)) if dist == "uniform" else skewed_scalars(sub, int(n))))
    return out
