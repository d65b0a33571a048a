"""Helpers shared by the tests: golden fixtures and MSM runs through the C ABI."""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
P = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
MONT = 1 << 256


def limbs(x: int, n: int = 8) -> np.ndarray:
    return np.array([(x >> (32 * i)) & 0xFFFFFFFF for i in range(n)], dtype=np.uint32)


def to_int(a) -> int:
    return sum(int(a[i]) << (32 * i) for i in range(len(a)))


def load_g_bases():
    pts = []
    for line in open(os.path.join(GOLDEN, "g_bases.txt")):
        if line.startswith("#"):
            continue
        x, y = line.split()
        pts.append((int(x, 16), int(y, 16)))
    return pts


def load_known_points():
    pts = []
    for line in open(os.path.join(GOLDEN, "known_points.txt")):
        if line.startswith("#"):
            continue
        x, y = line.split()
        pts.append((int(x, 16), int(y, 16)))
    return pts


def load_json(name):
    return json.load(open(os.path.join(GOLDEN, name)))


def mont_point_array(points) -> np.ndarray:
    out = np.zeros((len(points), 16), np.uint32)
    for i, (x, y) in enumerate(points):
        out[i, :8] = limbs(x * MONT % P)
        out[i, 8:] = limbs(y * MONT % P)
    return out


def mont_scalar_array(values) -> np.ndarray:
    return np.stack([limbs(v * MONT % R) for v in values]).astype(np.uint32) if len(values) else np.zeros((0, 8), np.uint32)


def expected_point(case):
    return (bool(case["infinity"]), int(case["x"], 16), int(case["y"], 16))


def table_workload(n: int, seed: int):
    """Reference-test style inputs (tests/msm_test.cu:17-25): bases drawn from the
    256-entry table (i+1)*G, uniform scalars.  Returns (bases_mont, scalars_mont, k_std)."""
    import synth
    g = np.random.Generator(np.random.PCG64(np.random.SeedSequence([seed, 99])))
    idx = g.integers(0, 256, n)
    table = mont_point_array(load_g_bases())
    bases = np.ascontiguousarray(table[idx])
    k = np.zeros((n, 8), np.uint32)
    k[:, 0] = (idx + 1).astype(np.uint32)
    scalars = synth.uniform_scalars(seed, n)
    return bases, scalars, k
