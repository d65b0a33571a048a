"""The product field and curve code (era-bellman-cuda_b200/csrc/bn254_*.cuh),
compiled for the host: the exact carry-chain instruction sequences run against
an emulated carry flag and are checked against big-integer arithmetic and the
oracle.  Covers the lazy-reduction bounds the way the reference's montmul test
does with its corner inputs (p-1, 0, 2p-1; tests/montmul_test.cu:36-74)."""
import ctypes

import numpy as np
import pytest

import msm_helpers as H

P, R = H.P, H.R
RINV = pow(2, -256, P)
EDGE = [0, 1, 2, P - 1, P, P + 1, 2 * P - 2, 2 * P - 1, P // 2, 0xFFFFFFFF, 1 << 32, 1 << 224, (1 << 254) - 1]


def arr(values, n=8):
    return np.concatenate([H.limbs(v, n) for v in values]).astype(np.uint32) if values else np.zeros(0, np.uint32)


def ints(a, n=8):
    return [H.to_int(a[i * n:(i + 1) * n]) for i in range(len(a) // n)]


def ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


@pytest.fixture(scope="module")
def pairs():
    rng = np.random.Generator(np.random.PCG64(3))
    xs = [int.from_bytes(rng.bytes(32), "little") % (2 * P) for _ in range(1500)]
    ys = [int.from_bytes(rng.bytes(32), "little") % (2 * P) for _ in range(1500)]
    xs += [e for e in EDGE for _ in EDGE]
    ys += [e for _ in EDGE for e in EDGE]
    return xs, ys


OPS = {
    0: (lambda x, y: x * y * RINV, 2 * P),  # mul, lazy output
    1: (lambda x, y: x * x * RINV, 2 * P),  # sqr
    2: (lambda x, y: x + y, 2 * P),
    3: (lambda x, y: x - y, 2 * P),
    4: (lambda x, y: -x, 2 * P),
    5: (lambda x, y: x, P),                 # reduce_full
    6: (lambda x, y: x * RINV, P),          # from_mont
    7: (lambda x, y: x * (1 << 256), P),    # to_mont
    9: (lambda x, y: 2 * x, 2 * P),
}


def test_neg_nonzero(field_check, pairs):
    xs = [x for x in pairs[0] if 0 < x < 2 * P]
    a = arr(xs)
    out = np.zeros_like(a)
    field_check.fc_fq_op(10, ptr(a), ptr(a), ptr(out), len(xs))
    for x, r in zip(xs, ints(out)):
        assert 0 < r < 2 * P and (r + x) % P == 0


@pytest.mark.parametrize("op", sorted(OPS))
def test_fq_ops(field_check, pairs, op):
    xs, ys = pairs
    fn, bound = OPS[op]
    a, b = arr(xs), arr(ys)
    out = np.zeros_like(a)
    field_check.fc_fq_op(op, ptr(a), ptr(b), ptr(out), len(xs))
    for x, y, r in zip(xs, ys, ints(out)):
        assert r < bound and r % P == fn(x, y) % P, (op, hex(x), hex(y), hex(r))


def test_fq_inverse(field_check):
    rng = np.random.Generator(np.random.PCG64(4))
    xs = [int.from_bytes(rng.bytes(32), "little") % P for _ in range(8)] + [1, P - 1]
    a = arr(xs)
    out = np.zeros_like(a)
    field_check.fc_fq_op(8, ptr(a), ptr(a), ptr(out), len(xs))
    for x, r in zip(xs, ints(out)):
        assert (r * x * RINV) % P == (1 << 256) % P


def test_fq_inverse_binary(field_check):
    """Binary extended-Euclid inverse of canonical standard-form values
    (the on-device final reduction's inversion): a * a^-1 = 1 mod p, 0 -> 0."""
    rng = np.random.Generator(np.random.PCG64(12))
    xs = [int.from_bytes(rng.bytes(32), "little") % P for _ in range(2000)]
    xs += [0, 1, 2, 3, P - 1, P - 2, P // 2, (P + 1) // 2, 1 << 128, (1 << 253) - 1, 0xFFFFFFFF, 1 << 32]
    a = arr(xs)
    out = np.zeros_like(a)
    field_check.fc_fq_op(11, ptr(a), ptr(a), ptr(out), len(xs))
    for x, r in zip(xs, ints(out)):
        assert r == (pow(x, -1, P) if x else 0), hex(x)


def test_fq_mul_sub_mul(field_check, pairs):
    xs, ys = pairs
    rng = np.random.Generator(np.random.PCG64(5))
    cs = [int.from_bytes(rng.bytes(32), "little") % (2 * P) for _ in xs]
    ds = [int.from_bytes(rng.bytes(32), "little") % (2 * P) for _ in xs]
    a, b, c, d = arr(xs), arr(ys), arr(cs), arr(ds)
    out = np.zeros_like(a)
    field_check.fc_fq_mul_sub_mul(ptr(a), ptr(b), ptr(c), ptr(d), ptr(out), len(xs))
    for x, y, cc, dd, r in zip(xs, ys, cs, ds, ints(out)):
        assert r < 2 * P and r % P == (x * y - cc * dd) * RINV % P


def test_fr_from_mont_any_input(field_check):
    rng = np.random.Generator(np.random.PCG64(6))
    xs = [int.from_bytes(rng.bytes(32), "little") for _ in range(1000)] + [0, 1, R - 1, R, R + 1, (1 << 256) - 1]
    a = arr(xs)
    out = np.zeros_like(a)
    field_check.fc_fr_op(6, ptr(a), ptr(a), ptr(out), len(xs))
    for x, r in zip(xs, ints(out)):
        assert r == x * pow(2, -256, R) % R


def test_fq_is_zero(field_check):
    for v, z in [(0, 1), (P, 1), (1, 0), (P - 1, 0), (P + 1, 0), (2 * P - 1, 0)]:
        assert field_check.fc_fq_is_zero(ptr(H.limbs(v))) == z


# ---- curve ---------------------------------------------------------------
def xyzz_to_affine(p):
    x, y, zz, zzz = (H.to_int(p[i * 8:(i + 1) * 8]) % P for i in range(4))
    if zz == 0:
        return (True, 0, 0)
    inv_zz = pow(zz * RINV % P, -1, P)  # coordinates are Montgomery form
    inv_zzz = pow(zzz * RINV % P, -1, P)
    return (False, (x * RINV) * inv_zz % P, (y * RINV) * inv_zzz % P)


def affine_mont(pt):
    return H.mont_point_array([pt])[0]


def test_curve_identities(field_check, oracle):
    """x + 0 = x, x + 1 = next, x + x = 2x, x + (-x) = 0 (reference tests/ec_test.cu identities)."""
    table = H.load_g_bases()
    f = field_check
    out = np.zeros(32, np.uint32)
    inf = np.zeros(32, np.uint32)
    f.fc_infinity(ptr(inf))
    for i in (0, 1, 5, 40, 77, 84):
        a = affine_mont(table[i])
        f.fc_add_affine(ptr(inf), ptr(a), ptr(out))  # 0 + x
        assert xyzz_to_affine(out) == (False, *table[i])
        p = np.zeros(32, np.uint32)
        f.fc_from_affine(ptr(a), ptr(p))
        g = affine_mont(table[0])
        f.fc_add_affine(ptr(p), ptr(g), ptr(out))  # x + G = (i+2) G
        assert xyzz_to_affine(out) == (False, *table[i + 1])
        f.fc_add_affine(ptr(p), ptr(a), ptr(out))  # x + x via the madd doubling branch
        assert xyzz_to_affine(out) == (False, *table[2 * i + 1])
        neg = affine_mont((table[i][0], P - table[i][1]))
        f.fc_add_affine(ptr(p), ptr(neg), ptr(out))  # x - x
        assert xyzz_to_affine(out)[0]
        assert f.fc_add_affine_finite(ptr(p), ptr(neg), ptr(out)) == 1  # flagged, not computed
        assert f.fc_add_affine_finite(ptr(p), ptr(g), ptr(out)) == 0
        assert xyzz_to_affine(out) == (False, *table[i + 1])
        assert f.fc_add_affine_finite(ptr(p), ptr(a), ptr(out)) == 0  # doubling branch
        assert xyzz_to_affine(out) == (False, *table[2 * i + 1])
        f.fc_dbl(ptr(p), ptr(out))
        assert xyzz_to_affine(out) == (False, *table[2 * i + 1])
        q = out.copy()
        f.fc_add(ptr(p), ptr(q), ptr(out))  # x + 2x = 3x (XYZZ + XYZZ)
        assert xyzz_to_affine(out) == (False, *table[3 * i + 2])
        f.fc_add(ptr(p), ptr(p), ptr(out))  # doubling branch of add
        assert xyzz_to_affine(out) == (False, *table[2 * i + 1])
        jac = np.zeros(24, np.uint32)
        f.fc_to_jacobian(ptr(q), ptr(jac))
        assert oracle.normalize(jac) == (False, *table[2 * i + 1])


def full_words(rng, count):
    """Uniform 256-bit words and the carry corner cases of the 128-bit halves."""
    vals = [int.from_bytes(rng.bytes(32), "little") for _ in range(count)]
    corners = [0, 1, (1 << 256) - 1, (1 << 128) - 1, 1 << 128, ((1 << 128) - 1) << 128, (1 << 255) | 1, 2 * P - 1, P]
    return vals + corners


def test_wide_products_exact(field_check):
    """The schoolbook 512-bit product against Python integers, on arbitrary
    256-bit operands and the carry corner cases of both halves."""
    kind = 0
    rng = np.random.Generator(np.random.PCG64(11 + kind))
    xs = full_words(rng, 3000)
    ys = list(reversed(full_words(rng, 3000)))
    pairs_ = [(x, y) for x in xs[-9:] for y in ys[:9]] + list(zip(xs, ys))
    a, b = arr([p[0] for p in pairs_]), arr([p[1] for p in pairs_])
    out = np.zeros(16 * len(pairs_), np.uint32)
    field_check.fc_fq_wide(kind, ptr(a), ptr(b), ptr(out), len(pairs_))
    for (x, y), got in zip(pairs_, ints(out, 16)):
        assert got == x * y


def test_square_matches_cios(field_check, pairs):
    """The squaring (off-diagonal products once + REDC) and the CIOS product
    of a value with itself give the same lazy residue class and range."""
    xs, _ = pairs
    a = arr(xs)
    out_c = np.zeros_like(a)
    out_s = np.zeros_like(a)
    field_check.fc_fq_wide(3, ptr(a), ptr(a), ptr(out_c), len(xs))
    field_check.fc_fq_wide(5, ptr(a), ptr(a), ptr(out_s), len(xs))
    for x, c_, s_ in zip(xs, ints(out_c), ints(out_s)):
        assert c_ < 2 * P and s_ < 2 * P
        assert c_ % P == s_ % P == x * x * RINV % P


def test_jacobian_round_trip_and_standard_affine(field_check, oracle):
    """from_jacobian / to_affine_standard (the final-sum kernel's input and
    output conversions): Jacobian points with random Z, infinity with Z = 0."""
    table = H.load_g_bases()
    f = field_check
    rng = np.random.Generator(np.random.PCG64(13))
    for i in (0, 3, 17, 100, 255):
        x, y = table[i]
        z = int.from_bytes(rng.bytes(32), "little") % P or 1
        jac = arr([x * z * z % P * (1 << 256) % P, y * z ** 3 % P * (1 << 256) % P, z * (1 << 256) % P])
        p = np.zeros(32, np.uint32)
        f.fc_from_jacobian(ptr(jac), ptr(p))
        assert xyzz_to_affine(p) == (False, x, y)
        out = np.zeros(16, np.uint32)
        assert f.fc_to_affine_standard(ptr(p), ptr(out)) == 0
        assert (H.to_int(out[:8]), H.to_int(out[8:])) == (x, y)
    inf_jac = arr([0, (1 << 256) % P, 0])  # the reference encoding (0, 1, 0)
    p = np.zeros(32, np.uint32)
    f.fc_from_jacobian(ptr(inf_jac), ptr(p))
    out = np.ones(16, np.uint32)
    assert f.fc_to_affine_standard(ptr(p), ptr(out)) == 1
    assert not out.any()
