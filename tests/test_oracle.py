"""Pinning the CPU oracle: golden vectors of the reference's own tests, MSM
fixtures computed by the reference's host code, and (when the reference host
build is present) random cross-checks against that code."""
import ctypes
import os

import numpy as np
import pytest

import msm_helpers as H
import synth

P, R = H.P, H.R


def test_g_bases_are_multiples_of_g(oracle):
    """tests/msm_bases.cuh: g_bases[i] = (i+1) * G."""
    table = H.load_g_bases()
    assert len(table) == 256
    for i in (0, 1, 2, 3, 17, 100, 254, 255):
        inf, x, y = oracle.affine_mul(1, 2, i + 1)
        assert not inf and (x, y) == table[i]
    mont = H.mont_point_array(table)
    assert all(oracle.on_curve(mont[i]) for i in range(256))


def test_known_points(oracle):
    """tests/ec_test.cu:7-25: 1G..4G, and x + 1 = next (ec_test x[i]+1 identity)."""
    pts = H.load_known_points()
    for k, (x, y) in enumerate(pts, start=1):
        assert oracle.affine_mul(1, 2, k) == (False, x, y)
    g = (False, 1, 2)
    acc = g
    for k in range(2, 5):
        acc = oracle.affine_add(acc, g)
        assert acc == (False, *pts[k - 1])
    # x + (-x) = infinity, x + x = 2x
    neg = (False, pts[2][0], (P - pts[2][1]) % P)
    assert oracle.affine_add((False, *pts[2]), neg)[0]
    assert oracle.affine_add((False, *pts[1]), (False, *pts[1])) == (False, *pts[3])


@pytest.mark.parametrize("case", H.load_json("msm_small.json")["cases"], ids=lambda c: c["name"])
def test_small_msm_fixtures(oracle, case):
    """Fixtures computed by the reference's host code: naive, Pippenger and checksum agree."""
    table = H.load_g_bases()
    bases = H.mont_point_array([table[i] for i in case["bases"]])
    values = [int(s, 16) for s in case["scalars"]]
    scalars = H.mont_scalar_array(values)
    exp = H.expected_point(case)
    assert oracle.msm_naive(bases, scalars) == exp
    assert oracle.msm_pippenger(bases, scalars, 1) == exp
    assert oracle.msm_pippenger(bases, scalars, 4) == exp
    k = np.zeros((len(values), 8), np.uint32)
    k[:, 0] = np.array(case["bases"]) + 1
    assert oracle.msm_checksum(k, scalars) == exp


def test_config0_fixture(oracle):
    """N = 2^12, seed 0: the generator reproduces the committed input digests and
    the oracle reproduces the reference-computed result."""
    import hashlib
    cfg = H.load_json("config0.json")
    scalars, k = synth.workload("uniform", cfg["n"], cfg["seed"])
    assert hashlib.sha256(scalars.tobytes()).hexdigest() == cfg["scalars_sha256"]
    assert hashlib.sha256(k.tobytes()).hexdigest() == cfg["k_sha256"]
    bases = oracle.gen_bases(k)
    assert hashlib.sha256(bases.tobytes()).hexdigest() == cfg["bases_sha256"]
    exp = H.expected_point(cfg)
    assert oracle.msm_checksum(k, scalars) == exp
    assert oracle.msm_pippenger(bases, scalars) == exp


def test_pippenger_vs_checksum_skewed(oracle):
    n = 3000
    scalars, k = synth.workload("skewed", n, 2)
    bases = oracle.gen_bases(k)
    assert oracle.msm_pippenger(bases, scalars) == oracle.msm_checksum(k, scalars)


def test_horner_of_single_point(oracle):
    """R_0 = P, others infinity -> P; R_i = P -> 2^i P."""
    jac = np.zeros((254, 24), np.uint32)
    inf_one = H.limbs(H.MONT % P)
    for i in range(254):
        jac[i, 8:16] = inf_one  # (0, 1, 0) in Montgomery form
    g = H.mont_point_array([(1, 2)])[0]
    jac[5, :16] = g
    jac[5, 16:] = inf_one
    assert oracle.horner(jac) == oracle.affine_mul(1, 2, 32)


REF_HOST = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libref_host.so")


@pytest.mark.skipif(not os.path.exists(REF_HOST), reason="reference host build absent (make -C oracle ref)")
def test_oracle_matches_reference_host_code(oracle):
    """Random field products and small MSMs against the reference's own host code."""
    ref = ctypes.CDLL(REF_HOST)
    u32p = ctypes.POINTER(ctypes.c_uint32)
    rng = np.random.Generator(np.random.PCG64(11))
    for _ in range(200):
        a = int.from_bytes(rng.bytes(32), "little") % P
        b = int.from_bytes(rng.bytes(32), "little") % P
        out = np.zeros(8, np.uint32)
        ref.ref_fq_mul(H.limbs(a).ctypes.data_as(u32p), H.limbs(b).ctypes.data_as(u32p), out.ctypes.data_as(u32p))
        assert H.to_int(out) == a * b * pow(2, -256, P) % P
    for trial in range(5):
        n = 8
        scalars, k = synth.workload("uniform", n, 50 + trial)
        bases = oracle.gen_bases(k)
        jac = np.zeros(24, np.uint32)
        ref.ref_msm_naive(bases.ctypes.data_as(u32p), scalars.ctypes.data_as(u32p), ctypes.c_uint(n), jac.ctypes.data_as(u32p))
        assert oracle.normalize(jac) == oracle.msm_naive(bases, scalars) == oracle.msm_checksum(k, scalars)
