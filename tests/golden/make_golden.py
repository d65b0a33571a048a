"""Generates the committed golden fixtures in tests/golden/.

Run where the reference source tree exists (its path as the first argument,
else the REF environment variable, else a `reference` directory beside this
repository) and the reference host build (make -C oracle ref REF=...):

    python tests/golden/make_golden.py [/path/to/era-bellman-cuda]

Outputs
  g_bases.txt      the reference MSM test table g_bases[i] = (i+1) * G
                   (reference tests/msm_bases.cuh:8-520), "x y" hex, standard form
  known_points.txt 1G..4G from the reference curve test (tests/ec_test.cu:7-25)
  msm_small.json   small MSMs whose expected values are computed by the
                   reference's own host code (ref_msm_naive in
                   oracle/ref_host_shim.cu: double-and-add per term)
  config0.json     the N = 2^12, seed 0 workload: input digests and the
                   expected normalised MSM (reference host code, cross-checked
                   by the oracle's checksum and Pippenger)
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "era-bellman-cuda_b200"))

import oracle as orc  # noqa: E402
import synth  # noqa: E402

P, R = orc.P, orc.R


def parse_point_table(text: str):
    """All {{8 limbs}, {8 limbs}} pairs in a C initializer, as (x, y) ints."""
    pts = []
    for m in re.finditer(r"\{\{([^{}]*)\},\s*\{([^{}]*)\}\}", text):
        xs = [int(v, 16) for v in re.findall(r"0x[0-9a-fA-F]+", m.group(1))]
        ys = [int(v, 16) for v in re.findall(r"0x[0-9a-fA-F]+", m.group(2))]
        if len(xs) == 8 and len(ys) == 8:
            pts.append((sum(v << (32 * i) for i, v in enumerate(xs)), sum(v << (32 * i) for i, v in enumerate(ys))))
    return pts


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main(ref_root: str) -> None:
    o = orc.Oracle()
    ref = ctypes.CDLL(orc.REF_HOST)
    u32p = ctypes.POINTER(ctypes.c_uint32)

    # --- fixture tables from the reference tests ---------------------------
    g_bases = parse_point_table(open(os.path.join(ref_root, "tests", "msm_bases.cuh")).read())
    assert len(g_bases) == 256, len(g_bases)
    with open(os.path.join(HERE, "g_bases.txt"), "w") as f:
        f.write("# g_bases[i] = (i+1)*G, standard-form affine x y (reference tests/msm_bases.cuh)\n")
        for x, y in g_bases:
            f.write(f"{x:064x} {y:064x}\n")
    ec_text = open(os.path.join(ref_root, "tests", "ec_test.cu")).read()
    known = [(1, 2)] + parse_point_table(ec_text)[:3]
    with open(os.path.join(HERE, "known_points.txt"), "w") as f:
        f.write("# kG for k = 1..4, standard-form affine x y (reference tests/ec_test.cu)\n")
        for x, y in known:
            f.write(f"{x:064x} {y:064x}\n")

    def mont_bases(points):
        out = np.zeros((len(points), 16), np.uint32)
        for i, (x, y) in enumerate(points):
            out[i, :8] = orc.int_to_limbs(o.fq_to_mont(x))
            out[i, 8:] = orc.int_to_limbs(o.fq_to_mont(y))
        return out

    def ref_msm(bases_mont, scalars_mont):
        jac = np.zeros(24, np.uint32)
        ref.ref_msm_naive(bases_mont.ctypes.data_as(u32p), scalars_mont.ctypes.data_as(u32p), ctypes.c_uint(len(scalars_mont)),
                          jac.ctypes.data_as(u32p))
        return o.normalize(jac)

    def mont_scalars(values):
        return np.stack([orc.int_to_limbs((v * (1 << 256)) % R) for v in values]).astype(np.uint32)

    rng = np.random.Generator(np.random.PCG64(np.random.SeedSequence([2024, 7])))
    cases = []

    def add_case(name, base_idx, values):
        pts = [g_bases[i] for i in base_idx]
        bm = mont_bases(pts)
        sm = mont_scalars(values)
        inf, x, y = ref_msm(bm, sm)
        cases.append({"name": name, "bases": [int(i) for i in base_idx], "scalars": [f"{v:064x}" for v in values],
                      "infinity": inf, "x": f"{x:064x}", "y": f"{y:064x}"})

    def rand_fr(k):
        return [int.from_bytes(rng.bytes(32), "little") % R for _ in range(k)]

    add_case("uniform16", list(range(16)), rand_fr(16))
    add_case("single", [5], rand_fr(1))
    add_case("special", list(range(12)), [0, 1, 2, R - 1, R - 2, (R - 1) // 2, (R + 1) // 2, 1 << 253, (1 << 253) - 1, 0xFFFF, 1 << 16, 3])
    add_case("all_zero", list(range(8)), [0] * 8)
    add_case("cancel", [7, 7, 9, 9], [5, R - 5, 123456789, R - 123456789])
    add_case("duplicates64", [int(v) for v in rng.integers(0, 4, 64)], rand_fr(64))
    add_case("ones32", list(range(32)), [1] * 32)
    add_case("table256", list(range(256)), rand_fr(256))
    with open(os.path.join(HERE, "msm_small.json"), "w") as f:
        json.dump({"source": "reference host code (ref_msm_naive)", "cases": cases}, f, indent=1)

    # --- config 0: N = 2^12, seed 0 -------------------------------------------
    n = 1 << 12
    scalars, k = synth.workload("uniform", n, 0)
    bases = o.gen_bases(k)
    expected_ref = ref_msm(bases, scalars)
    checksum = o.msm_checksum(k, scalars)
    pip = o.msm_pippenger(bases, scalars)
    assert expected_ref == checksum == pip, (expected_ref, checksum, pip)
    cfg0 = {
        "n": n, "seed": 0, "distribution": "uniform",
        "scalars_sha256": digest(scalars), "k_sha256": digest(k), "bases_sha256": digest(bases),
        "infinity": expected_ref[0], "x": f"{expected_ref[1]:064x}", "y": f"{expected_ref[2]:064x}",
        "source": "reference host code (ref_msm_naive); equal to the oracle checksum and Pippenger",
    }
    with open(os.path.join(HERE, "config0.json"), "w") as f:
        json.dump(cfg0, f, indent=1)
    print("golden fixtures written:", len(cases), "small cases; config0", cfg0["x"][:16])


if __name__ == "__main__":
    repo = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF") or os.path.join(os.path.dirname(repo), "reference"))
