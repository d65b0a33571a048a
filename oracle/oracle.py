"""Python wrapper of the CPU oracle (liboracle_bn254.so) and of the reference
builds under oracle/_ref.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, always as the checker or as the
timed CPU baseline, never on the product path.

Normalised points are (is_infinity, x, y) with x, y standard-form integers.
"""
from __future__ import annotations

import ctypes
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_bn254.so")
REF_HOST = os.path.join(HERE, "_ref", "libref_host.so")
REF_GPU = os.path.join(HERE, "_ref", "libbellman-cuda-ref.so")

P = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001

_u32p = ctypes.POINTER(ctypes.c_uint32)


def _p(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u32p)


def limbs_to_int(a) -> int:
    return sum(int(a[i]) << (32 * i) for i in range(len(a)))


def int_to_limbs(x: int, n: int = 8) -> np.ndarray:
    return np.array([(x >> (32 * i)) & 0xFFFFFFFF for i in range(n)], dtype=np.uint32)


class Oracle:
    def __init__(self, path: str = LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        self.lib = ctypes.CDLL(path)
        for name in ("orc_msm_naive", "orc_msm_pippenger", "orc_msm_checksum", "orc_horner", "orc_jacobian_normalize",
                     "orc_gen_bases", "orc_affine_is_on_curve", "orc_affine_mul", "orc_affine_add"):
            getattr(self.lib, name).restype = ctypes.c_int

    @staticmethod
    def _point(inf: int, out: np.ndarray):
        return (bool(inf), limbs_to_int(out[:8]), limbs_to_int(out[8:]))

    def fq_to_mont(self, x: int) -> int:
        out = np.zeros(8, np.uint32)
        self.lib.orc_fq_to_mont(_p(int_to_limbs(x)), _p(out))
        return limbs_to_int(out)

    def fr_to_mont_batch(self, a: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.uint32)
        out = np.empty_like(a)
        self.lib.orc_fr_to_mont_batch(_p(a), _p(out), ctypes.c_size_t(len(a)))
        return out

    def gen_bases(self, k_std: np.ndarray, threads: int = 0) -> np.ndarray:
        k_std = np.ascontiguousarray(k_std, dtype=np.uint32)
        out = np.empty((len(k_std), 16), np.uint32)
        rc = self.lib.orc_gen_bases(_p(k_std), ctypes.c_size_t(len(k_std)), _p(out), threads)
        if rc != 0:
            raise ValueError("k must be in [1, r)")
        return out

    def msm_naive(self, bases: np.ndarray, scalars: np.ndarray):
        out = np.zeros(16, np.uint32)
        inf = self.lib.orc_msm_naive(_p(np.ascontiguousarray(bases)), _p(np.ascontiguousarray(scalars)), ctypes.c_size_t(len(scalars)), _p(out))
        return self._point(inf, out)

    def msm_pippenger(self, bases: np.ndarray, scalars: np.ndarray, threads: int = 0):
        out = np.zeros(16, np.uint32)
        inf = self.lib.orc_msm_pippenger(_p(np.ascontiguousarray(bases)), _p(np.ascontiguousarray(scalars)), ctypes.c_size_t(len(scalars)),
                                         threads, _p(out))
        return self._point(inf, out)

    def msm_checksum(self, k_std: np.ndarray, scalars: np.ndarray):
        out = np.zeros(16, np.uint32)
        inf = self.lib.orc_msm_checksum(_p(np.ascontiguousarray(k_std)), _p(np.ascontiguousarray(scalars)), ctypes.c_size_t(len(scalars)), _p(out))
        return self._point(inf, out)

    def horner(self, results: np.ndarray):
        """results: (254, 24) uint32 Montgomery Jacobian points -> normalised sum 2^i R_i."""
        results = np.ascontiguousarray(results, dtype=np.uint32).reshape(-1, 24)
        out = np.zeros(16, np.uint32)
        inf = self.lib.orc_horner(_p(results), ctypes.c_size_t(len(results)), _p(out))
        return self._point(inf, out)

    def normalize(self, jac: np.ndarray):
        out = np.zeros(16, np.uint32)
        inf = self.lib.orc_jacobian_normalize(_p(np.ascontiguousarray(jac, dtype=np.uint32)), _p(out))
        return self._point(inf, out)

    def on_curve(self, aff_mont: np.ndarray) -> bool:
        return bool(self.lib.orc_affine_is_on_curve(_p(np.ascontiguousarray(aff_mont, dtype=np.uint32))))

    def affine_mul(self, x: int, y: int, k: int):
        pt = np.concatenate([int_to_limbs(x), int_to_limbs(y)])
        out = np.zeros(16, np.uint32)
        inf = self.lib.orc_affine_mul(_p(pt), _p(int_to_limbs(k)), _p(out))
        return self._point(inf, out)

    def affine_add(self, a, b):
        pa = np.concatenate([int_to_limbs(a[1]), int_to_limbs(a[2])])
        pb = np.concatenate([int_to_limbs(b[1]), int_to_limbs(b[2])])
        out = np.zeros(16, np.uint32)
        inf = self.lib.orc_affine_add(_p(pa), int(a[0]), _p(pb), int(b[0]), _p(out))
        return self._point(inf, out)


def time_cpu_pippenger(oracle: Oracle, bases: np.ndarray, scalars: np.ndarray, threads: int = 0):
    """Wall-clock seconds of one host Pippenger over the given points."""
    t0 = time.perf_counter()
    pt = oracle.msm_pippenger(bases, scalars, threads)
    return time.perf_counter() - t0, pt
