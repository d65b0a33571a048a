"""The request server's admission arena (csrc/device_arena.h), built for the
host: first-fit allocation, 256-byte rounding, coalescing on release, and a
randomised run against a byte-map model (no overlaps, exact accounting)."""
import ctypes
import os
import random
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "era-bellman-cuda_b200", "csrc")


@pytest.fixture(scope="module")
def arena():
    out = os.path.join(HERE, "native", "_build")
    os.makedirs(out, exist_ok=True)
    so = os.path.join(out, "libarena_check.so")
    src = os.path.join(HERE, "native", "arena_check.cpp")
    hdr = os.path.join(CSRC, "device_arena.h")
    if not os.path.exists(so) or max(os.path.getmtime(src), os.path.getmtime(hdr)) > os.path.getmtime(so):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I" + CSRC, "-o", so, src], check=True)
    lib = ctypes.CDLL(so)
    lib.arena_reset.argtypes = [ctypes.c_size_t]
    lib.arena_allocate.argtypes = [ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    lib.arena_release.argtypes = [ctypes.c_size_t, ctypes.c_size_t]
    for f in ("arena_largest_free", "arena_used", "arena_free_blocks"):
        getattr(lib, f).restype = ctypes.c_size_t
    return lib


def alloc(lib, n):
    off = ctypes.c_size_t()
    return off.value if lib.arena_allocate(n, ctypes.byref(off)) else None


def test_first_fit_and_coalescing(arena):
    arena.arena_reset(4096)
    a, b, c = alloc(arena, 1000), alloc(arena, 256), alloc(arena, 1)
    assert (a, b, c) == (0, 1024, 1280)
    assert arena.arena_used() == 1536
    assert alloc(arena, 4096) is None
    arena.arena_release(b, 256)
    assert alloc(arena, 200) == 1024  # first fit reuses the hole
    arena.arena_release(1024, 200)
    arena.arena_release(a, 1000)
    arena.arena_release(c, 1)
    assert arena.arena_used() == 0 and arena.arena_free_blocks() == 1 and arena.arena_largest_free() == 4096


def test_randomised_against_model(arena):
    size = 1 << 20
    arena.arena_reset(size)
    rng = random.Random(7)
    live = {}
    owner = bytearray(size // 256)
    for _ in range(4000):
        if live and rng.random() < 0.45:
            off = rng.choice(list(live))
            n = live.pop(off)
            arena.arena_release(off, n)
            blocks = -(-n // 256)
            owner[off // 256: off // 256 + blocks] = bytes(blocks)
        else:
            n = rng.randint(1, 40000)
            off = alloc(arena, n)
            blocks = -(-n // 256)
            if off is None:
                # refused only when no free run of `blocks` exists
                run = best = 0
                for x in owner:
                    run = run + 1 if x == 0 else 0
                    best = max(best, run)
                assert best < blocks
                continue
            assert off % 256 == 0 and off + blocks * 256 <= size
            assert not any(owner[off // 256: off // 256 + blocks])
            owner[off // 256: off // 256 + blocks] = b"\x01" * blocks
            live[off] = n
        assert arena.arena_used() == 256 * sum(owner)
