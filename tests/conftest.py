"""Shared fixtures.  `-m "not gpu"` runs the CPU suite (oracle pinning, host
emulation of the product field code, ABI layout); `-m gpu` runs the parity
tests on a B200 through the C ABI."""
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "era-bellman-cuda_b200")
ORACLE_DIR = os.path.join(REPO, "oracle")
NATIVE = os.path.join(REPO, "tests", "native")
for p in (PKG, ORACLE_DIR, os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs through the C ABI")


def _make(target_dir, *targets):
    subprocess.run(["make", "-s", "-C", target_dir, *targets], check=True)


@pytest.fixture(scope="session")
def oracle():
    _make(ORACLE_DIR)
    import oracle as orc
    return orc.Oracle()


@pytest.fixture(scope="session")
def field_check():
    """The product field/curve headers compiled for the host (emulated carries)."""
    import ctypes
    out_dir = os.path.join(NATIVE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    so = os.path.join(out_dir, "libfield_check.so")
    src = os.path.join(NATIVE, "field_check.cpp")
    hdrs = [os.path.join(PKG, "csrc", h) for h in ("bn254_field.cuh", "bn254_curve.cuh")]
    if not os.path.exists(so) or any(os.path.getmtime(f) > os.path.getmtime(so) for f in [src] + hdrs):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I" + os.path.join(PKG, "csrc"), "-o", so, src], check=True)
    return ctypes.CDLL(so)


@pytest.fixture(scope="session")
def product_lib_path():
    path = os.path.join(PKG, "lib", "libbellman_cuda_b200.so")
    if not os.path.exists(path):
        _make(PKG)
    return path
