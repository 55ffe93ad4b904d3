"""Shared test setup: import paths, markers, and on-demand builds.

The product library (jump-cannon_b200/libjc_layout.so) and the CPU oracle
(oracle/liboracle.so) are built here if they are missing or stale; nvcc and
g++ are present both here and on the GPU box.
"""
import importlib.util
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "jump-cannon_b200"
for p in (str(ROOT), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


def _load_build_module():
    spec = importlib.util.spec_from_file_location("jc_build", PKG / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    _load_build_module().build()
    import oracle.oracle as orc
    orc.build()
    yield


@pytest.fixture(scope="session")
def jc():
    import jc_layout
    return jc_layout


@pytest.fixture(scope="session")
def orc():
    import oracle.oracle as orc
    return orc


def spiral_seed(n: int, z: float = 0.0) -> np.ndarray:
    """Golden-angle spiral (crates/graph-compute/tests/gpu_engines.rs:24-36)."""
    ga = np.float32(np.pi) * (np.float32(3.0) - np.sqrt(np.float32(5.0)))
    out = np.zeros(3 * n, np.float32)
    for i in range(n):
        r = np.sqrt(np.float32(i) + np.float32(1.0))
        a = np.float32(i) * ga
        out[3 * i] = r * np.cos(a)
        out[3 * i + 1] = r * np.sin(a)
        out[3 * i + 2] = z
    return out


def ring_seed(n: int) -> np.ndarray:
    """ring_positions (crates/graph-compute/src/engines/sgd_stress.rs:401-409)."""
    p = np.zeros(3 * n, np.float32)
    for i in range(n):
        t = np.float32(i) / np.float32(max(n, 1)) * np.float32(2 * np.pi)
        p[3 * i] = np.cos(t)
        p[3 * i + 1] = np.sin(t)
    return p


def gpu_available() -> bool:
    if os.environ.get("JC_FORCE_NO_GPU"):
        return False
    try:
        import ctypes
        rt = ctypes.CDLL("libcudart.so.12")
        cnt = ctypes.c_int(0)
        return rt.cudaGetDeviceCount(ctypes.byref(cnt)) == 0 and cnt.value > 0
    except OSError:
        return False
