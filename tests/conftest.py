"""Shared test setup: import paths, the `gpu` marker, small synthetic inputs."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "mg-glam-durham_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import ctypes
        cudart = ctypes.CDLL("libcudart.so")
    except OSError:
        try:
            import torch
            return torch.cuda.is_available()
        except Exception:
            return False
    n = ctypes.c_int(0)
    return cudart.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0


def random_particles(nrow, ngrid, seed=0, vscale=0.1, clustered=False):
    """Positions in [1, ngrid+1) as float32 SoA, velocities ~ N(0, vscale)."""
    rng = np.random.default_rng(seed)
    n = nrow ** 3
    if clustered:
        # half uniform, half in a few compact clumps (exercises dense rows/cells)
        u = rng.random((n, 3))
        m = n // 2
        centers = rng.random((8, 3))
        pick = rng.integers(0, 8, m)
        u[:m] = (centers[pick] + 0.01 * rng.standard_normal((m, 3))) % 1.0
    else:
        u = rng.random((n, 3))
    pos = (1.0 + u * ngrid).astype(np.float32)
    pos = np.where(pos >= ngrid + 1, np.float32(ngrid + 1) - np.float32(1e-3), pos).astype(np.float32)
    vel = (vscale * rng.standard_normal((n, 3))).astype(np.float32)
    return [pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(),
            vel[:, 0].copy(), vel[:, 1].copy(), vel[:, 2].copy()]


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle
