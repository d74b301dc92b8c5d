import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path through the C-ABI)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle as O
    O.build()
    return O


def perturb(case, seed=0, amp=0.01):
    """Seeded smooth + random perturbation of the freestream state on every
    block (all nodes, ghosts included), so every term of the residual is
    exercised."""
    rng = np.random.default_rng(seed)
    for b in case.blocks:
        q = b.fields["q"]
        nz, ny, nx, _ = q.shape
        k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        smooth = np.sin(0.3 * i + 0.2 * j + 0.5 * k + b.m)
        q[..., 0] *= 1.0 + amp * (smooth + 0.3 * rng.standard_normal(smooth.shape))
        for c in (1, 2, 3):
            q[..., c] += amp * (np.cos(0.25 * i * c + 0.4 * j + 0.3 * k) + 0.3 * rng.standard_normal(smooth.shape))
        q[..., 4] *= 1.0 + amp * (0.5 * smooth + 0.3 * rng.standard_normal(smooth.shape))
        if case.cfg.turbulence:
            b.fields["nut"][...] *= 1.0 + amp * rng.standard_normal(b.fields["nut"].shape)


def relerr(a, b):
    """max |a-b| / max |b| over finite entries (NaN positions must agree)."""
    a = np.asarray(a); b = np.asarray(b)
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb), "NaN positions differ"
    m = ~nb
    if not m.any():
        return 0.0
    scale = np.max(np.abs(b[m]))
    if scale == 0.0:
        return float(np.max(np.abs(a[m])))
    return float(np.max(np.abs(a[m] - b[m])) / scale)
