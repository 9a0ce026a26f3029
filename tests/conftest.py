import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "antimatter-kernel_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

E = 1.602176634e-19


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls libamk.so")


@pytest.fixture(scope="module")
def sim():
    import amk
    s = amk.Simulation()
    yield s
    s.close()


def gaussian_cloud(n, seed, sigma=(1e-4, 1e-4, 3e-4), mixed=True):
    rng = np.random.default_rng(seed)
    x = rng.normal(0.0, sigma[0], n)
    y = rng.normal(0.0, sigma[1], n)
    z = rng.normal(0.0, sigma[2], n)
    q = np.where(rng.random(n) < 0.5, E, -E) if mixed else np.full(n, E)
    return x, y, z, q


def rel_errors(f, g):
    """Per-particle |dF|/|F| and the global ratio ||dF||/||F||."""
    f = np.asarray(f).reshape(3, -1) if np.ndim(f) == 2 and np.shape(f)[0] == 3 else np.asarray(f)
    num = np.sqrt(sum((a - b) ** 2 for a, b in zip(f, g)))
    den = np.sqrt(sum(b ** 2 for b in g))
    ok = den > 0
    rel = num[ok] / den[ok]
    return rel, float(np.sqrt(np.sum(num ** 2) / max(np.sum(den ** 2), 1e-300)))
