"""Shared test set-up: import paths, the `gpu` marker, helpers."""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "deep-green_b200" / "python", ROOT / "oracle", ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) and the built libdeepgreen.so")


INTERIOR = (slice(2, -2),) * 3


def rel_l1(a, b):
    """sum |a - b| / sum |b| over interior cells (b is the reference)."""
    a = np.asarray(a, dtype=np.float64)[INTERIOR]
    b = np.asarray(b, dtype=np.float64)[INTERIOR]
    den = np.abs(b).sum()
    return float(np.abs(a - b).sum() / den) if den > 0 else float(np.abs(a - b).sum())


def random_primitives(shape, seed):
    """Smooth-ish random primitive state on a ghosted grid (positive rho, p)."""
    rng = np.random.default_rng(seed)
    n = tuple(s + 4 for s in shape)
    return [rng.uniform(0.5, 2.0, n), rng.uniform(-0.5, 0.5, n), rng.uniform(-0.5, 0.5, n),
            rng.uniform(-0.5, 0.5, n), rng.uniform(0.5, 2.0, n)]
