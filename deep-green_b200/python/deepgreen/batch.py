"""The batched workload: many independent grids of uneven sizes, each a
random two-state Riemann problem (setups.riemann_random), stepped together
by dg_batch.  Also the autotuning cache: the chosen tiling per batch
signature is kept in a JSON file."""
from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path

import numpy as np

from . import capi, setups


def grid_shapes(n_grids=64, lo=32, hi=160, seed=2024):
    """Edge lengths log-uniform in [lo, hi] per axis (seeded)."""
    rng = np.random.default_rng(seed)
    e = np.exp(rng.uniform(np.log(lo), np.log(hi), size=(n_grids, 3)))
    return [tuple(int(round(v)) for v in row) for row in e]


def make_batch(shapes, seed=2024, limiter=capi.LIMITER_MINMOD, bcs=(capi.OUTFLOW,) * 6, device=0, reorient=False):
    """A Batch with grid i holding riemann_random(shapes[i], seed + i)
    (reorient: capi.Batch's stored-axis choice)."""
    specs, prims = [], []
    for i, sh in enumerate(shapes):
        prim, ds, b = setups.riemann_random(sh, seed + i, bcs=bcs)
        specs.append({"shape": sh, "ds": ds, "bcs": b, "limiter": limiter})
        prims.append(prim)
    bt = capi.Batch(specs, device=device, reorient=reorient)
    for i, p in enumerate(prims):
        bt.set_primitives(i, p)
    return bt, specs, prims


def signature(shapes, device_name, reorient=False):
    # the tiling candidates belong to the kernel: its name is part of the key,
    # and so is the stored layout
    key = [sorted(shapes), device_name, "sweep14"] + (["reoriented"] if reorient else [])
    h = hashlib.sha1(json.dumps(key).encode()).hexdigest()[:16]
    return h


def tuned(bt, shapes, device_name, cache_path=None, steps=3, reorient=False):
    """Tiling for this batch: from the JSON cache if present, else timed by
    dg_batch_autotune and stored."""
    path = Path(cache_path or os.environ.get("DG_AUTOTUNE_CACHE", Path.home() / ".cache" / "deepgreen_tuning.json"))
    key = signature(shapes, device_name, reorient)
    cache = {}
    if path.exists():
        try:
            cache = json.loads(path.read_text())
        except (OSError, ValueError):
            cache = {}
    if key in cache:
        rows, chunk = cache[key]["tile_rows"], cache[key]["chunk"]
        bt.set_tiling(rows, chunk)
        return rows, chunk, cache[key].get("ms_per_step"), True
    rows, chunk, ms = bt.autotune(steps)
    cache[key] = {"tile_rows": rows, "chunk": chunk, "ms_per_step": ms}
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_text(json.dumps(cache, indent=1))
    except OSError:
        pass
    return rows, chunk, ms, False
