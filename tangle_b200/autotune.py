"""Launch-shape autotuner with a per-(GPU, workload shape) cache.

The relaxation kernels take a few launch shapes that never change a result
(the C ABI's `tgl_launch_params`): lanes per fiber in the curvature sweeps,
contact-pass blocks per SM, the Verlet build's staging chunk and the
contact-list skin. `tgl_autotune` times candidates of each on the world's
own state and keeps the fastest; this module caches the choice per GPU
model and workload shape, so a later world of the same shape applies it
without searching.

The cache is a JSON file: `TGL_AUTOTUNE_CACHE`, else
`~/.cache/tangle_b200/autotune.json`. Entries are keyed by the GPU name and
the world's shape: vertex, segment, fiber and cell counts, the cell grid,
the neighbor-list block, the number of specimens (arenas), the longest
fiber and the motion model. The reference has no counterpart (its CubeCL
kernels take fixed launch shapes).
"""

from __future__ import annotations

import json
import os
import tempfile
from pathlib import Path
from typing import Optional

from .settings import RelaxationConfig


def cache_path(path: Optional[str] = None) -> Path:
    if path:
        return Path(path)
    env = os.environ.get("TGL_AUTOTUNE_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "tangle_b200" / "autotune.json"


def gpu_name() -> str:
    import torch

    return torch.cuda.get_device_name(torch.cuda.current_device())


def workload_key(gpu: str, shape: dict) -> str:
    """The cache key: the GPU's name and the world's shape, as a stable
    JSON string."""
    return json.dumps({"gpu": gpu, **{k: shape[k] for k in sorted(shape)}}, sort_keys=True)


def world_shape(world, config: RelaxationConfig) -> dict:
    return {
        "vertices": int(world.vertex_count),
        "segments": int(world.segment_count),
        "cells": int(world.cell_count),
        "cell_dims": [int(x) for x in world.cell_dims],
        "neighbor_block": int(world.neighbor_block),
        "specimens": len(getattr(world, "specimen_vertices", None) or [0]),
        "contact_lists": bool(world.contact_list_info()["block"] > 0),
        "motion_model": str(config.motion_model),
    }


def load(path: Path) -> dict:
    try:
        with open(path) as fh:
            data = json.load(fh)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def store(path: Path, key: str, entry: dict) -> None:
    """Adds `entry` under `key`, written atomically (temporary file renamed
    over the cache)."""
    data = load(path)
    data[key] = entry
    path.parent.mkdir(parents=True, exist_ok=True)
    fd, tmp = tempfile.mkstemp(prefix=path.name + ".", suffix=".tmp", dir=str(path.parent))
    try:
        with os.fdopen(fd, "w") as fh:
            json.dump(data, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except BaseException:
        if os.path.exists(tmp):
            os.unlink(tmp)
        raise


def autotune(world, config: RelaxationConfig, *, trial_iterations: int = 32, path: Optional[str] = None,
             force: bool = False, gpu: Optional[str] = None) -> dict:
    """Applies the cached launch shapes of this GPU and workload shape, or
    searches them on `world` (leaving its state as it was) and caches the
    result. Returns {"params", "cached", "report"}."""
    where = cache_path(path)
    key = workload_key(gpu or gpu_name(), world_shape(world, config))
    if not force:
        entry = load(where).get(key)
        if entry and "params" in entry:
            try:
                world.set_launch_params(entry["params"])
                return {"params": entry["params"], "cached": True, "report": entry.get("report")}
            except (RuntimeError, ValueError, KeyError):
                pass  # a stale or foreign entry: search again
    params, report = world.autotune_trials(config, trial_iterations)
    store(where, key, {"params": params, "report": report})
    return {"params": params, "cached": False, "report": report}
