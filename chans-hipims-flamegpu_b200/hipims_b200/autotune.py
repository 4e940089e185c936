"""Autotuner for the fused step's launch shape.

For a batch of catchments it times a few steps of each candidate (cells per
lane -- 2 with 32 x 64 tiles, 1 with 32 x 32 or 64 x 32 tiles -- tile height and
resident-CTA count) on scratch copies of the catchments, keeps the fastest,
and caches the choice in a JSON file keyed by the GPU name, the dtype and the
batch's shape (number of instances, total cells, largest side).

Each candidate is timed after a spin-up of SPINUP_STEPS untimed steps: the
first steps from a dry start leave most faces dry, where the one-cell kernel's
dry-face shortcuts make it the fastest, while from the first few steps of
rain on the two-cells-per-lane build is faster by 15-30 % on the 64-catchment
ensemble (measured on a B200: 1.14 vs 1.11 ms per step after 3 steps,
1.15 vs 1.33 after 8, 1.16 vs 1.50 after 20).  The cache
lives at $HIPIMS_B200_TUNE_CACHE, default ~/.cache/hipims_b200/autotune.json.
"""
from __future__ import annotations

import json
import os
from typing import Sequence

import torch

from .fused import Catchment, FusedSolver

# tile = (rows, cols); cols / 32 cells per lane
DEFAULT_CANDIDATES = ({"tile": (32, 64), "minb": 4}, {"tile": (32, 64), "minb": 3},
                      {"tile": (64, 32), "minb": 4}, {"tile": (32, 32), "minb": 5},
                      {"tile": (32, 32), "minb": 6})


# untimed steps before a candidate is timed (see the module docstring)
SPINUP_STEPS = 16


def cells_per_lane(cfg: dict) -> int:
    return int(cfg["tile"][1]) // 32


def cache_path() -> str:
    return os.environ.get("HIPIMS_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "hipims_b200",
                                       "autotune.json"))


def batch_key(catchments: Sequence[Catchment], dtype: torch.dtype, device) -> str:
    name = torch.cuda.get_device_name(device)
    cells = sum(int(c.mask.size) for c in catchments)
    side = max(max(c.mask.shape) for c in catchments)
    return (f"{name}|{str(dtype).split('.')[-1]}|n={len(catchments)}|cells={cells}|side={side}"
            f"|spinup={SPINUP_STEPS}")


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(db: dict) -> None:
    p = cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(db, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def time_config(catchments: Sequence[Catchment], dtype, device, cfg: dict, steps: int = 6,
                warmup: int = SPINUP_STEPS) -> float:
    """Milliseconds per step of one candidate (CUDA events, after `warmup`
    untimed steps from the catchments' initial state)."""
    fs = FusedSolver(list(catchments), dtype=dtype, device=device, tile=cfg["tile"],
                     grid_blocks=cfg.get("grid_blocks", 0), minb=cfg.get("minb", 0))
    fs.step(warmup)
    st = torch.cuda.current_stream(device)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    fs.step(steps)
    b.record(st)
    torch.cuda.synchronize(device)
    ms = a.elapsed_time(b) / steps
    del fs
    torch.cuda.empty_cache()
    return ms


def tune(catchments: Sequence[Catchment], dtype=torch.float32, device="cuda",
         candidates: Sequence[dict] = DEFAULT_CANDIDATES, use_cache: bool = True,
         steps: int = 6) -> dict:
    """Best launch configuration for this batch: {"tile": (ty, tx), ...}."""
    device = torch.device(device)
    if dtype == torch.float64:
        return {"tile": (32, 32)}  # the only FP64 rows-kernel build
    key = batch_key(catchments, dtype, device)
    db = _load() if use_cache else {}
    if key in db:
        c = db[key]["best"]
        return {"tile": tuple(c["tile"]), "grid_blocks": c.get("grid_blocks", 0),
                "minb": c.get("minb", 0)}
    results = []
    for cfg in candidates:
        ms = time_config(catchments, dtype, device, cfg, steps=steps)
        results.append((ms, cfg))
    ms, best = min(results, key=lambda r: r[0])
    if use_cache:
        db[key] = {"best": {"tile": list(best["tile"]), "grid_blocks": best.get("grid_blocks", 0),
                            "minb": best.get("minb", 0)},
                   "ms_per_step": ms,
                   "tried": [{"tile": list(c["tile"]), "grid_blocks": c.get("grid_blocks", 0),
                              "minb": c.get("minb", 0), "ms": m} for m, c in results]}
        _store(db)
    return {"tile": tuple(best["tile"]), "grid_blocks": best.get("grid_blocks", 0),
            "minb": best.get("minb", 0), "tried": [(c, m) for m, c in results]}
