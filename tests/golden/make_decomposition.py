"""Generate tests/golden/multigpu/decomposition.npz from the reference's own
multi-GPU decomposition functions.

HP/MultiGPU_CatchFlood_main.py splits a raster into row strips
(`ave_loadStep`) and numbers the overlap cells that its ranks exchange
(`ave_overlapMask`).  This script executes those two functions from the
reference file in place (only their definitions, parsed out of the file; the
module itself is not imported, since it needs GIS libraries and a process
group) on seeded synthetic catchments -- square urban rasters and ragged
random masks with holes -- and stores each mask with the split rows and the
overlap numbering, which pin baseline/ref_loop.py's restatement
(`row_splits`, `overlap_mask`) wherever the reference tree is absent.

    python tests/golden/make_decomposition.py [--ref <reference root>]
"""
from __future__ import annotations

import argparse
import ast
import math
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "chans-hipims-flamegpu_b200"))

from hipims_b200 import scenarios as S  # noqa: E402
from hipims_b200.topology import boundary_codes  # noqa: E402
from oracle.build_ref import DEFAULT_REF  # noqa: E402

SIZES = (2, 3, 4)


def ragged_mask(seed: int, frac: float, ny: int = 70, nx: int = 55) -> np.ndarray:
    """A ragged catchment: smoothed noise thresholded into no-data (a fraction
    `frac` of the cells), a ring."""
    rng = np.random.default_rng(seed)
    noise = rng.uniform(size=(ny + 2, nx + 2))
    for _ in range(3):
        noise = (noise + np.roll(noise, 1, 0) + np.roll(noise, -1, 0) + np.roll(noise, 1, 1) +
                 np.roll(noise, -1, 1)) / 5.0
    nodata = noise < np.quantile(noise, frac)
    nodata[0, :] = nodata[-1, :] = nodata[:, 0] = nodata[:, -1] = True
    return boundary_codes(nodata, default_bc=50)


def masks() -> list:
    out = [np.asarray(S.urban_catchment(n, dx=2.0, seed=seed)["mask"])
           for n, seed in ((120, 5), (97, 1), (64, 11))]
    # with no-data codes counted (they are nonzero), the last split of many
    # ranks over a mostly-no-data raster indexes past the valid cells: the
    # reference raises IndexError there, and so must the restatement
    return out + [ragged_mask(1, 0.1), ragged_mask(2, 0.15), ragged_mask(3, 0.3)]


def reference_functions(ref_root: str) -> dict:
    path = os.path.join(ref_root, "CHANS-HiPIMS", "hipims", "pythonHipims",
                        "MultiGPU_CatchFlood_main.py")
    tree = ast.parse(open(path).read())
    ns = {"np": np, "torch": torch, "math": math}
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and node.name in ("ave_loadStep", "ave_overlapMask"):
            exec(compile(ast.Module(body=[node], type_ignores=[]), path, "exec"), ns)
    return ns


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=DEFAULT_REF)
    args = ap.parse_args()
    fn = reference_functions(args.ref)
    arrays = {}
    k = 0
    for m in masks():
        mask = torch.as_tensor(m)
        for size in SIZES:
            arrays[f"mask_{k}"] = m.astype(np.int32)
            arrays[f"size_{k}"] = np.int32(size)
            try:
                splits = np.asarray(fn["ave_loadStep"](mask, size), dtype=np.int32)
                overlap = fn["ave_overlapMask"](mask, 0, size).numpy().astype(np.int32)
            except IndexError:
                splits = overlap = np.zeros(0, dtype=np.int32)
                arrays[f"raises_{k}"] = np.int32(1)
            arrays[f"splits_{k}"] = splits
            arrays[f"overlap_{k}"] = overlap
            k += 1
    np.savez_compressed(os.path.join(HERE, "multigpu", "decomposition.npz"), n_cases=np.int32(k),
                        **arrays)
    print(f"wrote {k} cases")


if __name__ == "__main__":
    main()
