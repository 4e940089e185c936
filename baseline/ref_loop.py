"""Run the reference's own solver class, unmodified, on a chosen set of op
modules.

BENCHMARK AND TEST INFRASTRUCTURE ONLY.  HP/SWE_CUDA.py imports its 13 torch
extension modules by bare name at module load (HP/SWE_CUDA.py:29-41) and calls
them positionally (:339-424, 497-502, 780-831).  `load_swe_cuda(modules)`
executes the staged copy of that file (baseline/install_ref_py.py) as a fresh
module while sys.modules maps those 13 names to the given module objects, then
restores sys.modules, so one process can hold the reference class bound to
this library's drop-in modules (`b200_modules()`) and, separately, bound to
the reference's own kernels built for sm_100a (`reference_kernel_modules()`,
the plain FP64 GPU baseline).  `load_parallel_swe(modules)` does the same
for the reference's multi-GPU subclass (HP/Parallel_SWE_CUDA.py), with its
`SWE_CUDA` import resolved to the module load_swe_cuda made.  Nothing in the
reference files is changed.
"""
from __future__ import annotations

import importlib
import importlib.util
import itertools
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "chans-hipims-flamegpu_b200")
REF_PY = os.path.join(HERE, "_ref", "pythonHipims")

# the extension modules HP/SWE_CUDA.py imports at load (HP/SWE_CUDA.py:29-41)
OP_MODULES = ("frictionCalculation", "timeControl", "euler_update", "infiltrationCalculation",
              "station_PrecipitationCalculation", "frictionCalculation_implicit",
              "friction_implicit_andUpdate_jh", "fluxMask", "fluxCalculation_jh_modified_surface",
              "fluxCal_2ndOrder_jh_improved", "sedi_mass_momentum_update", "sedi_c_euler_update",
              "fluxCalculation_convectionTranport")

_count = itertools.count()


def available() -> bool:
    return os.path.isfile(os.path.join(REF_PY, "SWE_CUDA.py"))


def b200_modules() -> dict:
    """This library's drop-in modules (chans-hipims-flamegpu_b200/<name>.py)."""
    if PKG not in sys.path:
        sys.path.insert(0, PKG)
    return {name: importlib.import_module(name) for name in OP_MODULES}


def reference_kernel_modules() -> dict:
    """Modules of the same names whose ops are the reference's own kernels
    built for sm_100a (baseline/build_ref_cuda.py, bound by baseline.ref_gpu)."""
    from baseline import ref_gpu

    ops = ref_gpu.RefGpuOps()

    def unbound(name):
        def f(*args, **kwargs):
            raise NotImplementedError(f"{name} is not bound to the reference kernels here")
        return f

    table = {
        "fluxCal_2ndOrder_jh_improved": {"addFlux": ops.flux_2nd_order},
        "fluxCalculation_jh_modified_surface": {"addFlux": ops.flux_1st_order},
        "friction_implicit_andUpdate_jh": {"addFriction_eulerUpdate": ops.friction_update},
        "timeControl": {"updateTimestep": ops.update_timestep},
        "station_PrecipitationCalculation": {"addStation_Precipitation": ops.station_rain},
        "fluxMask": {"update": ops.flux_mask},
        "euler_update": {"update": unbound("euler_update.update")},
        "infiltrationCalculation": {"addinfiltration": unbound("infiltrationCalculation")},
    }
    out = {}
    for name in OP_MODULES:
        m = types.ModuleType(name)
        for attr, fn in table.get(name, {}).items():
            setattr(m, attr, fn)
        out[name] = m
    return out


def load_swe_cuda(modules: dict) -> types.ModuleType:
    """The reference's SWE_CUDA module, executed with `modules` standing in
    for its 13 extension imports."""
    path = os.path.join(REF_PY, "SWE_CUDA.py")
    if not os.path.isfile(path):
        raise FileNotFoundError(f"{path} is not staged (python baseline/install_ref_py.py)")
    saved = {k: sys.modules.get(k) for k in OP_MODULES}
    sys.modules.update({k: modules[k] for k in OP_MODULES})
    try:
        spec = importlib.util.spec_from_file_location(f"_ref_SWE_CUDA_{next(_count)}", path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    return mod


def load_parallel_swe(modules: dict) -> types.ModuleType:
    """The reference's Parallel_SWE_CUDA module (class Parallel_SWE), executed
    with `SWE_CUDA` and the op modules it imports by bare name
    (HP/Parallel_SWE_CUDA.py:16-26) resolved to load_swe_cuda(modules) and
    `modules`."""
    path = os.path.join(REF_PY, "Parallel_SWE_CUDA.py")
    if not os.path.isfile(path):
        raise FileNotFoundError(f"{path} is not staged (python baseline/install_ref_py.py)")
    swe = load_swe_cuda(modules)
    names = OP_MODULES + ("SWE_CUDA",)
    saved = {k: sys.modules.get(k) for k in names}
    sys.modules.update({k: modules[k] for k in OP_MODULES})
    sys.modules["SWE_CUDA"] = swe
    try:
        spec = importlib.util.spec_from_file_location(f"_ref_Parallel_SWE_CUDA_{next(_count)}",
                                                      path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    return mod


# --- ranks of the reference's multi-GPU subclass (HP/Parallel_SWE_CUDA.py) --
# Its driver, HP/MultiGPU_CatchFlood_main.py, splits the raster into row
# strips with two overlap rows each side and exchanges the overlap cells with
# SUM all_reduces and the time step with a MIN all_reduce.  The functions
# below restate that decomposition (pinned to the driver's own functions by
# tests/golden/multigpu/decomposition.npz); run_parallel_loop runs the ranks in
# one process and carries each collective out by its definition (every rank's
# tensor replaced, in place, by the sum or minimum over ranks).

def row_splits(mask, size):
    """Split rows of MultiGPU_CatchFlood_main.py:59-70: for k = 1 .. size-1,
    one row above the row of the valid cell at position floor(k / size * n)
    in row-major order, n the number of NONZERO codes (no-data codes such as
    -9999 included, as there)."""
    m = np.asarray(mask)
    rows = np.nonzero(m > 0)[0]
    n = np.count_nonzero(m)
    return [int(rows[int(float(k) / float(size) * float(n))]) - 1 for k in range(1, size)]


def rank_rows(splits, rank, size, n_rows):
    """Raster rows of a rank, its two overlap rows included (:139-146)."""
    if rank == 0:
        return 0, splits[0] + 2
    if rank == size - 1:
        return splits[-1] - 2, n_rows
    return splits[rank - 1] - 2, splits[rank] + 2


def overlap_mask(mask, splits, size):
    """Segment id of every overlap value (:113-136): rank i's rows below its
    upper split and above its lower split, two rows each."""
    v = np.asarray(mask) > 0
    ids = []
    for i in range(size):
        if i > 0:
            ids += [2 * i - 1] * int(v[splits[i - 1] - 2:splits[i - 1]].sum())
        if i < size - 1:
            ids += [2 * i] * int(v[splits[i]:splits[i] + 2].sum())
    return torch.tensor(ids, dtype=torch.int32)


_OVERLAPS = ("get_h_overlap", "get_wl_overlap", "get_z_overlap", "get_qx_overlap",
             "get_qy_overlap")


def run_parallel_loop(PSWE, d, dev, steps, size=2):
    """Ranks of the reference's Parallel_SWE class PSWE stepping the loop of
    MultiGPU_CatchFlood_main.py:374-410 (without the infiltration source) on
    catchment d (rasters and settings as tests/golden cases hold them), in
    FP64 and 1st order (the class builds the 1st-order neighbour table only,
    HP/Parallel_SWE_CUDA.py:241-265).  Returns the ranks and the splits."""
    mask = np.asarray(d["mask"])
    splits = row_splits(mask, size)
    overlap = overlap_mask(mask, splits, size)
    wl_full = np.asarray(d["z"]) + np.asarray(d["h"])
    rm = d.get("rain_mask")
    rm = np.zeros(mask.shape, np.int16) if rm is None else np.asarray(rm)
    ranks = []
    for r in range(size):
        a, b = rank_rows(splits, r, size, mask.shape[0])
        g = PSWE(dev, d["dx"], d["cfl"], 1e30, r, size, secondOrder=False,
                 firstTimeStep=d["first_dt"], tensorType=torch.float64)
        cut = lambda x: torch.as_tensor(np.asarray(x, dtype=np.float64)[a:b])
        mk = torch.as_tensor(mask[a:b])
        g.init__fluidField_tensor(mk, overlap, cut(d["h"]), cut(d["qx"]), cut(d["qy"]),
                                  cut(wl_full), cut(d["z"]), dev)
        g.set__frictionField_tensor(torch.as_tensor(np.atleast_1d(d["manning"]), device=dev), dev)
        if d.get("landuse") is not None:
            g.set_landuse_cpu_to_gpu(mk, torch.as_tensor(np.asarray(d["landuse"])[a:b]), dev)
        g.set_distributed_rainfall_station_Mask_cpu_to_gpu(mk, torch.as_tensor(rm[a:b]), dev)
        ranks.append(g)

    def exchange():
        for g in ranks:
            g.update_overlap_send()
        for get in _OVERLAPS:
            ts = [getattr(g, get)() for g in ranks]
            total = ts[0].clone()
            for t in ts[1:]:
                total += t
            for t in ts:
                t.copy_(total)

    rain = d.get("rain")
    rain = np.array([[0.0, 0.0], [1e9, 0.0]]) if rain is None else np.asarray(rain)
    exchange()
    for _ in range(steps):
        for g in ranks:
            g.update_overlap_receive()
            g.addFlux()
            g.addStation_PrecipitationSource(rain, dev)
            g.time_friction_euler_update_cuda(dev)
        dt = torch.stack([g.dt.reshape(()) for g in ranks]).min()
        for g in ranks:
            g.dt.copy_(dt.reshape(g.dt.shape))
        exchange()
        for g in ranks:
            g.timeAddStep()
    return ranks, splits
