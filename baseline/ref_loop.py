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
the plain FP64 GPU baseline).  Nothing in the reference file is changed.
"""
from __future__ import annotations

import importlib
import importlib.util
import itertools
import os
import sys
import types

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
