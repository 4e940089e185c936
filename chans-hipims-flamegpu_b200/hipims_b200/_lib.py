"""ctypes loader of libhipims_b200.so and mirrors of its C records.

The library is the only compute path: if it is missing or fails to load, every
op raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libhipims_b200.so")
REPO_ROOT = os.path.dirname(PKG_DIR)
HEADER_PATHS = [
    os.path.join(REPO_ROOT, "include", "hipims_b200.h"),
    os.path.join(REPO_ROOT, "include", "hipims_b200_fused.h"),
]

HB_F32 = 0
HB_F64 = 1
HB_MAX_CLASSES = 16
HB_NODATA_CLASS = 15
HB_MAX_ZONES = 16
HB_DATUM_BLOCK = 64
HB_PAD_Y = 2
HB_PAD_X = 4
HB_CODE_PAD_X = 16

c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
c_vp = ctypes.c_void_p
c_dbl = ctypes.c_double


class HbCtrl(ctypes.Structure):
    _fields_ = [
        ("t", c_dbl), ("dt", c_dbl), ("export_step", c_dbl), ("t_end", c_dbl),
        ("volume", c_dbl), ("volume0", c_dbl), ("rain_volume", c_dbl),
        ("outflow_volume", c_dbl), ("rain_rate", c_dbl), ("rain_mult", c_dbl),
        ("step", c_i64),
        ("export_n", c_i32), ("cur", c_i32), ("halted", c_i32), ("halt_on_export", c_i32),
        ("exports", c_i32), ("rain_index", c_i32), ("tiles_done", ctypes.c_uint32),
        ("status", c_i32),
        ("bc_vals", (ctypes.c_float * 4) * HB_MAX_CLASSES),
        ("external_dt", c_i32), ("pad1", c_i32), ("ext", c_dbl * 2),
    ]


class HbInstance(ctypes.Structure):
    _fields_ = [
        ("rows", c_i32), ("cols", c_i32), ("tiles_x", c_i32), ("tiles_y", c_i32),
        ("tile_begin", c_i32), ("pitch", c_i32), ("code_pitch", c_i32),
        ("datum_nx", c_i32), ("datum_ny", c_i32), ("bug_y", c_i32), ("bug_x", c_i32),
        ("rain_rows", c_i32), ("rain_cols", c_i32), ("depth_rows", c_i32),
        ("depth_cols", c_i32), ("wl_rows", c_i32), ("wl_cols", c_i32), ("q_rows", c_i32),
        ("q_cols", c_i32), ("pad0", c_i32),
        ("h", c_vp * 2), ("qx", c_vp * 2), ("qy", c_vp * 2), ("z", c_vp), ("h_max", c_vp),
        ("code", c_vp), ("datum", c_vp), ("ctrl", c_vp), ("rain_tab", c_vp),
        ("given_depth", c_vp), ("given_wl", c_vp), ("given_q", c_vp),
        ("dx", c_dbl), ("cfl", c_dbl),
        ("manning", c_dbl * HB_MAX_ZONES),
        ("bc_type", c_i32 * HB_MAX_CLASSES), ("bc_id", c_i32 * HB_MAX_CLASSES),
        ("n_valid", c_i64),
        ("dt_replay", c_vp), ("n_replay", c_i64),
        ("cum", c_vp), ("ks", c_dbl * HB_MAX_ZONES), ("psi", c_dbl * HB_MAX_ZONES),
        ("dtheta", c_dbl * HB_MAX_ZONES),
        ("rain_station", c_vp), ("station_rate", c_vp), ("station_cells", c_vp),
        ("n_stations", c_i32), ("pad2", c_i32),
        ("halo_up", c_vp * 6), ("halo_down", c_vp * 6), ("halo_up_rows", c_i32), ("pad3", c_i32),
    ]


class HbFusedBatch(ctypes.Structure):
    _fields_ = [
        ("dtype", c_i32), ("n_instances", c_i32), ("n_tiles", c_i32), ("tile_y", c_i32),
        ("tile_x", c_i32), ("grid_blocks", c_i32), ("order", c_i32), ("flags", c_i32),
        ("instances", c_vp), ("tile_instance", c_vp), ("workspace", c_vp),
        ("instances_host", c_vp),
    ]


# name -> (restype, argtypes)
_I, _P, _L = c_i32, c_vp, c_i64
class HbAdjointArgs(ctypes.Structure):
    """Mirror of hb_adjoint_args (include/hipims_b200.h)."""
    _fields_ = [
        ("instance", c_vp), ("rows", c_i32), ("cols", c_i32), ("pitch", c_i32),
        ("code_pitch", c_i32),
        ("h", c_vp), ("qx", c_vp), ("qy", c_vp),
        ("lam_h", c_vp), ("lam_qx", c_vp), ("lam_qy", c_vp),
        ("out_h", c_vp), ("out_qx", c_vp), ("out_qy", c_vp),
        ("mu", c_vp), ("mu_stride", c_i64), ("grad", c_vp),
        ("t", c_dbl), ("dt", c_dbl), ("rain_rate", c_dbl), ("rain_base", c_dbl),
        ("h_reg", c_dbl), ("first", c_i32), ("pad", c_i32),
        ("faces", c_vp), ("face_stride", c_i64),
    ]


SIGNATURES = {
    "hb_abi_version": (_I, []),
    "hb_last_error": (ctypes.c_char_p, []),
    "hb_record_sizes": (None, [ctypes.POINTER(ctypes.c_size_t)]),
    "hb_flux_mask": (_I, [_I, _L, _P, _P, _P, _P, _P]),
    "hb_flux": (_I, [_I, _I, _L, _L, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I,
                     _P, _I, _I, _P, _I, _I, _P, _P, _P, _P]),
    "hb_friction_update": (_I, [_I, _L, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                _P]),
    "hb_timestep": (_I, [_I, _L, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "hb_rain_station": (_I, [_I, _L, _P, _P, _P, _P, _P]),
    "hb_euler_update": (_I, [_I, _L, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "hb_infiltration": (_I, [_I, _L, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "hb_min_reduce_workspace_size": (ctypes.c_size_t, [_L]),
    "hb_min_reduce": (_I, [_I, _L, _P, _P, _P, _P]),
    "hb_fused_workspace_size": (ctypes.c_size_t, [_P]),
    "hb_fused_prepare": (_I, [_P, _P]),
    "hb_fused_step": (_I, [_P, _I, _P]),
    "hb_fused_run": (_I, [_P, _I, ctypes.c_longlong, _P]),
    "hb_fused_step_noalloc": (_I, [_P, _I, _I, _P]),
    "hb_fused_finish": (_I, [_P, _P, _P]),
    "hb_adjoint_step": (_I, [_P, _P]),
    "hb_adjoint_gauge": (_I, [_L, _P, _P, _P, _P, ctypes.c_double, _P]),
    "hb_gather": (_I, [_I, _L, _P, _P, _P, _P, _P, _P, _P, _P]),
    "hb_state_layout": (_I, [_I, _L, _P, _I, _P, _P, _P, _P, _P, _P, _P]),
}

_lock = threading.Lock()
_lib = None


def lib() -> ctypes.CDLL:
    """Load libhipims_b200.so once; raise if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is not built; run `python chans-hipims-flamegpu_b200/build.py`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        sizes = (ctypes.c_size_t * 3)()
        L.hb_record_sizes(sizes)
        want = (ctypes.sizeof(HbCtrl), ctypes.sizeof(HbInstance), ctypes.sizeof(HbFusedBatch))
        if tuple(sizes) != want:
            raise RuntimeError(f"record layout mismatch: library {tuple(sizes)} vs ctypes {want}")
        _lib = L
        return _lib


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        msg = lib().hb_last_error().decode(errors="replace")
        raise RuntimeError(f"{what or 'hipims_b200'} failed ({rc}): {msg}")


def declared_symbols() -> list[str]:
    """Function names declared in include/*.h (for the export test)."""
    import re

    names = []
    for p in HEADER_PATHS:
        with open(p, "r", encoding="utf-8") as f:
            text = f.read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(hb_[a-z0-9_]+)\s*\(", text):
            names.append(m.group(1))
    return sorted(set(names))
