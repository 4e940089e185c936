"""Python front end of the CPU oracle.

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU
baseline legs use it as the checker / timed baseline.  Nothing in the product
package imports it.

Two CPU back ends share one step driver (or_godunov_step in hipims_oracle.c,
the reference's step order of HP/SWE_CUDA.py:339-424, 497-502, 780-831):
  * the restatement (libhipims_oracle.so, built by oracle/Makefile), and
  * the reference's own kernels compiled for the host (_ref/libhipims_ref_host.so,
    built by oracle/build_ref.py when the reference tree is available).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libhipims_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libhipims_ref_host.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_L = ctypes.c_int64
_D = ctypes.c_double


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "hipims_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE, "libhipims_oracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return LIB


_lib = None
_ref = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.or_flux.argtypes = [_I, _L, _L, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I,
                              _I, _P, _I, _I, _P, _I, _I, _D, _D, _D]
        L.or_friction_update.argtypes = [_L, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D]
        L.or_timestep.argtypes = [_L, _P, _P, _P, _P, _P, _P, _D, _D]
        L.or_rain_station.argtypes = [_L, _P, _P, _P, _D]
        L.or_flux_mask.argtypes = [_L, _P, _P, _P, _D]
        L.or_euler_update.argtypes = [_L, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        L.or_infiltration.argtypes = [_L, _P, _P, _P, _P, _P, _P, _P, _P, _D]
        L.or_build_index.argtypes = [_L, _L, _P, _P]
        L.or_build_index.restype = _L
        L.or_decode_bc.argtypes = [ctypes.c_int32, _P, _P]
        L.or_godunov_step.argtypes = [_P]
        L.or_godunov_run.argtypes = [_P, _L, _D]
        L.or_godunov_run.restype = _L
        L.or_godunov_sizeof.restype = ctypes.c_size_t
        L.or_set_threads.argtypes = [_I]
        L.or_get_threads.restype = _I
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(f"{REF_LIB} not built (python oracle/build_ref.py)")
        _ref = ctypes.CDLL(REF_LIB)
    return _ref


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


def get_threads() -> int:
    return int(lib().or_get_threads())


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


# ----------------------------------------------------------------- kernels
def build_index(mask: np.ndarray) -> np.ndarray:
    m = np.ascontiguousarray(mask, dtype=np.int32)
    n = lib().or_build_index(m.shape[0], m.shape[1], _p(m), None)
    idx = np.empty(5 * n, dtype=np.int32)
    lib().or_build_index(m.shape[0], m.shape[1], _p(m), _p(idx))
    return idx


def decode_bc(code: int) -> tuple[int, int]:
    t, i = ctypes.c_int32(), ctypes.c_int32()
    lib().or_decode_bc(int(code), ctypes.byref(t), ctypes.byref(i))
    return t.value, i.value


def flux(order, wet, hf, qxf, qyf, h, wl, z, qx, qy, index, normal, gd, gw, gq, dx, t, dt):
    gd, gw, gq = (np.atleast_2d(np.ascontiguousarray(a, dtype=np.float64)) for a in (gd, gw, gq))
    lib().or_flux(order, len(wet), len(h), _p(wet), _p(hf), _p(qxf), _p(qyf), _p(h), _p(wl),
                  _p(z), _p(qx), _p(qy), _p(index), _p(normal), _p(gd), gd.shape[0],
                  gd.shape[1], _p(gw), gw.shape[0], gw.shape[1], _p(gq), gq.shape[0],
                  gq.shape[1], float(dx), float(t), float(dt))


def friction_update(wet, hu, qxu, qyu, zu, landuse, h, wl, qx, qy, z, manning, dt):
    lib().or_friction_update(len(wet), _p(wet), _p(hu), _p(qxu), _p(qyu), _p(zu), _p(landuse),
                             _p(h), _p(wl), _p(qx), _p(qy), _p(z), _p(manning), float(dt))


def timestep(wet, accel, h_max, h, qx, qy, dx, cfl):
    lib().or_timestep(len(wet), _p(wet), _p(accel), _p(h_max), _p(h), _p(qx), _p(qy),
                      float(dx), float(cfl))


def rain_station(hu, mask, data, dt):
    lib().or_rain_station(len(hu), _p(hu), _p(mask), _p(data), float(dt))


def flux_mask(out, h, index, t):
    lib().or_flux_mask(len(h), _p(out), _p(h), _p(index), float(t))


def euler_update(lst, hu, qxu, qyu, zu, h, wl, z, qx, qy):
    lib().or_euler_update(len(lst), _p(lst), _p(hu), _p(qxu), _p(qyu), _p(zu), _p(h), _p(wl),
                          _p(z), _p(qx), _p(qy))


def infiltration(wet, hu, landuse, h, ks, psi, dth, cum, dt):
    lib().or_infiltration(len(wet), _p(wet), _p(hu), _p(landuse), _p(h), _p(ks), _p(psi),
                          _p(dth), _p(cum), float(dt))


# ------------------------------------------------------------------ driver
class _RefKernels(ctypes.Structure):
    _fields_ = [("flux2", _P), ("flux1", _P), ("friction", _P), ("timestep", _P),
                ("rain", _P), ("mask", _P), ("infil", _P)]


class _Godunov(ctypes.Structure):
    _fields_ = [
        ("N", _L), ("order", _I), ("dx", _D), ("cfl", _D), ("export_step", _D),
        ("export_n", _I), ("t", _D), ("dt", _D),
        ("h", _P), ("wl", _P), ("qx", _P), ("qy", _P), ("z", _P), ("h_max", _P),
        ("h_upd", _P), ("qx_upd", _P), ("qy_upd", _P), ("z_upd", _P),
        ("index", _P), ("landuse", _P), ("manning", _P), ("normal", _P),
        ("given_depth", _P), ("depth_rows", _I), ("depth_cols", _I),
        ("given_wl", _P), ("wl_rows", _I), ("wl_cols", _I),
        ("given_q", _P), ("q_rows", _I), ("q_cols", _I),
        ("rain", _P), ("rain_rows", _I), ("rain_cols", _I),
        ("rain_mask", _P), ("rain_index", _I), ("rain_rate", _P), ("exports", _I),
        ("list", _P), ("fmask", _P), ("accel", _P), ("ref", _P),
        ("ks", _P), ("psi", _P), ("dtheta", _P), ("cum", _P),
    ]


class Sim:
    """FP64 CPU run of the reference step on raster inputs.

    d: dict with mask, z, h, qx, qy, (wl), landuse, manning, dx, cfl, first_dt
    and optional rain [T, 1+S], rain_mask raster, given_depth/given_wl/given_q,
    export_step, t0, infiltration = {"ks", "psi", "dtheta": per-zone lists,
    "cum": optional initial cumulative depth raster}.  backend: "oracle"
    (restatement) or "ref" (the reference kernels built for the host).
    """

    def __init__(self, d: dict, order: int = 2, backend: str = "oracle",
                 export_step: float | None = None):
        L = lib()
        if ctypes.sizeof(_Godunov) != L.or_godunov_sizeof():
            raise RuntimeError("oracle record layout mismatch")
        mask = np.asarray(d["mask"])
        valid = mask > 0
        self.valid = valid
        f64 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64)[valid])
        self.h = f64(d["h"])
        self.qx = f64(d["qx"]) if d.get("qx") is not None else np.zeros_like(self.h)
        self.qy = f64(d["qy"]) if d.get("qy") is not None else np.zeros_like(self.h)
        self.z = f64(d["z"])
        self.wl = f64(d["wl"]) if d.get("wl") is not None else self.z + self.h
        self.h_max = self.h.copy()
        N = len(self.h)
        self.N = N
        self.h_upd, self.qx_upd, self.qy_upd, self.z_upd = (np.zeros(N) for _ in range(4))
        self.index = build_index(np.where(valid, mask, -9999).astype(np.int32))
        lu = d.get("landuse")
        self.landuse = (np.zeros(N, np.uint8) if lu is None else
                        np.ascontiguousarray(np.asarray(lu)[valid].astype(np.uint8)))
        self.manning = np.ascontiguousarray(np.atleast_1d(np.asarray(d["manning"], np.float64)))
        self.normal = np.array([1.0, 0.0, 0.0, 1.0, -1.0, 0.0, 0.0, -1.0])
        tab = lambda a, w: np.ascontiguousarray(
            np.atleast_2d(np.asarray(a if a is not None else np.zeros((1, w)), np.float64)))
        self.gd = tab(d.get("given_depth"), 2)
        self.gw = tab(d.get("given_wl"), 2)
        self.gq = tab(d.get("given_q"), 3)
        self.rain = None if d.get("rain") is None else tab(d["rain"], 2)
        rm = d.get("rain_mask")
        self.rain_mask = None if rm is None else np.ascontiguousarray(
            np.asarray(rm)[valid].astype(np.int16))
        ncols = self.rain.shape[1] if self.rain is not None else 2
        self.rain_rate = np.zeros(ncols - 1)
        self.list = np.zeros(N, np.int32)
        self.fmask = np.zeros(N, np.uint8)
        self.accel = np.zeros(N)
        g = _Godunov()
        g.N, g.order = N, order
        g.dx, g.cfl = float(d["dx"]), float(d["cfl"])
        es = export_step if export_step is not None else d.get("export_step", 1.0e30)
        g.export_step = float(es)
        g.t, g.dt = float(d.get("t0", 0.0)), float(d["first_dt"])
        for name in ("h", "wl", "qx", "qy", "z", "h_max", "h_upd", "qx_upd", "qy_upd", "z_upd",
                     "index", "landuse", "manning", "normal", "list", "fmask", "accel",
                     "rain_rate"):
            setattr(g, name, getattr(self, name).ctypes.data)
        g.given_depth, (g.depth_rows, g.depth_cols) = self.gd.ctypes.data, self.gd.shape
        g.given_wl, (g.wl_rows, g.wl_cols) = self.gw.ctypes.data, self.gw.shape
        g.given_q, (g.q_rows, g.q_cols) = self.gq.ctypes.data, self.gq.shape
        if self.rain is not None:
            g.rain, (g.rain_rows, g.rain_cols) = self.rain.ctypes.data, self.rain.shape
        g.rain_mask = _p(self.rain_mask)
        inf = d.get("infiltration")
        self.cum = None
        if inf is not None:
            par = lambda a: np.ascontiguousarray(np.atleast_1d(np.asarray(a, np.float64)))
            self.ks, self.psi, self.dtheta = par(inf["ks"]), par(inf["psi"]), par(inf["dtheta"])
            self.cum = (np.zeros(N) if inf.get("cum") is None else f64(inf["cum"])).copy()
            g.ks, g.psi, g.dtheta = (self.ks.ctypes.data, self.psi.ctypes.data,
                                     self.dtheta.ctypes.data)
            g.cum = self.cum.ctypes.data
        self._kern = None
        if backend == "ref":
            R = ref_lib()
            k = _RefKernels()
            for f, sym in (("flux2", "ref_flux2"), ("flux1", "ref_flux1"),
                           ("friction", "ref_friction_update"), ("timestep", "ref_timestep"),
                           ("rain", "ref_rain_station"), ("mask", "ref_flux_mask"),
                           ("infil", "ref_infiltration")):
                setattr(k, f, ctypes.cast(getattr(R, sym), _P).value)
            self._kern = k
            g.ref = ctypes.addressof(k)
        elif backend != "oracle":
            raise ValueError(backend)
        self.g = g

    @property
    def t(self) -> float:
        return self.g.t

    @property
    def dt(self) -> float:
        return self.g.dt

    _steps = 0

    def step(self, n: int = 1) -> None:
        for _ in range(n):
            lib().or_godunov_step(ctypes.byref(self.g))
        self._steps += n

    def run(self, n: int, t_end: float = float("inf")) -> int:
        k = int(lib().or_godunov_run(ctypes.byref(self.g), int(n), float(t_end)))
        self._steps += k
        return k

    def run_record(self, n: int, t_end: float = float("inf")) -> np.ndarray:
        """Step n times (or to t_end); return the dt chosen after each step."""
        dts = []
        for _ in range(n):
            if not self.g.t < t_end:
                break
            lib().or_godunov_step(ctypes.byref(self.g))
            self._steps += 1
            dts.append(self.g.dt)
        return np.asarray(dts)

    def state(self) -> dict:
        st = dict(h=self.h.copy(), qx=self.qx.copy(), qy=self.qy.copy(), wl=self.wl.copy(),
                  h_max=self.h_max.copy(), t=self.g.t, dt=self.g.dt)
        if self.cum is not None:
            st["cum"] = self.cum.copy()
        return st
