"""The Godunov API's other step paths on the GPU compat ops against the
oracle's kernels composed the same way: RK2 with uniform rain
(HP/SWE_CUDA.py:870-892, 517-549) and the frictionless Euler update with its
own time control (HP/SWE_CUDA.py:712-764, used by the multi-GPU solver)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

NORMAL = np.array([1.0, 0.0, 0.0, 1.0, -1.0, 0.0, 0.0, -1.0])
DEFAULT_TABLES = (np.zeros((1, 2)), np.zeros((1, 2)), np.zeros((1, 3)))


class OracleState:
    """Compacted FP64 state and the reference's per-op sequence on the CPU."""

    def __init__(self, d):
        valid = np.asarray(d["mask"]) > 0
        c = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64)[valid])
        self.h, self.qx, self.qy, self.z = c(d["h"]), c(d["qx"]), c(d["qy"]), c(d["z"])
        self.wl = self.z + self.h
        self.h_max = self.h.copy()
        n = len(self.h)
        self.hu, self.qxu, self.qyu, self.zu = (np.zeros(n) for _ in range(4))
        self.index = O.build_index(np.where(valid, d["mask"], -9999).astype(np.int32))
        self.landuse = np.ascontiguousarray(np.asarray(d["landuse"])[valid].astype(np.uint8))
        self.manning = np.ascontiguousarray(np.atleast_1d(np.asarray(d["manning"], np.float64)))
        self.dx, self.cfl = float(d["dx"]), float(d["cfl"])
        self.t, self.dt = 0.0, float(d["first_dt"])

    def flux(self):
        fm = np.zeros(len(self.h), np.uint8)
        O.flux_mask(fm, self.h, self.index, self.t)
        wet = np.flatnonzero(fm).astype(np.int32)
        O.flux(2, wet, self.hu, self.qxu, self.qyu, self.h, self.wl, self.z, self.qx, self.qy,
               self.index, NORMAL, *DEFAULT_TABLES, self.dx, self.t, self.dt)

    def friction(self):
        lst = np.flatnonzero((np.abs(self.hu) > 0) | (self.h >= 0)).astype(np.int32)
        O.friction_update(lst, self.hu, self.qxu, self.qyu, self.zu, self.landuse, self.h,
                          self.wl, self.qx, self.qy, self.z, self.manning, self.dt)
        for a in (self.hu, self.qxu, self.qyu, self.zu):
            a[:] = 0.0

    def rk2(self, rate):
        h0, qx0, qy0 = self.h.copy(), self.qx.copy(), self.qy.copy()
        for _ in range(2):
            self.flux()
            self.hu += rate * self.dt
            self.friction()
        self.h[:] = (self.h + h0) / 2.0
        self.qx[:] = (self.qx + qx0) / 2.0
        self.qy[:] = (self.qy + qy0) / 2.0
        self.wl[:] = self.h + self.z

    def euler_and_time(self):
        self.flux()
        lst = np.flatnonzero((np.abs(self.hu) > 0) | (self.h > 1e-6)).astype(np.int32)
        O.euler_update(lst, self.hu, self.qxu, self.qyu, self.zu, self.h, self.wl, self.z,
                       self.qx, self.qy)
        for a in (self.hu, self.qxu, self.qyu, self.zu):
            a[:] = 0.0
        upper = self.dt * 10.0
        wet = np.flatnonzero(self.h > 1e-6).astype(np.int32)
        acc = np.full(len(wet), 60.0)
        O.timestep(wet, acc, self.h_max, self.h, self.qx, self.qy, self.dx, self.cfl)
        dt = acc.min() if len(wet) else self.dt
        self.dt = min(dt, upper)
        self.t += self.dt


def godunov(d, dev):
    from hipims_b200.solver import Godunov

    g = Godunov(dev, d["dx"], d["cfl"], 1e30, secondOrder=True, firstTimeStep=d["first_dt"],
                tensorType=torch.float64)
    g._export_enabled = False
    T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64))
    mask = torch.as_tensor(np.asarray(d["mask"]))
    g.init__fluidField_tensor(mask, T(d["h"]), T(d["qx"]), T(d["qy"]),
                              T(np.asarray(d["z"]) + np.asarray(d["h"])), T(d["z"]), dev)
    g.set__frictionField_tensor(torch.as_tensor(np.atleast_1d(d["manning"]), device=dev), dev)
    g.set_landuse(mask, torch.as_tensor(np.asarray(d["landuse"])), dev)
    return g


def test_rk2_uniform_rain_matches_oracle(cuda):
    from hipims_b200 import scenarios as S

    d = S.dam_break(48)
    rain = np.array([[0.0, 2e-4], [100.0, 2e-4]])
    ref = OracleState(d)
    g = godunov(d, cuda)
    for _ in range(5):
        ref.rk2(2e-4)
        g.rungeKutta_update(rain, cuda)
    for k, x in (("h", g._h_internal), ("qx", g._qx_internal), ("qy", g._qy_internal)):
        np.testing.assert_allclose(x.cpu().numpy(), getattr(ref, k), rtol=0, atol=1e-12,
                                   err_msg=k)


def test_euler_update_and_time_control_match_oracle(cuda):
    from hipims_b200 import scenarios as S

    d = S.dam_break(48)
    ref = OracleState(d)
    g = godunov(d, cuda)
    for _ in range(40):
        ref.euler_and_time()
        g.addFlux()
        g.euler_update()
        g.time_update_cuda(cuda)
    assert g.t.item() == pytest.approx(ref.t, rel=1e-12)
    for k, x in (("h", g._h_internal), ("qx", g._qx_internal), ("qy", g._qy_internal),
                 ("h_max", g._h_max)):
        np.testing.assert_allclose(x.cpu().numpy(), getattr(ref, k), rtol=0, atol=1e-10,
                                   err_msg=k)
