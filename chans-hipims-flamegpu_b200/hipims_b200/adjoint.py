"""Discrete adjoint of the FP64 fused step: gradients of a gauge misfit with
respect to the Manning coefficient of every zone and the rain multiplier.

The forward is the fused FP64 solver (one ``hb_fused_step`` per step) with the
time-step schedule frozen (``Catchment.dt_replay``): the gradient is that of
the discrete map for fixed dt, which is what a central finite difference of the
same frozen-dt forward measures.  The loss is

    J = w * sum_{s, g} (h^{s * every}[gauge g] - obs[s, g])^2,

sampled after every ``every`` steps.  The reverse sweep keeps a state
checkpoint every ``checkpoint`` steps during the forward, recomputes one
segment at a time (storing its states) and runs ``hb_adjoint_step`` backwards
through it; ``hb_adjoint_gauge`` adds the misfit gradient at sampled steps.

Cells shallower than ``h_reg`` (default 1e-5 m, ten times the scheme's
wet/dry threshold h_small) carry no state adjoint.  The step never clamps
h >= 0 (as the reference), and films of a few h_small sit on bumps between
deeper cells with discharges at rounding level; there the linearised step has
gains above one per step (|dq'/dq| of 2-4 with alternating sign was measured)
that the nonlinear step saturates, so the exact adjoint through such cells
grows without bound while the loss stays smooth.  Masking them drops only the
sensitivity carried by sub-0.01 mm films; h_reg = 0 masks negative depths
only.
With ``forward_dtype=torch.float32`` the forward, its checkpoints and the
recomputed segments run in the FP32 product (the two-cells-per-lane step), and
the reverse sweep linearises the FP64 step at those FP32 states: the
gradient of the loss the FP32 run computes, to within the FP32 trajectory's
distance from FP64.  Its FP64 reference gradient is the same problem with
``forward_dtype=torch.float64``.

The reference has no adjoint; the forward it differentiates is the reference
step (HP/SWE_CUDA.py:339-424 with HC/fluxCal_2ndOrder_jh_improved_Kernel.cu,
HC/friction_implicit_andUpdate_jh_Kernel.cu and HP/SWE_CUDA.py:472-495 for rain).
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
from typing import Sequence

import numpy as np
import torch

from . import _lib
from .fused import Catchment, FusedSolver

_CTRL_DOUBLES = 10  # t, dt, export_step, t_end, volume, volume0, rain_volume, outflow, rain_rate, rain_mult


def record_schedule(catchment: Catchment, nsteps: int, device="cuda") -> np.ndarray:
    """Run the adaptive FP64 forward for nsteps and return the dt of every step
    (dt[0] is the catchment's first dt)."""
    c = dataclasses.replace(catchment, dt_replay=None, export_step=0.0, t_end=math.inf,
                            halt_on_export=False)
    fs = FusedSolver(c, dtype=torch.float64, device=device)
    ctrlf = fs.ctrl.view(torch.float64)
    log = torch.empty(nsteps, dtype=torch.float64, device=fs.device)
    for k in range(nsteps):
        log[k].copy_(ctrlf[1])
        fs.step(1)
    return log.cpu().numpy()


def _rain_base(rain: np.ndarray | None, t: float) -> float:
    """Rain rate at t without the multiplier (HP/SWE_CUDA.py:472-495: linear
    interpolation, zero from the last row on)."""
    if rain is None or len(rain) < 2:
        return 0.0
    r = np.asarray(rain, dtype=np.float64)
    if not t < r[-1, 0]:
        return 0.0
    return float(np.interp(t, r[:, 0], r[:, 1]))


class GaugeMisfit:
    """Squared gauge misfit of one catchment over ``nsteps`` frozen-dt FP64
    steps, with its gradient by the discrete adjoint.

    ``dt_schedule`` is the dt of each step (as returned by record_schedule);
    ``obs`` is [nsteps // every, n_gauges] (zeros if omitted)."""

    def __init__(self, catchment: Catchment, gauge_rows, gauge_cols, nsteps: int,
                 dt_schedule: np.ndarray, every: int = 10, checkpoint: int = 100,
                 obs=None, weight: float = 1.0, h_reg: float = 1.0e-5,
                 store_faces: bool = True, device="cuda",
                 forward_dtype: torch.dtype = torch.float64):
        dts = np.asarray(dt_schedule, dtype=np.float64)
        if dts.shape[0] < nsteps:
            raise ValueError(f"dt schedule has {dts.shape[0]} steps, {nsteps} needed")
        if every < 1 or checkpoint < 1:
            raise ValueError("every and checkpoint must be >= 1")
        if catchment.infiltration is not None or catchment.rain_station is not None:
            raise ValueError("the adjoint covers uniform rain without infiltration")
        self.catchment = dataclasses.replace(
            catchment, dt0=float(dts[0]), dt_replay=dts[1:nsteps].copy() if nsteps > 1 else
            np.zeros(1), export_step=0.0, t_end=math.inf, halt_on_export=False)
        self.nsteps, self.every, self.K = int(nsteps), int(every), int(checkpoint)
        self.weight = float(weight)
        self.h_reg = float(h_reg)
        self.store_faces = bool(store_faces)
        if forward_dtype not in (torch.float32, torch.float64):
            raise ValueError("forward_dtype must be float32 or float64")
        self.forward_dtype = forward_dtype
        self.fs = FusedSolver(self.catchment, dtype=forward_dtype, device=device)
        # the reverse sweep reads the FP64 instance record (bed, codes, tables)
        # and FP64 states on the same dense layout
        self.fs64 = self.fs if forward_dtype == torch.float64 else FusedSolver(
            self.catchment, dtype=torch.float64, device=device, origin=self.fs.inst[0].origin)
        self.device = self.fs.device
        self.n_zones = len(catchment.manning)
        self.offsets = self.fs.cell_offsets(0, np.asarray(gauge_rows), np.asarray(gauge_cols))
        self.n_gauges = int(self.offsets.numel())
        self.n_samples = self.nsteps // self.every
        if obs is None:
            obs = torch.zeros(self.n_samples, self.n_gauges, dtype=torch.float64)
        self.obs = torch.as_tensor(obs, dtype=torch.float64).to(self.device).contiguous()
        if tuple(self.obs.shape) != (self.n_samples, self.n_gauges):
            raise ValueError(f"obs must be [{self.n_samples}, {self.n_gauges}]")
        ins = self.fs.inst[0]
        self._shape = (ins.rows_s, ins.pitch)
        self._numel = ins.rows_s * ins.pitch
        self._ckpt: dict[int, tuple[torch.Tensor, torch.Tensor]] = {}
        self._h_last = None
        self.samples = None
        self._params = None

    # ----------------------------------------------------------------- forward
    def _cur(self, k: int) -> int:
        return k % 2  # reset() starts at buffer 0 and every step flips it

    def _state(self, k: int) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        ins, b = self.fs.inst[0], self._cur(k)
        return ins.h[b], ins.qx[b], ins.qy[b]

    def simulate(self, manning: Sequence[float], rain_mult: float = 1.0) -> torch.Tensor:
        """Forward run; returns the gauge samples [n_samples, n_gauges] and keeps
        the checkpoints for gradient()."""
        self._params = ([float(v) for v in manning], float(rain_mult))
        self.fs.set_manning(0, self._params[0])
        if self.fs64 is not self.fs:
            self.fs64.set_manning(0, self._params[0])
        self.fs.reset(rain_mult=self._params[1])
        samples = torch.empty(self.n_samples, self.n_gauges, dtype=torch.float64,
                              device=self.device)
        self._ckpt = {}
        events = sorted(set(range(0, self.nsteps, self.K)) |
                        set(range(self.every, self.nsteps + 1, self.every)) | {self.nsteps})
        k = 0
        for e in events:
            if e > k:
                self.fs.step(e - k)
                k = e
            if k % self.every == 0 and k > 0:
                samples[k // self.every - 1] = self._state(k)[0].view(-1)[self.offsets]
            if k % self.K == 0 and k < self.nsteps:
                h, qx, qy = self._state(k)
                self._ckpt[k] = (torch.stack([h, qx, qy]), self.fs.ctrl.clone())
        self._h_last = self._state(self.nsteps)[0].double().clone()
        self.samples = samples
        return samples

    def loss(self, samples: torch.Tensor | None = None) -> torch.Tensor:
        s = self.samples if samples is None else samples
        return self.weight * ((s - self.obs) ** 2).sum()

    # ---------------------------------------------------------------- reverse
    def gradient(self, with_state: bool = False):
        """d loss / d(manning of each zone, rain multiplier) at the parameters of
        the last simulate(); with_state=True also returns d loss / d(h, qx, qy)
        of the initial state as raster views."""
        if self._params is None:
            raise RuntimeError("simulate() first")
        L = _lib.lib()
        dev, shape, n = self.device, self._shape, self._numel
        lam = torch.zeros((3,) + shape, dtype=torch.float64, device=dev)
        out = torch.zeros_like(lam)
        mu = torch.zeros(3 * n, dtype=torch.float64, device=dev)
        grad = torch.zeros(_lib.HB_MAX_ZONES + 1, dtype=torch.float64, device=dev)
        states = torch.empty((min(self.K, self.nsteps), 3) + shape, dtype=torch.float64,
                             device=dev)
        ctrl_log = torch.empty(min(self.K, self.nsteps), _CTRL_DOUBLES, dtype=torch.float64,
                               device=dev)
        ins = self.fs64.inst[0]
        stream = torch.cuda.current_stream(dev).cuda_stream
        rain = self.catchment.rain
        w = self.weight

        def gauge(h: torch.Tensor, k: int, lam_h: torch.Tensor) -> None:
            _lib.check(L.hb_adjoint_gauge(self.n_gauges, self.offsets.data_ptr(), h.data_ptr(),
                                          self.obs[k // self.every - 1].data_ptr(),
                                          lam_h.data_ptr(), w, stream), "hb_adjoint_gauge")

        if self.nsteps % self.every == 0 and self.nsteps > 0:
            gauge(self._h_last, self.nsteps, lam[0])
        a = _lib.HbAdjointArgs()
        a.instance = self.fs64.record_ptr(0)
        a.rows, a.cols, a.pitch, a.code_pitch = ins.rows, ins.cols, ins.pitch, ins.code_pitch
        a.mu, a.mu_stride, a.grad = mu.data_ptr(), n, grad.data_ptr()
        a.h_reg = self.h_reg
        faces = None
        if self.store_faces:  # each face's forward values once per reverse step
            stride = (ins.rows + 1) * (ins.cols + 1)
            faces = torch.empty(10 * stride, dtype=torch.float64, device=dev)
            a.faces, a.face_stride = faces.data_ptr(), stride
        ctrlf = self.fs.ctrl.view(torch.float64)
        with torch.cuda.device(dev):
            for s0 in sorted(self._ckpt, reverse=True):
                s1 = min(s0 + self.K, self.nsteps)
                st, ctrl = self._ckpt[s0]
                h, qx, qy = self._state(s0)
                h.copy_(st[0])
                qx.copy_(st[1])
                qy.copy_(st[2])
                self.fs.ctrl.copy_(ctrl)
                self.fs.prepare()
                for k in range(s0, s1):
                    cur = self._state(k)
                    for j in range(3):
                        states[k - s0, j].copy_(cur[j])
                    ctrl_log[k - s0].copy_(ctrlf[:_CTRL_DOUBLES])
                    if k + 1 < s1:
                        self.fs.step(1)
                log = ctrl_log[: s1 - s0].cpu().numpy()
                for k in range(s1 - 1, s0 - 1, -1):
                    t, dt, rate = float(log[k - s0, 0]), float(log[k - s0, 1]), float(log[k - s0, 8])
                    u = states[k - s0]
                    a.h, a.qx, a.qy = u[0].data_ptr(), u[1].data_ptr(), u[2].data_ptr()
                    a.lam_h, a.lam_qx, a.lam_qy = (lam[0].data_ptr(), lam[1].data_ptr(),
                                                   lam[2].data_ptr())
                    a.out_h, a.out_qx, a.out_qy = (out[0].data_ptr(), out[1].data_ptr(),
                                                   out[2].data_ptr())
                    a.t, a.dt, a.rain_rate = t, dt, rate
                    a.rain_base = _rain_base(rain, t)
                    a.first = 1 if t == 0.0 else 0
                    _lib.check(L.hb_adjoint_step(ctypes.byref(a), stream), "hb_adjoint_step")
                    if k % self.every == 0 and k > 0:
                        gauge(u[0], k, out[0])
                    lam, out = out, lam
        g = grad.cpu().numpy()
        res = np.concatenate([g[: self.n_zones], g[_lib.HB_MAX_ZONES:]])
        if not with_state:
            return res
        return res, {name: ins.raster(lam[j]) for j, name in enumerate(("h", "qx", "qy"))}


class _MisfitFunction(torch.autograd.Function):
    """J(manning, rain multiplier) with the adjoint as its backward."""

    @staticmethod
    def forward(ctx, manning: torch.Tensor, rain_mult: torch.Tensor, problem: GaugeMisfit):
        samples = problem.simulate(manning.detach().double().cpu().tolist(),
                                   float(rain_mult.detach().cpu()))
        ctx.problem = problem
        return problem.loss(samples).to(manning.device)

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        g = torch.as_tensor(ctx.problem.gradient(), dtype=torch.float64)
        go = grad_out.detach().double().cpu()
        gm = (go * g[:-1]).to(grad_out.device)
        gr = (go * g[-1]).to(grad_out.device)
        return gm, gr, None


def gauge_misfit(problem: GaugeMisfit, manning: torch.Tensor,
                 rain_mult: torch.Tensor) -> torch.Tensor:
    """Differentiable loss: ``gauge_misfit(p, n, r).backward()`` fills n.grad and
    r.grad through the discrete adjoint."""
    return _MisfitFunction.apply(manning, rain_mult, problem)
