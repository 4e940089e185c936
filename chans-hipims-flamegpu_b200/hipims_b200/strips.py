"""One catchment split into row strips: on one GPU as instances of one batch,
or one strip per GPU (rank) with torch.distributed.

The reference's multi-GPU solver (HP/Parallel_SWE_CUDA.py, driven by
HP/MultiGPU_CatchFlood_main.py) splits the raster into row blocks with two
overlapping rows each side (MUSCL reads two cells each way,
HC/flucCal_2ndOrder_jh_improved_Kernel.cu:410-485) and sums padded buffers
with all_reduce every step.  Here every strip keeps its neighbours' two
boundary rows in the two halo rows the dense layout already has above and
below the raster, so the step kernel runs unchanged; per time step:

  1. halo exchange: the first two and last two rows of h, qx, qy go to the
     neighbouring strips (device copies on one GPU; NCCL send/recv, or gloo
     on CPU tensors, across ranks);
  2. the fused step on every strip, with the control block's external_dt
     set: the step publishes its largest wave speed and any-dry flag;
  3. the maximum of those over all strips (taken by hb_fused_finish itself
     on one GPU, by all_reduce(MAX) across ranks) feeds hb_fused_finish,
     which advances every strip's clock identically (CFL dt, 10x cap, export
     clip).

Every face is evaluated from the same inputs as in the undivided run and the
clock sees the same global speed, so the strips reproduce the single-domain
result bit for bit.  Volumes and rain totals are per strip (sum them).
Each strip must have at least three rows.

Halo forwarding (the default for StripSolver, `peer=True` for
DistributedStrips) folds step 1 into step 2: the step kernel stores the new
state of each strip's first and last two rows also into the neighbour's halo
rows of the same output buffer (hb_instance.halo_up / halo_down), which no
kernel reads during that step.  Across ranks the neighbour's arrays are mapped
with CUDA IPC, the stores are plain peer stores, each thread that made them
issues a system-scope fence (__threadfence_system) before the tile's partial
sum and count, and the clock all_reduce that follows every step orders them
before the neighbour's next step.  One exchange at start-up fills the halos of
the initial state.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Sequence

import numpy as np
import torch

from . import _lib
from .fused import Catchment, FusedSolver, block_datum

HALO = _lib.HB_PAD_Y  # two rows


def split_rows(n_rows: int, parts: int, align: int = 64) -> list[tuple[int, int]]:
    """Contiguous, nearly equal row ranges [a, b) covering n_rows, with the
    inner edges on multiples of `align` rows when every strip can keep at
    least one block (the FP32 bed datum is per 64 x 64 block, so aligned
    strips see the undivided run's datum and round z identically)."""
    if parts < 1 or n_rows < 3 * parts:
        raise ValueError(f"cannot split {n_rows} rows into {parts} strips of >= 3 rows")
    edges = np.linspace(0, n_rows, parts + 1)
    if align > 1 and n_rows >= parts * align:
        edges = np.round(edges / align) * align
        edges[-1] = n_rows
    edges = edges.round().astype(int)
    if np.any(np.diff(edges) < 3):
        edges = np.linspace(0, n_rows, parts + 1).round().astype(int)
    return [(int(edges[k]), int(edges[k + 1])) for k in range(parts)]


def strip_catchment(c: Catchment, a: int, b: int) -> Catchment:
    """Rows [a, b) of a catchment (every raster field cut, settings kept)."""
    cut = lambda x: None if x is None else np.asarray(x)[a:b]
    return dataclasses.replace(
        c, mask=cut(c.mask), z=cut(c.z), h=cut(c.h), qx=cut(c.qx), qy=cut(c.qy),
        zone=cut(c.zone), h_max=cut(c.h_max), cum=cut(c.cum), rain_station=cut(c.rain_station))


def _first_valid(mask: np.ndarray) -> tuple[int, int]:
    flat = np.flatnonzero(np.asarray(mask).ravel() > 0)
    if flat.size == 0:
        return (-1, -1)
    return (int(flat[0] // mask.shape[1]), int(flat[0] % mask.shape[1]))


def _static_halos(fs: FusedSolver, k: int, c: Catchment, a: int, b: int) -> None:
    """Fill instance k's halo rows of z and code from the full catchment's
    rows a-2, a-1 (above) and b, b+1 (below)."""
    ins = fs.inst[k]
    PY, PX, CPX = _lib.HB_PAD_Y, _lib.HB_PAD_X, _lib.HB_CODE_PAD_X
    mask = np.asarray(c.mask)
    z = np.asarray(c.z, dtype=np.float64)
    nrow, ncol = mask.shape
    gdatum = block_datum(mask > 0, z) if fs.dtype == torch.float32 else None
    cls_interior = 0  # any class of this instance: only validity matters for halo cells
    for side, rows in (("top", [a - 2, a - 1]), ("bottom", [b, b + 1])):
        for j, r in enumerate(rows):
            pr = j if side == "top" else PY + (b - a) + j  # padded row index
            if r < 0 or r >= nrow:
                continue  # outside the raster: stays no-data
            valid = mask[r] > 0
            code = np.full(ins.code_pitch, _lib.HB_NODATA_CLASS << 4, dtype=np.uint8)
            code[CPX:CPX + ncol] = np.where(valid, cls_interior << 4, _lib.HB_NODATA_CLASS << 4)
            ins.code[pr].copy_(torch.as_tensor(code, device=fs.device))
            zrow = np.zeros(ins.pitch, dtype=np.float64)
            if fs.dtype == torch.float32:
                # The undivided run stores this row relative to its own block's
                # datum and the kernel shifts it by (that datum - the tile's) in
                # FP32; the strip's kernel shifts halo rows by 0 (its edge block
                # is the tile's block), so store the shifted FP32 value.
                own = np.repeat(gdatum[r // 64], 64)[:ncol].astype(np.float32)
                edge = np.repeat(ins.datum_np[0 if side == "top" else -1], 64)[:ncol]
                rel = (z[r] - own.astype(np.float64)).astype(np.float32)
                val = rel + (own - edge.astype(np.float32))
                zrow[PX:PX + ncol] = np.where(valid, val.astype(np.float64), 0.0)
            else:
                zrow[PX:PX + ncol] = np.where(valid, z[r], 0.0)
            ins.z[pr].copy_(torch.as_tensor(zrow, dtype=fs.dtype, device=fs.device))


def _unshifted(solver_kw: dict) -> dict:
    """Strips keep the tile grid at the raster's origin: their halo rows,
    datum blocks and strip edges are laid out on it."""
    kw = dict(solver_kw)
    if tuple(kw.get("origin") or (0, 0)) != (0, 0):
        raise ValueError("strips run with the tile grid at the raster origin")
    kw["origin"] = (0, 0)
    return kw


def _state_arrays(ins) -> list[torch.Tensor]:
    """[h0, h1, qx0, qx1, qy0, qy1] of one instance (the halo_* order)."""
    return [ins.h[0], ins.h[1], ins.qx[0], ins.qx[1], ins.qy[0], ins.qy[1]]


def _link(fs: FusedSolver, k: int, up: Sequence[int] | None, up_rows: int,
          down: Sequence[int] | None) -> None:
    """Set instance k's halo forwarding targets (device addresses of the
    neighbours' six state arrays, or None) in the host records."""
    r = fs._recs_host[k]
    for j in range(6):
        r.halo_up[j] = up[j] if up is not None else None
        r.halo_down[j] = down[j] if down is not None else None
    r.halo_up_rows = up_rows if up is not None else 0


def _upload_records(fs: FusedSolver) -> None:
    fs.records.copy_(torch.frombuffer(bytearray(fs._recs_host), dtype=torch.uint8))


class StripSolver:
    """A catchment split into `parts` row strips, all on one device, advanced
    with FusedSolver steps and hb_fused_finish.  forward_halos (default): the
    step kernel writes the neighbours' halo rows; False: a halo copy before
    every step."""

    def __init__(self, c: Catchment, parts: int, dtype=torch.float32, device="cuda",
                 forward_halos: bool = True, **solver_kw):
        mask = np.asarray(c.mask)
        self.ranges = split_rows(mask.shape[0], parts)
        self.catchment = c
        strips = [strip_catchment(c, a, b) for a, b in self.ranges]
        self.fs = FusedSolver(strips, dtype=dtype, device=device, **_unshifted(solver_kw))
        self.device = self.fs.device
        gbug = _first_valid(mask)
        for k, (a, b) in enumerate(self.ranges):
            _static_halos(self.fs, k, c, a, b)
            inside = a <= gbug[0] < b
            bug = (gbug[0] - a, gbug[1]) if inside else (-1, -1)
            self.fs.inst[k].bug = bug
            self.fs._recs_host[k].bug_y, self.fs._recs_host[k].bug_x = bug
        self.forward_halos = forward_halos
        if forward_halos:
            inst = self.fs.inst
            ptrs = [[t.data_ptr() for t in _state_arrays(ins)] for ins in inst]
            if any(ins.pitch != inst[0].pitch for ins in inst):
                raise ValueError("strips of one catchment share the row pitch")
            for k in range(len(inst)):
                _link(self.fs, k, ptrs[k - 1] if k > 0 else None,
                      inst[k - 1].rows if k > 0 else 0,
                      ptrs[k + 1] if k + 1 < len(inst) else None)
        _upload_records(self.fs)
        self.fs.set_external_dt(True)
        self._cur = self.fs.controls()[0].cur
        self.exchange()  # halos of the initial state

    def exchange(self) -> None:
        """Copy every strip's two edge rows of h, qx, qy into its neighbours' halos."""
        PY, cur = HALO, self._cur
        inst = self.fs.inst
        for k in range(len(inst) - 1):
            up, dn = inst[k], inst[k + 1]
            ru = up.rows
            for f in ("h", "qx", "qy"):
                U, D = getattr(up, f)[cur], getattr(dn, f)[cur]
                D[0:PY].copy_(U[PY + ru - PY:PY + ru])      # up's last rows -> dn's top halo
                U[PY + ru:PY + ru + PY].copy_(D[PY:2 * PY])  # dn's first rows -> up's bottom halo

    def step(self, nsteps: int = 1) -> None:
        L = _lib.lib()
        for _ in range(nsteps):
            if not self.forward_halos:
                self.exchange()
            self.fs.step(1)
            # NULL ext: the finish kernel takes the maximum over the strips itself
            with torch.cuda.device(self.device):
                _lib.check(L.hb_fused_finish(ctypes.byref(self.fs.batch), None,
                                             self.fs._stream()), "hb_fused_finish")
            self._cur = 1 - self._cur

    def state(self) -> dict[str, torch.Tensor]:
        """The whole raster, strips stacked."""
        parts = [self.fs.state(k) for k in range(len(self.fs.inst))]
        return {f: torch.cat([p[f] for p in parts], dim=0) for f in ("h", "qx", "qy", "h_max")}

    def controls(self):
        return self.fs.controls()


class DistributedStrips:
    """This rank's strip of a catchment split over `world` ranks of an
    initialised torch.distributed process group (NCCL on GPUs; the exchange
    and reduction also run with gloo on CPU tensors).  peer=True: the
    neighbours' state arrays are mapped with CUDA IPC (ranks on one node) and
    the step kernel writes their halo rows; otherwise a halo exchange before
    every step."""

    def __init__(self, c: Catchment, rank: int, world: int, dtype=torch.float32,
                 device="cuda", peer: bool = False, **solver_kw):
        mask = np.asarray(c.mask)
        self.rank, self.world = rank, world
        self.ranges = split_rows(mask.shape[0], world)
        a, b = self.ranges[rank]
        self.fs = FusedSolver(strip_catchment(c, a, b), dtype=dtype, device=device,
                              **_unshifted(solver_kw))
        self.device = self.fs.device
        _static_halos(self.fs, 0, c, a, b)
        gbug = _first_valid(mask)
        bug = (gbug[0] - a, gbug[1]) if a <= gbug[0] < b else (-1, -1)
        self.fs.inst[0].bug = bug
        self.fs._recs_host[0].bug_y, self.fs._recs_host[0].bug_x = bug
        self.peer = peer
        self._peer_arrays: list[torch.Tensor] = []  # keeps the IPC mappings open
        if peer:
            self._map_neighbours()
        _upload_records(self.fs)
        self.fs.set_external_dt(True)
        self._ext_off = _lib.HbCtrl.ext.offset // 8
        self._cur = self.fs.controls()[0].cur
        self.exchange()  # halos of the initial state

    def _map_neighbours(self) -> None:
        """CUDA IPC handles of every rank's state arrays go round the group;
        this rank opens its neighbours' and points its halo forwarding at them."""
        import torch.distributed as dist
        from torch.multiprocessing.reductions import reduce_tensor

        ins = self.fs.inst[0]
        mine = ([reduce_tensor(t) for t in _state_arrays(ins)], ins.rows, ins.pitch)
        every = [None] * self.world
        dist.all_gather_object(every, mine)
        ptr = {}
        for nb in (self.rank - 1, self.rank + 1):
            if 0 <= nb < self.world:
                handles, rows, pitch = every[nb]
                if pitch != ins.pitch:
                    raise ValueError("strips of one catchment share the row pitch")
                ts = [fn(*args) for fn, args in handles]
                self._peer_arrays += ts
                ptr[nb] = ([t.data_ptr() for t in ts], rows)
        up, down = ptr.get(self.rank - 1), ptr.get(self.rank + 1)
        _link(self.fs, 0, up[0] if up else None, up[1] if up else 0, down[0] if down else None)
        dist.barrier()

    def exchange(self) -> None:
        ins = self.fs.inst[0]
        exchange_halos([getattr(ins, f)[self._cur] for f in ("h", "qx", "qy")], ins.rows,
                       self.rank, self.world)

    def step(self, nsteps: int = 1) -> None:
        import torch.distributed as dist

        L = _lib.lib()
        for _ in range(nsteps):
            if not self.peer:
                self.exchange()
            self.fs.step(1)
            ext = self.fs.ctrl.view(torch.float64)[self._ext_off:self._ext_off + 2].clone()
            if dist.get_backend() == "gloo":  # host staging (gloo ranks sharing a device)
                host = ext.cpu()
                dist.all_reduce(host, op=dist.ReduceOp.MAX)
                ext = host.to(self.device)
            else:
                dist.all_reduce(ext, op=dist.ReduceOp.MAX)
            _lib.check(L.hb_fused_finish(ctypes.byref(self.fs.batch), ext.data_ptr(),
                                         self.fs._stream()), "hb_fused_finish")
            self._cur = 1 - self._cur


def exchange_halos(fields: Sequence[torch.Tensor], rows: int, rank: int, world: int) -> None:
    """Halo exchange of dense padded [rows + 2 * HALO + ..., pitch] arrays
    between row strips: this rank's first HALO rows go to rank - 1 (its bottom
    halo), its last HALO rows to rank + 1 (its top halo), and the neighbours'
    rows arrive in this rank's halos.  Works for any backend that supports
    point-to-point (NCCL, gloo)."""
    import torch.distributed as dist

    PY = HALO
    if dist.get_backend() == "gloo" and fields and fields[0].is_cuda:
        # gloo sends host tensors: stage the edge rows through host memory
        host = [F.cpu() for F in fields]
        exchange_halos(host, rows, rank, world)
        for F, H in zip(fields, host):
            F[0:PY].copy_(H[0:PY])
            F[PY + rows:PY + rows + PY].copy_(H[PY + rows:PY + rows + PY])
        return
    ops, recvs = [], []
    for F in fields:
        if rank > 0:
            ops.append(dist.P2POp(dist.isend, F[PY:2 * PY].contiguous(), rank - 1))
            buf = torch.empty_like(F[0:PY])
            ops.append(dist.P2POp(dist.irecv, buf, rank - 1))
            recvs.append((F, 0, buf))
        if rank < world - 1:
            ops.append(dist.P2POp(dist.isend, F[rows:rows + PY].contiguous(), rank + 1))
            buf = torch.empty_like(F[0:PY])
            ops.append(dist.P2POp(dist.irecv, buf, rank + 1))
            recvs.append((F, PY + rows, buf))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for F, at, buf in recvs:
        F[at:at + PY].copy_(buf)
