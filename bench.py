"""Benchmark of the fused HiPIMS step on the synthetic urban catchment.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the configuration the headline metric is quoted on): a 2048 x 2048
urban catchment, 2 m cells, seeded Gaussian-random-field DEM (k^-3, 0-50 m)
with 8 % of cells raised 10 m as buildings, 30 % road cells (n = 0.035, else
0.08), open boundary ring, dry start, uniform rain 50 mm/h.  A step advances
every valid cell (4,194,304) by one time step: the general-tile and the
all-valid-tile builds of the fused step kernel, launched at once.

Timing: 8 untimed spin-up steps (the dry start becomes wet everywhere), W
untimed warm-up steps, then K timed steps.  Each timed step is bracketed by
CUDA events on the launching stream; a 256 MiB buffer is written between timed
steps to flush the 126 MB L2.  nvidia-smi samples the SM clock every 200 ms
from before the first timed step to after the last (the default K keeps the
timed region near 0.6 s, four or more samples).  N > 1 (torchrun): every rank advances its own
replica (weak scaling; the catchment does not shard without a halo exchange),
the time is the max over ranks and `value` counts the cells of all ranks.

--impl reference times the reference's own HiPIMS kernels compiled for the
host (oracle/_ref) under the reference's step order on this machine's CPU
cores, on the same catchment: up to K full steps, stopping after 60 s of
timed steps (the default K = 5000 would take about 13 minutes), so the run
ends within a few minutes; `cpu_baseline.sample` names the steps timed.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "chans-hipims-flamegpu_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "Gcell-updates/s"
N_CELLS = 2048
SPINUP = 8
BYTES_PER_CELL_FP32 = 37  # read h,qx,qy,z,h_max (5 x 4) + code (1); write h,qx,qy,h_max (4 x 4)
FALLBACK_HBM_GBS = 6650.0


def workload(n: int = N_CELLS) -> dict:
    from hipims_b200 import scenarios as S

    return S.urban_catchment(n, dx=2.0, seed=0)


def config_of(n: int, world: int, extra: dict | None = None) -> dict:
    cfg = {"workload": f"urban catchment {n}x{n}, 2 m cells, GRF DEM + 8% buildings, "
                       f"2 Manning zones, open ring, dry start, rain 50 mm/h",
           "cells_per_instance": n * n, "instances_per_gpu": 1,
           "parallelism": f"replicas x{world}", "spinup_steps": SPINUP,
           "l2": "flushed between timed steps (256 MiB write)"}
    if extra:
        cfg.update(extra)
    return cfg


class Clocks:
    """nvidia-smi sampler for the timed region."""

    def wait_first_sample(self, timeout: float = 5.0) -> None:
        """Block until the sampler has written its first line (nvidia-smi
        takes a few hundred ms to start)."""
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < timeout:
            try:
                if os.path.getsize(self.path) > 0:
                    return
            except OSError:
                pass
            time.sleep(0.05)

    def __init__(self, gpu: int):
        self.path = tempfile.mktemp(suffix=".csv")
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for ln in f:
                parts = [p.strip() for p in ln.split(",")]
                if len(parts) >= 7:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[3 + k] == "Active"})
        busy = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def measured_peak() -> tuple[float, str]:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic() -> float | None:
    """DRAM bytes per fused-step launch from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "fused_step_traffic.json")) as f:
            return float(json.load(f)["dram_bytes_per_launch_full_size"])
    except (OSError, KeyError, ValueError):
        return None


def cpu_reference_rate(d: dict, steps: int, warmup: int, threads: int | None = None,
                       budget_s: float = 60.0) -> dict:
    """Cells x steps / s of the reference's host-built kernels (or the
    restatement when oracle/_ref is absent) on catchment d: up to `steps`
    full steps, stopping once `budget_s` seconds of timed steps have run (a
    full 2048^2 step takes ~0.15 s on 16 host threads, so a default
    5000-step request is a bounded sample of the same workload)."""
    from oracle import oracle as O

    kind = "reference" if O.ref_available() else "port"
    threads = threads or os.cpu_count() or 1
    O.set_threads(threads)
    sim = O.Sim(d, order=2, backend="ref" if kind == "reference" else "oracle")
    sim.run(SPINUP + warmup)
    done, el = 0, 0.0
    while done < steps and el < budget_s:
        t0 = time.perf_counter()
        sim.run(1)
        el += time.perf_counter() - t0
        done += 1
    return {"value": sim.N * done / el / 1e9, "unit": METRIC, "cores": threads, "kind": kind,
            "seconds": el, "steps": done,
            "sample": f"{done} steps of the full {int(np.sqrt(sim.N))}^2 catchment after "
                      f"{SPINUP + warmup} untimed steps (at most {steps}, at most "
                      f"{budget_s:.0f} s), FP64, {threads} threads"}


def cpu_dam_break_rates(steps: int = 1000) -> dict:
    """Config 1 on the host: the 256 x 256 dam break, 1000 FP64 steps of the
    reference's kernels built for the host, with 1 thread and with all."""
    from hipims_b200 import scenarios as S
    from oracle import oracle as O

    kind = "reference" if O.ref_available() else "port"
    out = {"kind": kind, "steps": steps, "cells": 256 * 256, "cores": os.cpu_count() or 1,
           "sample": f"config 1: 256^2 dam break, {steps} FP64 steps, 1 thread and all threads"}
    for threads in (1, os.cpu_count() or 1):
        O.set_threads(threads)
        sim = O.Sim(S.dam_break(256), order=2, backend="ref" if kind == "reference" else "oracle")
        t0 = time.perf_counter()
        sim.run(steps)
        el = time.perf_counter() - t0
        out[f"threads_{threads}"] = {"value": sim.N * steps / el / 1e9, "unit": METRIC,
                                     "seconds": el}
    return out


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    d = workload(args.cells)
    cb = cpu_reference_rate(d, args.steps, args.warmup)
    line = {"metric": METRIC, "value": cb["value"], "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cb["seconds"] / cb["steps"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": config_of(args.cells, 1),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import torch.distributed as dist

    from hipims_b200 import _lib
    from hipims_b200.fused import FusedSolver
    from hipims_b200.scenarios import catchment_from

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    strips = None
    if args.strips:
        # one catchment of (ranks x n) x n cells split in row strips, one per
        # rank (weak scaling with a halo exchange and a clock all_reduce per
        # step); on one GPU, the n x n catchment in two strips of one batch
        from hipims_b200 import scenarios as S
        from hipims_b200.strips import DistributedStrips, StripSolver

        d = S.urban_catchment(args.cells, dx=2.0, seed=0, n_rows=args.cells * max(world, 1))
        if world > 1:
            strips = DistributedStrips(catchment_from(d), rank, world, dtype=torch.float32,
                                       tile=tuple(args.tile), device=dev, minb=args.minb,
                                       peer=args.peer)
        else:
            strips = StripSolver(catchment_from(d), 2, dtype=torch.float32,
                                 tile=tuple(args.tile), device=dev, minb=args.minb)
        fs = strips.fs
    else:
        d = workload(args.cells)
        fs = FusedSolver(catchment_from(d), dtype=torch.float32, tile=tuple(args.tile),
                         device=dev, minb=args.minb)
    n_valid = sum(i.n_valid for i in fs.inst)  # this rank's cells
    total_cells = n_valid
    if world > 1:
        tc = torch.tensor([float(n_valid)], device=dev, dtype=torch.float64)
        dist.all_reduce(tc)
        total_cells = int(tc.item())
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stepper = strips if strips is not None else fs

    stepper.step(SPINUP + args.warmup)
    torch.cuda.synchronize(dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    clocks = Clocks(local)
    clocks.wait_first_sample()
    barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for a, b in ev:
        flush.fill_(1)
        a.record(stream)
        stepper.step(1)
        b.record(stream)
    barrier()
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = total_cells * args.steps / (total_ms * 1e-3) / 1e9
    c = fs.controls()[0]

    # end to end through the C ABI with host buffers: H2D of the state from
    # pinned memory, one fused step, D2H of the new state, every step
    e2e_steps = min(args.steps, 200)
    if strips is None:
        # HostStepper: the inbound copy of a step overlaps the outbound copy
        # of the previous one (PCIe is full duplex)
        from hipims_b200.fused import HostStepper

        hst = HostStepper(fs, layout="compact")
        host_in = hst.in_buffers
        e2e_path = ("HostStepper: pinned host h, qx, qy in the reference's compacted layout "
                    "(valid cells, row-major) -> device, hb_state_layout into the dense "
                    "arrays, hb_fused_step, hb_state_layout back -> pinned host, every step; "
                    "inbound copy of step k+1 overlapping the outbound copy of step k")
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            hst.step()
        hst.finish()
        e1.record(stream)
        barrier()
    else:
        state = lambda b: [x for ins in fs.inst for x in (ins.h[b], ins.qx[b], ins.qy[b])]
        host_in = [torch.empty_like(x, device="cpu").pin_memory() for x in state(0)]
        host_out = [torch.empty_like(x).pin_memory() for x in host_in]
        for hsrc, x in zip(host_in, state(c.cur)):
            hsrc.copy_(x)
        cur = c.cur
        e2e_path = ("pinned host h, qx, qy -> device; halo exchange + hb_fused_step + "
                    "hb_fused_finish; device -> pinned host, every step")
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            for hsrc, x in zip(host_in, state(cur)):
                x.copy_(hsrc, non_blocking=True)
            stepper.step(1)
            cur = 1 - cur
            for hdst, x in zip(host_out, state(cur)):
                hdst.copy_(x, non_blocking=True)
        e1.record(stream)
        barrier()
    e2e_ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = total_cells * e2e_steps / (e2e_ms * 1e-3) / 1e9
    bytes_io = sum(x.numel() * x.element_size() for x in host_in)

    if rank == 0:
        peak, peak_kind = measured_peak()
        avg_s = total_ms / args.steps * 1e-3
        alg_bytes = BYTES_PER_CELL_FP32 * n_valid
        achieved = alg_bytes / avg_s / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "ours",
            "config": config_of(args.cells, world, strip_config(args, world)),
            "launch": {"tile": list(args.tile), "min_blocks_per_sm": args.minb,
                       "cells_per_lane": args.tile[1] // 32,
                       "sim_time_s": c.t, "dt_s": c.dt},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "kernel": f"{step_kernel_name(args)}; timed as the step",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "traffic": profiled_traffic()},
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": bytes_io,
                    "d2h_bytes_per_step": bytes_io, "steps": e2e_steps,
                    "path": e2e_path},
            # per step: the one-launch step kernel, or the general-tile and
            # all-valid-tile builds (+ hb_fused_finish for strips)
            "gpu_launches": args.steps * ((1 if one_launch_step(args) else 2) +
                                          (1 if strips is not None else 0)),
            "clocks": clk,
            "step_ms_min": min(step_ms), "step_ms_max": max(step_ms),
        }
        if args.accuracy and world == 1 and not args.strips:
            line["accuracy"] = accuracy_vs_fp64(d, dev)
        if args.first_order and world == 1:
            line["first_order"] = first_order_rates(d, dev, args, flush, stream)
        if args.plain and world == 1:
            pl = plain_fp64_rate(d, dev, reference_kernels=True)
            if pl.get("value"):
                pl["fused_fp32_over_plain"] = value / pl["value"]
            line["fp64_plain"] = pl
            pc = plain_fp64_rate(d, dev, reference_kernels=False)
            pc["fused_fp32_over_compat"] = value / pc["value"]
            line["fp64_compat"] = pc
        if args.ensemble and world == 1:
            en = ensemble_rate(dev, args.ensemble_steps)
            if line.get("fp64_plain", {}).get("value"):
                en["over_plain_fp64"] = en["value"] / line["fp64_plain"]["value"]
            line["ensemble"] = en
        if args.coupled and world == 1:
            line["coupled"] = coupled_rate(dev, args.coupled_cells)
        if args.adjoint and world == 1:
            line["adjoint"] = adjoint_cost(dev, args.adjoint_cells, args.adjoint_steps)
        if args.cpu_c1 and world == 1:
            line["cpu_dam_break"] = cpu_dam_break_rates()
        if args.cpu_baseline and world == 1:
            line["cpu_baseline"] = {k: v for k, v in cpu_reference_rate(
                d, args.cpu_steps, 0).items() if k in ("value", "unit", "cores", "kind",
                                                       "sample")}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    del _lib


def one_launch_step(args) -> bool:
    """The 64-wide tiles at the default register cap run the step as one
    launch over both tile lists (pairs_mixed_kernel); other shapes launch the
    general-tile and all-valid-tile builds at once on two streams."""
    return args.tile[1] == 64 and args.minb in (0, 4)


def step_kernel_name(args) -> str:
    if one_launch_step(args):
        return (f"pairs_mixed_kernel<{args.tile[0]}> (two cells per lane, one launch over the "
                f"general and all-valid tiles)")
    if args.tile[1] == 64:
        return (f"pairs_step_kernel<{args.tile[0]},minb={args.minb}> (two cells per lane) "
                f"general-tile and all-valid-tile builds, run at once")
    return (f"rows_step_kernel<float,{args.tile[0]},minb={args.minb}> general-tile and "
            f"all-valid-tile builds, run at once")


def strip_config(args, world: int) -> dict:
    if not args.strips:
        return {}
    if world > 1:
        halo = ("halo rows written by the step kernel through CUDA IPC peer mappings"
                if args.peer else "NCCL halo exchange (2 rows of h, qx, qy each way)")
        return {"decomposition": f"one {args.cells * world}x{args.cells} catchment in {world} "
                                 f"row strips, one per GPU: {halo} and all_reduce(MAX) of the "
                                 f"clock inputs per step", "parallelism": f"strips x{world}"}
    return {"decomposition": f"one {args.cells}x{args.cells} catchment in 2 row strips on one "
                             f"GPU (halo rows written by the step kernel, clock inputs reduced "
                             f"by hb_fused_finish)"}


def plain_fp64_rate(d: dict, dev, steps: int = 50, reference_kernels: bool = True,
                    order: int = 2, repeats: int = 3) -> dict:
    """The plain FP64 GPU path on the same catchment, wall clock per step: the
    reference's own solver class (HP/SWE_CUDA.py Godunov, unmodified, staged
    in baseline/_ref by baseline/install_ref_py.py) and its step loop
    (CHANS-HiPIMS_server.py:246-256: compacted cells, gather-based per-cell
    fluxes, nonzero / empty_cache / .item() per step), with its 13 extension
    modules resolved to the reference's own kernels built for sm_100a
    (reference_kernels; baseline/build_ref_cuda.py) or to this library's
    drop-in modules.  Where the reference class is not staged, the restated
    loop of hipims_b200.solver runs instead and `loop` says so.  The loop's
    per-step allocator and host round trips make single timings noisy, so
    `repeats` runs of `steps` steps are timed one after another and `value`
    is their median (`runs` lists all)."""
    from baseline import ref_loop

    if reference_kernels:
        from baseline import ref_gpu

        if not ref_gpu.available():
            return {"value": None, "unavailable": "baseline/_ref not built"}
    kernels = ("the reference's own kernels built for sm_100a (flux, fluxMask, friction-update, "
               "timeControl, station rain)" if reference_kernels
               else "this library's drop-in op modules (compat kernels)")
    if ref_loop.available():
        mods = ref_loop.reference_kernel_modules() if reference_kernels else ref_loop.b200_modules()
        cls = ref_loop.load_swe_cuda(mods).Godunov
        loop = "reference HP/SWE_CUDA.py Godunov, unmodified"
        kw = {}
    else:
        from hipims_b200.solver import Godunov as cls

        loop = "restated Godunov (hipims_b200.solver): the reference class is not staged"
        kw = {"ops_impl": __import__("baseline.ref_gpu", fromlist=["RefGpuOps"]).RefGpuOps()
              if reference_kernels else None}
    g = cls(dev, d["dx"], d["cfl"], 1.0e30, secondOrder=order == 2, firstTimeStep=d["first_dt"],
            tensorType=torch.float64, **kw)
    if hasattr(g, "_export_enabled"):
        g._export_enabled = False
    T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64))
    mask = torch.as_tensor(d["mask"])
    g.init__fluidField_tensor(mask, T(d["h"]), T(d["qx"]), T(d["qy"]), T(d["wl"]), T(d["z"]),
                              dev)
    g.set__frictionField_tensor(torch.tensor(d["manning"], dtype=torch.float64, device=dev), dev)
    g.set_landuse(mask, torch.as_tensor(d["landuse"]), dev)
    g.set_distributed_rainfall_station_Mask(mask, torch.zeros(mask.shape, dtype=torch.int16), dev)

    def one():
        g.addFlux()
        g.addStation_PrecipitationSource(d["rain"], dev)
        g.time_friction_euler_update_cuda(dev)

    import contextlib
    import io

    # the reference's 1st-order addFlux prints t every step: kept, but not on stdout
    n = int(g._h_internal.numel())
    runs = []
    with contextlib.redirect_stdout(io.StringIO()):
        for _ in range(SPINUP):
            one()
        torch.cuda.synchronize(dev)
        for _ in range(repeats):
            t0 = time.perf_counter()
            for _ in range(steps):
                one()
            torch.cuda.synchronize(dev)
            runs.append(n * steps / (time.perf_counter() - t0) / 1e9)
    return {"value": float(np.median(runs)), "unit": METRIC, "steps": steps, "repeats": repeats,
            "runs": runs, "dtype": "f64", "loop": loop, "kernels": kernels,
            "path": f"{loop} on {kernels}, wall clock, median of {repeats} runs"}


def first_order_rates(d: dict, dev, args, flush: torch.Tensor, stream, steps: int = 500) -> dict:
    """The reference's 1st-order scheme (secondOrder False, the coupled
    server's choice) on the same catchment: the fused FP32 step timed like the
    main leg (CUDA events per step, L2 flushed between steps), and the
    reference's own 1st-order kernels on the B200 under the Godunov loop."""
    from hipims_b200.fused import FusedSolver
    from hipims_b200.scenarios import catchment_from

    fs = FusedSolver(catchment_from(d), dtype=torch.float32, tile=(32, 64), device=dev,
                     order=1)
    n = sum(i.n_valid for i in fs.inst)
    fs.step(SPINUP + args.warmup)
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    for a, b in ev:
        flush.fill_(1)
        a.record(stream)
        fs.step(1)
        b.record(stream)
    torch.cuda.synchronize(dev)
    fs.check()
    ms = sum(a.elapsed_time(b) for a, b in ev) / steps
    value = n / (ms * 1e-3) / 1e9
    out = {"value": value, "unit": METRIC, "steps": steps, "ms_per_step": ms, "dtype": "f32",
           "path": "FusedSolver(order=1), 64 x 32 tiles, two cells per lane: one launch per "
                   "step of the 1st-order step kernel over the general and all-valid tiles, "
                   "CUDA events per step, L2 flushed between steps"}
    del fs
    pl = plain_fp64_rate(d, dev, reference_kernels=True, order=1)
    out["fp64_plain_first_order"] = pl
    if pl.get("value"):
        out["fused_fp32_over_plain"] = value / pl["value"]
    return out


def ensemble_rate(dev, steps: int, count: int = 64, seed: int = 0, plain_sample: int = 8) -> dict:
    """Config 3: `count` catchments (sides 256-1536, own hyetographs) advanced
    together.  `value`: one persistent cooperative launch of `steps` steps for
    all of them (hb_fused_run), replayed from a CUDA graph.  Beside it: the
    same batch as one graph of `steps` per-step launches, the autotuned
    launch shape, 64 sequential single-instance fused runs, and the plain FP64
    path (the reference's solver class on its own kernels) on a sample of the
    catchments run one after another."""
    from hipims_b200 import autotune, scenarios as S
    from hipims_b200.fused import FusedSolver
    from hipims_b200.scenarios import catchment_from

    ds = S.ensemble(count, seed=seed)
    cs = [catchment_from(d) for d in ds]
    cfg = autotune.tune(cs, torch.float32, dev, steps=4)
    st = torch.cuda.current_stream(dev)

    def timed(fn) -> float:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        a.record(st)
        fn()
        b.record(st)
        torch.cuda.synchronize(dev)
        return a.elapsed_time(b)

    # persistent: one launch of `steps` steps, replayed from a graph
    fp = FusedSolver(cs, dtype=torch.float32, device=dev, tile=(32, 64),
                     minb=cfg.get("minb", 0) if tuple(cfg["tile"]) == (32, 64) else 0)
    cells = sum(i.n_valid for i in fp.inst)
    fp.step(SPINUP)
    fp.capture_persistent(steps)
    fp.replay()  # warm-up replay
    ms_p = timed(fp.replay)
    fp.check()
    del fp
    torch.cuda.empty_cache()
    # per-step launches, autotuned shape, replayed from a graph
    fs = FusedSolver(cs, dtype=torch.float32, device=dev, tile=cfg["tile"],
                     minb=cfg.get("minb", 0))
    fs.step(SPINUP)
    fs.capture(steps)
    fs.replay()
    ms_s = timed(fs.replay)
    del fs
    torch.cuda.empty_cache()
    # 64 sequential single-instance runs, each `steps` launches after spin-up
    ms_seq = 0.0
    for c in cs:
        f1 = FusedSolver(c, dtype=torch.float32, device=dev, tile=(32, 64))
        f1.step(SPINUP)
        ms_seq += timed(lambda: f1.step(steps))
        del f1
    torch.cuda.empty_cache()
    # the plain FP64 path on every (count // plain_sample)-th catchment, one after another
    plain = None
    picked = ds[:: max(count // plain_sample, 1)][:plain_sample]
    pl_cells, pl_s = 0, 0.0
    for d in picked:
        r = plain_fp64_rate(d, dev, steps=20, reference_kernels=True)
        if not r.get("value"):
            plain = r
            break
        n = int(np.sum(np.asarray(d["mask"]) > 0))
        pl_cells += n * 20
        pl_s += n * 20 / (r["value"] * 1e9)
    if plain is None and pl_s > 0:
        plain = {"value": pl_cells / pl_s / 1e9, "unit": METRIC, "catchments": len(picked),
                 "steps_each": 20, "path": r["path"] + " per catchment, catchments one after "
                                                      "another"}
    value = cells * steps / (ms_p * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    achieved = BYTES_PER_CELL_FP32 * cells * steps / (ms_p * 1e-3) / 1e9
    out = {"value": value, "unit": METRIC, "instances": count, "cells": cells, "steps": steps,
           "ms_per_step": ms_p / steps,
           "launch": f"one persistent cooperative launch (hb_fused_run) of {steps} steps for all "
                     f"instances, replayed from a CUDA graph",
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_source": peak_kind},
           "per_step_launches": {"value": cells * steps / (ms_s * 1e-3) / 1e9, "unit": METRIC,
                                 "tile": list(cfg["tile"]), "minb": cfg.get("minb", 0),
                                 "cells_per_lane": autotune.cells_per_lane(cfg),
                                 "launch": f"one CUDA-graph replay of {steps} per-step launches "
                                           f"(autotuned shape: one launch per step for 64-wide "
                                           f"tiles at 4 CTAs per SM, a pair otherwise)"},
           "sequential_single_runs": {"value": cells * steps / (ms_seq * 1e-3) / 1e9,
                                      "unit": METRIC,
                                      "path": f"{count} single-instance fused FP32 runs, one "
                                              f"after another, {steps} steps each"}}
    out["over_sequential_single_runs"] = value / out["sequential_single_runs"]["value"]
    if plain is not None:
        out["sequential_plain_fp64"] = plain
        if plain.get("value"):
            out["over_sequential_plain_fp64"] = value / plain["value"]
    return out


def adjoint_cost(dev, n: int = 1024, steps: int = 2000, K: int = 100, every: int = 10,
                 fd: bool = True) -> dict:
    """Config 4: Manning calibration on an n x n catchment with 16 Voronoi
    zones and 32 gauges sampled every 10 steps; cost of the checkpointed
    adjoint (recompute included) against the forward, and the gradient against
    central differences (relative step 1e-5) of the same frozen-dt forward."""
    from hipims_b200 import scenarios as S
    from hipims_b200.adjoint import GaugeMisfit, record_schedule
    from hipims_b200.scenarios import catchment_from

    d = S.adjoint_case(n, seed=0)
    c = catchment_from(d)
    dts = record_schedule(c, steps, device=dev)
    truth = GaugeMisfit(c, d["gauge_rows"], d["gauge_cols"], steps, dts, every, K, device=dev)
    obs = truth.simulate(d["manning"], 1.0).clone()
    del truth
    p = GaugeMisfit(c, d["gauge_rows"], d["gauge_cols"], steps, dts, every, K, obs=obs,
                    device=dev)
    start = [v * 1.25 for v in d["manning"]]
    p.simulate(start, 0.8)
    p.gradient()  # warm-up
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    p.simulate(start, 0.8)
    torch.cuda.synchronize(dev)
    t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter()
    g = p.gradient()
    torch.cuda.synchronize(dev)
    t_adj = time.perf_counter() - t0
    # the forward alone, without checkpoints or gauge samples
    p.fs.reset(0.8)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    p.fs.step(steps)
    torch.cuda.synchronize(dev)
    t_plain = time.perf_counter() - t0
    # the gradient along the FP32 product's trajectory (FP32 forward and
    # recompute, FP64 reverse sweep) against the FP64 adjoint above
    q = GaugeMisfit(c, d["gauge_rows"], d["gauge_cols"], steps, dts, every, K, obs=obs,
                    device=dev, forward_dtype=torch.float32)
    q.simulate(start, 0.8)
    q.gradient()  # warm-up
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    q.simulate(start, 0.8)
    torch.cuda.synchronize(dev)
    t_fwd32 = time.perf_counter() - t0
    t0 = time.perf_counter()
    g32 = q.gradient()
    torch.cuda.synchronize(dev)
    t_adj32 = time.perf_counter() - t0
    fp32_leg = {"forward_s": t_fwd32, "adjoint_s": t_adj32,
                "adjoint_over_forward": t_adj32 / t_fwd32,
                "max_rel_diff_vs_fp64_gradient": float(np.abs(g32 - g).max() / np.abs(g).max()),
                "gradient": [float(x) for x in g32],
                "path": "FP32 forward and recompute (pairs step), FP64 reverse sweep at the "
                        "FP32 states; reference: the FP64 adjoint of the same problem"}
    del q
    out = {"cells": int(p.fs.inst[0].n_valid), "steps": steps, "checkpoint": K,
           "zones": len(d["manning"]), "gauges": int(p.n_gauges), "sample_every": every,
           "forward_s": t_fwd, "forward_plain_s": t_plain, "adjoint_s": t_adj,
           "adjoint_over_forward": t_adj / t_fwd, "dtype": "f64",
           "grad_abs_max": float(np.abs(g).max()), "fp32_forward": fp32_leg}
    if fd:
        J = lambda m, r: float(p.loss(p.simulate(m, r)))

        def central(rel):
            res = []
            for z in range(len(start) + 1):
                base = start[z] if z < len(start) else 0.8
                e = rel * base
                if z < len(start):
                    up, dn = list(start), list(start)
                    up[z] += e
                    dn[z] -= e
                    res.append((J(up, 0.8) - J(dn, 0.8)) / (2 * e))
                else:
                    res.append((J(start, 0.8 + e) - J(start, 0.8 - e)) / (2 * e))
            return np.asarray(res)

        f4, f5, f6 = central(1e-4), central(1e-5), central(1e-6)
        scale = float(np.abs(f5).max())
        # a parameter in which the loss is differentiable at these scales has
        # difference quotients that agree across the three steps; the
        # wet/dry threshold, the flux mask and the limiter make the others
        # jump (their quotients differ by factors between steps)
        stable = (np.abs(f4 - f5) <= 1e-4 * scale) & (np.abs(f6 - f5) <= 1e-4 * scale)
        err = np.abs(g - f5) / scale
        out["fd"] = {
            "rel_steps": [1e-4, 1e-5, 1e-6], "params": len(g),
            "resolvable": int(stable.sum()),
            "resolvable_rule": "|fd(1e-4) - fd(1e-5)| and |fd(1e-6) - fd(1e-5)| <= 1e-4 max|fd|",
            "not_resolvable": [int(k) for k in np.flatnonzero(~stable)],
            "fd_1e-6": [float(x) for x in f6],
            "max_err_over_max_grad_resolvable": float(err[stable].max()) if stable.any()
            else None,
            "max_err_over_max_grad_all": float(err.max()),
            "adjoint": [float(x) for x in g], "fd_1e-5": [float(x) for x in f5],
            "fd_1e-4": [float(x) for x in f4]}
    return out


def coupled_rate(dev, n: int = 8192, sim_seconds: float = 120.0, period: float = 60.0,
                 agents: int = 100_000, tile=(32, 64), minb: int = 0) -> dict:
    """Config 5: an n x n catchment (1 m cells, rain 100 mm/h, Q_GIVEN inflow
    hydrograph on one edge) advanced by the fused FP32 step from a dry start,
    in the 1st-order scheme the reference's coupled server runs
    (CHANS-HiPIMS_server.py: secondOrder False); every `period` simulated
    seconds the agent cells' depth and velocities are gathered on the device,
    copied to the host and serialised with msgpack, as the RPC server's
    request_data answer.  Wall clock over the whole run."""
    import msgpack

    from hipims_b200 import scenarios as S
    from hipims_b200.coupling import FusedBackend
    from hipims_b200.fused import FusedSolver
    from hipims_b200.scenarios import catchment_from

    d = S.coupled_case(n, agents=agents)
    fs = FusedSolver(catchment_from(d, t_end=sim_seconds), dtype=torch.float32,
                     tile=tuple(tile), device=dev, minb=minb, order=1)
    be = FusedBackend(fs, d["agent_rows"], d["agent_cols"], velocities=True)
    cells = fs.inst[0].n_valid
    del d
    fs.step(3)  # warm-up (first launch, module load)
    torch.cuda.synchronize(dev)
    s0 = fs.controls()[0].step
    t_couple, nbytes = 0.0, 0
    t0 = time.perf_counter()
    k = 1
    while k * period <= sim_seconds + 1e-9:
        fs.run_until(k * period, chunk=128)
        c0 = time.perf_counter()
        payload = msgpack.packb(be.gather())
        t_couple += time.perf_counter() - c0
        nbytes = len(payload)
        k += 1
    torch.cuda.synchronize(dev)
    total = time.perf_counter() - t0
    c = fs.controls()[0]
    steps = c.step - s0
    peak, peak_kind = measured_peak()
    achieved = BYTES_PER_CELL_FP32 * cells * steps / total / 1e9
    return {"value": cells * steps / total / 1e9, "unit": METRIC, "cells": cells,
            "steps": steps, "sim_time_s": c.t, "wall_s": total, "agents": agents,
            "couplings": k - 1, "coupling_s": t_couple,
            "coupling_overhead": t_couple / total, "payload_bytes": nbytes,
            "hbm_achieved_gbs": achieved, "hbm_frac": achieved / peak,
            "peak_source": peak_kind,
            "scheme": "1st order (the coupled server's)",
            "path": "FusedSolver.run_until (chunks of 128 launches, control-block read per "
                    "chunk) + hb_gather of h, u, v + D2H + msgpack, wall clock"}


def accuracy_vs_fp64(d: dict, dev, horizons=(64, 1000), times=(300.0, 600.0)) -> dict:
    """Max depth / velocity difference of the FP32 fused run against the FP64
    fused run at identical simulated times (the FP64 dt sequence replayed), and
    the FP64 volume balance of the FP32 run, after each horizon: the step
    counts in `horizons` and the first steps that reach the simulated times in
    `times` (from the dry start).

    The horizons stop at 600 s of the 3600 s storm: from about 650 s on, the
    reference scheme draws water in through the OPEN ring (its zero-gradient
    ghost copies an edge cell whose velocity points inwards, so that cell never
    drains), and isolated cells reach 50-300 m/s; the reference's own kernels,
    the FP64 and the FP32 fused runs all do so, and their trajectories part
    (different step counts to the same time), so no pointwise comparison is
    meaningful there."""
    from hipims_b200.fused import FusedSolver
    from hipims_b200.scenarios import catchment_from

    f64 = FusedSolver(catchment_from(d), dtype=torch.float64, device=dev)
    dts, ref, k = [], {}, 0
    steps_set, pending = set(horizons), sorted(times)
    while k < max(horizons, default=0) or pending:
        f64.step(1)
        k += 1
        c = f64.controls()[0]
        dts.append(c.dt)
        hit = k in steps_set
        while pending and c.t >= pending[0]:
            pending.pop(0)
            hit = True
        if hit:
            ref[k] = f64.compacted()
    horizons = sorted(ref)
    del f64
    # the scheme's own sensitivity: the FP64 run again with the bed scaled by
    # (1 + 1e-15), same dt sequence
    zp = np.asarray(d["z"], dtype=np.float64) * (1.0 + 1e-15)
    f64p = FusedSolver(catchment_from(d, z=zp, dt_replay=np.asarray(dts)), dtype=torch.float64,
                       device=dev)
    sens, done = {}, 0
    for k in horizons:
        f64p.step(k - done)
        done = k
        sens[k] = float(np.abs(f64p.compacted()["h"] - ref[k]["h"]).max())
    del f64p
    f32 = FusedSolver(catchment_from(d, dt_replay=np.asarray(dts)), dtype=torch.float32,
                      device=dev)
    out, done = [], 0
    for k in horizons:
        f32.step(k - done)
        done = k
        a, b = f32.compacted(), ref[k]
        wet = b["h"] > 1e-3
        ua = np.where(wet, a["qx"] / np.maximum(a["h"], 1e-3), 0)
        ub = np.where(wet, b["qx"] / np.maximum(b["h"], 1e-3), 0)
        c = f32.controls()[0]
        bal = abs(c.volume - c.volume0 - c.rain_volume + c.outflow_volume) / max(
            c.rain_volume, 1e-30)
        dh = np.abs(a["h"] - b["h"])
        out.append({"steps": k, "sim_time_s": c.t,
                    "max_abs_dh_m": float(dh.max()),
                    "p99_99_abs_dh_m": float(np.quantile(dh, 0.9999)),
                    "cells_dh_over_1e-4": int((dh > 1e-4).sum()),
                    "cells_dh_over_1e-3": int((dh > 1e-3).sum()),
                    "max_abs_du_ms_wet": float(np.abs(ua - ub).max()),
                    "flooded_cells_fp64": int((b["h"] > 0.1).sum()),
                    "flooded_cells_differing": int(((a["h"] > 0.1) != (b["h"] > 0.1)).sum()),
                    "volume_balance_rel_err": bal,
                    "fp64_self_sensitivity_max_abs_dh_m": sens[k]})
    return {"horizons": out, "reference": "FP64 fused run, same dt sequence",
            "fp64_self_sensitivity": "max |dh| of the FP64 run with the bed scaled by "
                                     "(1 + 1e-15), same dt sequence"}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cells", type=int, default=N_CELLS)
    ap.add_argument("--tile", type=int, nargs=2, default=[32, 64],
                    help="tile rows, cols: 32 64 = two cells per lane (default), 32 32 or "
                         "64 32 = one cell per lane")
    ap.add_argument("--minb", type=int, default=0,
                    help="register cap as resident CTAs per SM (0: the build's default)")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-accuracy", dest="accuracy", action="store_false")
    ap.add_argument("--no-plain", dest="plain", action="store_false")
    ap.add_argument("--no-first-order", dest="first_order", action="store_false")
    ap.add_argument("--no-ensemble", dest="ensemble", action="store_false")
    ap.add_argument("--ensemble-steps", type=int, default=20)
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false")
    ap.add_argument("--no-coupled", dest="coupled", action="store_false")
    ap.add_argument("--peer", action="store_true",
                    help="with --strips on N > 1 GPUs: the step kernel writes the neighbour "
                         "ranks' halo rows through CUDA IPC mappings (one node)")
    ap.add_argument("--strips", action="store_true",
                    help="one catchment split in row strips over the GPUs (halo exchange) "
                         "instead of independent replicas")
    ap.add_argument("--no-cpu-c1", dest="cpu_c1", action="store_false",
                    help="skip the 256^2 dam break timed on the host (1 and all threads)")
    ap.add_argument("--coupled-cells", type=int, default=8192)
    ap.add_argument("--adjoint-cells", type=int, default=1024)
    ap.add_argument("--adjoint-steps", type=int, default=2000)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
