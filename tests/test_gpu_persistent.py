"""The persistent step (hb_fused_run): nsteps steps of a whole batch in one
cooperative launch with a grid barrier between steps, against nsteps
per-step launches (hb_fused_step), bit for bit; graph capture; an instance
that halts mid-run; and a barrier budget that runs out on purpose (a
bounded wait that gives up, reported through the status, no fault)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _batch(cuda, sizes=(150, 90, 230), seed=40, **over):
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver
    from hipims_b200.scenarios import catchment_from

    cs = [catchment_from(S.urban_catchment(n, seed=seed + k, rain_mm_h=150.0), **over)
          for k, n in enumerate(sizes)]
    return cs, lambda: FusedSolver(cs, dtype=torch.float32, device=cuda)


def _same(a, b):
    torch.cuda.synchronize()
    for k in range(len(a.inst)):
        x, y = a.compacted(k), b.compacted(k)
        for f in ("h", "qx", "qy", "h_max"):
            np.testing.assert_array_equal(x[f], y[f], err_msg=f"instance {k} {f}")
        ca, cb = a.controls()[k], b.controls()[k]
        assert (ca.t, ca.dt, ca.step, ca.cur) == (cb.t, cb.dt, cb.step, cb.cur)
        assert (ca.volume, ca.outflow_volume, ca.rain_volume) == \
            (cb.volume, cb.outflow_volume, cb.rain_volume)
        assert ca.status == cb.status == 0


def test_persistent_equals_per_step_launches(cuda):
    _, make = _batch(cuda)
    a, b = make(), make()
    a.step(25)
    b.run_persistent(25)
    _same(a, b)
    a.step(7)
    b.run_persistent(3)
    b.run_persistent(4)
    _same(a, b)


def test_persistent_graph_replay(cuda):
    _, make = _batch(cuda, sizes=(130, 200), seed=50)
    a, b = make(), make()
    a.step(30)
    b.capture_persistent(10)
    for _ in range(3):
        b.replay()
    _same(a, b)


def test_persistent_instance_halting_mid_run(cuda):
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver
    from hipims_b200.scenarios import catchment_from

    cs = [catchment_from(S.urban_catchment(120, seed=61, rain_mm_h=150.0), t_end=3.0),
          catchment_from(S.urban_catchment(140, seed=62, rain_mm_h=150.0))]
    a = FusedSolver(cs, dtype=torch.float32, device=cuda)
    b = FusedSolver(cs, dtype=torch.float32, device=cuda)
    a.step(40)
    b.run_persistent(40)
    _same(a, b)
    assert b.controls()[0].halted == 1 and b.controls()[0].step < 40
    assert b.controls()[1].step == 40


def test_persistent_barrier_budget_runs_out(cuda):
    """A budget of one cycle: the first block to reach the grid barrier gives
    up at once.  Every block leaves within a bounded time, bit 8 reports it,
    check() raises, and the context stays usable (a reset solver steps on)."""
    _, make = _batch(cuda, sizes=(300,), seed=70)
    b = make()
    b.run_persistent(5, budget_cycles=1)
    torch.cuda.synchronize()
    assert b.controls()[0].status & 8
    with pytest.raises(FloatingPointError, match="grid barrier"):
        b.check()
    b.reset()
    a = make()
    a.step(6)
    b.run_persistent(6)
    _same(a, b)
