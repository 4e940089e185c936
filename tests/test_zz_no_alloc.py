"""The allocation-free fused step (hb_fused_step_noalloc) against the regular
one (hb_fused_step with a caller-allocated workspace).

hb_fused_step_noalloc exists for callers that cannot allocate device memory:
host programs that manage a fixed device-memory budget themselves, such as
the agent runtime this solver is coupled to, and threads that cannot afford
the device-wide synchronisation of cudaMalloc/cudaFree while other kernels
run.  Its scratch is one fixed 4 MiB array inside the library.

This file is collected last so that a run stopping at the first failure has
run every other test first.  It must pass alone and after the other tests."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-6  # the FP32 tolerance of the fused tests; the two paths run the same kernel


def _pair(cuda):
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver
    from hipims_b200.scenarios import catchment_from

    d = S.urban_catchment(150, seed=3, rain_mm_h=200.0)
    a = FusedSolver(catchment_from(d), dtype=torch.float32, device=cuda)
    b = FusedSolver(catchment_from(d), dtype=torch.float32, device=cuda)
    return a, b


def _compare(a, b):
    torch.cuda.synchronize()
    ca, cb = a.controls()[0], b.controls()[0]
    assert ca.step == cb.step and ca.t == cb.t and ca.dt == cb.dt
    sa, sb = a.compacted(), b.compacted()
    for f in ("h", "qx", "qy", "h_max"):
        assert np.abs(sa[f] - sb[f]).max() <= TOL, f


def test_noalloc_matches_workspace_entry_over_two_calls(cuda):
    from hipims_b200 import _lib

    assert "hb_fused_step_noalloc" in _lib.declared_symbols()
    a, b = _pair(cuda)
    a.step(7)
    b.step_noalloc(7, prepare=True)  # first call: sets up the fixed scratch
    _compare(a, b)
    a.step(5)
    b.step_noalloc(5)  # second call reuses it
    _compare(a, b)


def _solvers(cuda, sizes, seed):
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver
    from hipims_b200.scenarios import catchment_from

    cs = [catchment_from(S.urban_catchment(n, seed=seed + k, rain_mm_h=200.0))
          for k, n in enumerate(sizes)]
    return (FusedSolver(cs, dtype=torch.float32, device=cuda),
            FusedSolver(cs, dtype=torch.float32, device=cuda))


def _compare_all(a, b):
    torch.cuda.synchronize()
    for k in range(len(a.inst)):
        ca, cb = a.controls()[k], b.controls()[k]
        assert ca.step == cb.step and ca.t == cb.t and ca.dt == cb.dt
        sa, sb = a.compacted(k), b.compacted(k)
        for f in ("h", "qx", "qy", "h_max"):
            assert np.abs(sa[f] - sb[f]).max() <= TOL, (k, f)


def test_noalloc_two_batches_in_turn(cuda):
    """Batch A, then batch B of another size and instance count (other tile
    counts, workspace offsets and tile order in the shared array), then A
    again: each call re-prepares the array for its batch and matches that
    batch's workspace twin."""
    a_ws, a_na = _solvers(cuda, (150,), 3)
    b_ws, b_na = _solvers(cuda, (90, 200), 11)
    for steps in (6, 4):
        a_ws.step(steps)
        a_na.step_noalloc(steps, prepare=True)
        _compare_all(a_ws, a_na)
        b_ws.step(steps)
        b_na.step_noalloc(steps, prepare=True)
        _compare_all(b_ws, b_na)
    a_ws.step(3)
    a_na.step_noalloc(3, prepare=True)
    _compare_all(a_ws, a_na)
    a_ws.step(2)
    a_na.step_noalloc(2)  # A was prepared last: no prepare needed
    _compare_all(a_ws, a_na)


def test_noalloc_refuses_a_batch_it_was_not_prepared_for(cuda):
    """A call without prepare for a batch other than the one the array was
    last prepared for returns HB_ERR_ARG and leaves that batch's state alone."""
    import ctypes

    from hipims_b200 import _lib

    a_ws, a_na = _solvers(cuda, (120,), 5)
    _, b_na = _solvers(cuda, (80,), 7)
    a_na.step_noalloc(2, prepare=True)
    before = b_na.compacted(0)["h"].copy()
    L = _lib.lib()
    with torch.cuda.device(cuda):
        rc = L.hb_fused_step_noalloc(ctypes.byref(b_na.batch), 1, 0,
                                     torch.cuda.current_stream(cuda).cuda_stream)
    assert rc == -1
    assert b"another batch" in L.hb_last_error()
    torch.cuda.synchronize()
    assert b_na.controls()[0].step == 0
    np.testing.assert_array_equal(b_na.compacted(0)["h"], before)
    # the array still belongs to A: A continues without a prepare
    a_ws.step(3)
    a_na.step_noalloc(1)
    _compare_all(a_ws, a_na)


def test_noalloc_rejects_batches_beyond_its_scratch(cuda):
    import ctypes

    from hipims_b200 import _lib

    a, _ = _pair(cuda)
    big = _lib.HbFusedBatch.from_buffer_copy(a.batch)
    big.n_tiles = 10_000_000  # workspace far beyond the fixed 4 MiB
    L = _lib.lib()
    rc = L.hb_fused_step_noalloc(ctypes.byref(big), 1, 1, None)
    assert rc == -3
    assert b"scratch" in L.hb_last_error()
