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
