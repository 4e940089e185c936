"""The C-ABI library loads, exports every symbol include/*.h declares, agrees
with the ctypes record layouts, and rejects bad arguments before touching a
GPU.  No compute call needs a GPU here."""
import ctypes
import subprocess

import pytest
import torch

from hipims_b200 import _lib


def test_library_loads_and_layouts_match():
    L = _lib.lib()
    assert L.hb_abi_version() == 1


def test_every_declared_symbol_is_exported():
    declared = _lib.declared_symbols()
    assert "hb_flux" in declared and "hb_fused_step" in declared
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    L = _lib.lib()
    for s in declared:
        assert hasattr(L, s)


@pytest.mark.parametrize("order", [0, 3])
def test_flux_rejects_bad_order(order):
    L = _lib.lib()
    rc = L.hb_flux(order, 1, 1, 1, *([None] * 12), 1, 2, None, 1, 2, None, 1, 3, None, None,
                   None, None)
    assert rc == -1
    assert b"order" in L.hb_last_error()


def test_ops_reject_bad_dtype_and_null():
    L = _lib.lib()
    assert L.hb_flux_mask(7, 10, None, None, None, None, None) == -1
    assert L.hb_flux_mask(1, 10, None, None, None, None, None) == -1
    assert b"null" in L.hb_last_error()
    # empty inputs are a no-op, as in the reference (M == 0 early return)
    assert L.hb_flux(2, 1, 0, 10, *([None] * 12), 1, 2, None, 1, 2, None, 1, 3, None, None,
                     None, None) == 0
    assert L.hb_min_reduce(1, 0, None, None, None, None) == -1


def test_fused_rejects_bad_record():
    L = _lib.lib()
    b = _lib.HbFusedBatch()
    assert L.hb_fused_step(ctypes.byref(b), 1, None) == -1
    assert L.hb_fused_prepare(ctypes.byref(b), None) == -1
    assert L.hb_fused_workspace_size(None) == 0


def test_adjoint_rejects_bad_arguments():
    L = _lib.lib()
    a = _lib.HbAdjointArgs()
    assert ctypes.sizeof(a) == 184
    assert L.hb_adjoint_step(ctypes.byref(a), None) == -1
    assert b"null" in L.hb_last_error()
    assert L.hb_adjoint_gauge(-1, None, None, None, None, 1.0, None) == -1
    assert L.hb_adjoint_gauge(0, None, None, None, None, 1.0, None) == 0
    assert L.hb_adjoint_gauge(3, None, None, None, None, 1.0, None) == -1


def test_state_layout_rejects_bad_arguments():
    L = _lib.lib()
    assert L.hb_state_layout(7, 4, None, 1, *([None] * 6), None) == -1
    assert b"dtype" in L.hb_last_error()
    assert L.hb_state_layout(1, -1, None, 1, *([None] * 6), None) == -1
    assert L.hb_state_layout(1, 0, None, 1, *([None] * 6), None) == 0
    assert L.hb_state_layout(1, 4, None, 0, *([None] * 6), None) == -1
    assert b"null" in L.hb_last_error()


def test_dropin_modules_have_reference_names():
    import euler_update
    import fluxCal_2ndOrder_jh_improved
    import fluxCalculation_jh_modified_surface
    import fluxMask
    import friction_implicit_andUpdate_jh
    import infiltrationCalculation
    import station_PrecipitationCalculation
    import timeControl

    assert callable(fluxCal_2ndOrder_jh_improved.addFlux)
    assert callable(fluxCalculation_jh_modified_surface.addFlux)
    assert callable(friction_implicit_andUpdate_jh.addFriction_eulerUpdate)
    assert callable(timeControl.updateTimestep)
    assert callable(station_PrecipitationCalculation.addStation_Precipitation)
    assert callable(fluxMask.update)
    assert callable(euler_update.update)
    assert callable(infiltrationCalculation.addinfiltration)
    import frictionCalculation
    import sedi_mass_momentum_update

    with pytest.raises(NotImplementedError):
        frictionCalculation.addFriction()
    with pytest.raises(NotImplementedError):
        sedi_mass_momentum_update.add_source()


def test_dropin_ops_check_inputs_like_the_reference():
    """CHECK_INPUT: non-CUDA tensors raise RuntimeError '<name> must be a CUDA tensor.'"""
    import fluxCal_2ndOrder_jh_improved as F

    x = torch.zeros(4, dtype=torch.float64)
    i = torch.zeros(4, dtype=torch.int32)
    with pytest.raises(RuntimeError, match="h must be a CUDA tensor"):
        F.addFlux(i, x, x, x, x, x, x, x, x, i, x, x, x, x, x, x, x)


def test_noalloc_limit_matches_the_documented_tile_counts():
    """hb_fused_step_noalloc keeps its scratch in 4 MiB: the header's limits
    (about 110,000 tiles, about 100,000 with 256 instances; 78,000 and 70,000
    with 64-wide tiles) hold for the workspace size the library computes
    (pure host arithmetic)."""
    L = _lib.lib()

    def size(tiles, instances, tile_x=32):
        b = _lib.HbFusedBatch()
        b.n_tiles, b.n_instances, b.tile_x = tiles, instances, tile_x
        return L.hb_fused_workspace_size(ctypes.byref(b))

    mib4 = 4 << 20
    assert size(110_000, 1) <= mib4 < size(115_000, 1)
    assert size(100_000, 256) <= mib4 < size(105_000, 256)
    # 64-wide tiles keep a 16-byte entry per tile: about 78,000 and 70,000
    assert size(78_000, 1, 64) <= mib4 < size(80_000, 1, 64)
    assert size(70_000, 256, 64) <= mib4 < size(72_000, 256, 64)
    # grows with tiles and instances (regions are 256-byte aligned, so by steps)
    assert size(1000, 1) < size(2000, 1) and size(1000, 1) < size(1000, 8)
