"""HostStepper (state held in pinned host memory, one fused step per call,
inbound and outbound copies overlapped across steps) against the same batch
stepped on the device: bitwise equal fields and equal clocks after every step,
with the host state in the reference's compacted layout (hb_state_layout
between it and the dense arrays) and in the dense layout."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _host_field(hst, buf, k):
    """A host buffer's cells of instance k in the compacted (row-major valid)
    order, as float64."""
    if hst.layout == "dense":
        return hst.raster(buf, k).numpy()[hst.fs.inst[k].valid].astype(np.float64)
    return buf.numpy().astype(np.float64)


@pytest.mark.parametrize("layout", ["compact", "dense"])
def test_host_stepper_equals_device_steps(cuda, layout):
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver, HostStepper

    ds = [S.urban_catchment(n, seed=k + 4, rain_mm_h=120.0) for k, n in enumerate((96, 150))]
    cs = [S.catchment_from(d) for d in ds]
    dev_run = FusedSolver(cs, dtype=torch.float32, device=cuda)
    host_run = FusedSolver(cs, dtype=torch.float32, device=cuda)
    dev_run.step(3)
    host_run.step(3)  # wet the catchments; both start the host loop from the same state
    hst = HostStepper(host_run, layout=layout)
    for step in range(6):
        dev_run.step(1)
        hst.step()
        hst.finish()
        torch.cuda.synchronize(cuda)
        for k in range(len(cs)):
            want = dev_run.compacted(k)
            for f, buf in zip(("h", "qx", "qy"), hst.out_buffers[3 * k:3 * k + 3]):
                np.testing.assert_array_equal(_host_field(hst, buf, k), want[f],
                                              err_msg=f"instance {k} field {f} step {step}")
            assert host_run.controls()[k].t == dev_run.controls()[k].t
        # the host loop: this step's result is the next step's input
        for src, dst in zip(hst.out_buffers, hst.in_buffers):
            dst.copy_(src)


@pytest.mark.parametrize("layout", ["compact", "dense"])
def test_host_stepper_async_steps_match_device(cuda, layout):
    """Several steps enqueued back to back (the overlapped form) with the input
    buffers left unchanged: every step restarts from the same state while the
    clock runs on.  The same sequence on the device (state reset before each
    step) must give the same last result and clock."""
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver, HostStepper

    d = S.urban_catchment(128, seed=9, rain_mm_h=150.0)
    c = S.catchment_from(d)
    a = FusedSolver(c, dtype=torch.float32, device=cuda)
    b = FusedSolver(c, dtype=torch.float32, device=cuda)
    a.step(4)
    b.step(4)
    cur = a.controls()[0].cur
    ins = a.inst[0]
    start = [x.clone() for x in (ins.h[cur], ins.qx[cur], ins.qy[cur])]
    hst = HostStepper(b, layout=layout)
    for _ in range(5):
        hst.step()
    hst.finish()
    torch.cuda.synchronize(cuda)
    for _ in range(5):
        cur = a.controls()[0].cur
        for x, s0 in zip((ins.h[cur], ins.qx[cur], ins.qy[cur]), start):
            x.copy_(s0)
        a.step(1)
    want = a.compacted(0)
    for f, buf in zip(("h", "qx", "qy"), hst.out_buffers):
        np.testing.assert_array_equal(_host_field(hst, buf, 0), want[f], err_msg=f)
    assert b.controls()[0].t == a.controls()[0].t
    assert b.controls()[0].step == a.controls()[0].step
