"""Row-strip decomposition of one catchment.

CPU: the row split, and the halo exchange and clock reduction of the
multi-rank path between two gloo ranks on CPU tensors.  GPU: strips of one
catchment on one device reproduce the undivided fused run bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from hipims_b200.strips import HALO, exchange_halos, split_rows


def test_split_rows_aligned_and_covering():
    for n, p in [(194, 2), (194, 3), (2050, 4), (10, 3), (300, 1)]:
        r = split_rows(n, p)
        assert r[0][0] == 0 and r[-1][1] == n and len(r) == p
        assert all(b - a >= 3 for a, b in r)
        assert all(r[k][1] == r[k + 1][0] for k in range(p - 1))
    assert [a for a, _ in split_rows(2050, 4)] == [0, 512, 1024, 1536]
    with pytest.raises(ValueError):
        split_rows(5, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, rows, pitch, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        # field f of rank r: value 1000 r + 100 f + padded row index (halos -1)
        fields = []
        for f in range(3):
            F = torch.full((rows + 2 * HALO + 3, pitch), -1.0, dtype=torch.float64)
            for pr in range(HALO, HALO + rows):
                F[pr] = 1000 * rank + 100 * f + pr
            fields.append(F)
        exchange_halos(fields, rows, rank, world)
        ext = torch.tensor([float(rank + 1), float(rank == 0)], dtype=torch.float64)
        dist.all_reduce(ext, op=dist.ReduceOp.MAX)
        q.put((rank, [F.numpy().copy() for F in fields], ext.numpy().copy()))
    finally:
        dist.destroy_process_group()


def test_halo_exchange_and_clock_reduction_gloo():
    world, rows, pitch = 2, 6, 8
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, rows, pitch, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, fields, ext = q.get(timeout=120)
        res[rank] = (fields, ext)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        fields, ext = res[r]
        np.testing.assert_array_equal(ext, [world, 1.0])
        for f, F in enumerate(fields):
            if r > 0:  # top halo = rank r-1's last two rows (padded rows rows, rows + 1)
                for j in range(HALO):
                    assert np.all(F[j] == 1000 * (r - 1) + 100 * f + rows + j)
            else:
                assert np.all(F[0:HALO] == -1.0)
            if r < world - 1:  # bottom halo = rank r+1's first two rows (padded HALO, HALO+1)
                for j in range(HALO):
                    assert np.all(F[HALO + rows + j] == 1000 * (r + 1) + 100 * f + HALO + j)
            else:
                assert np.all(F[HALO + rows:HALO + rows + HALO] == -1.0)
            for pr in range(HALO, HALO + rows):  # own rows untouched
                assert np.all(F[pr] == 1000 * r + 100 * f + pr)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("parts", [2, 3])
@pytest.mark.parametrize("forward", [True, False])
def test_strips_reproduce_the_undivided_run(cuda, dtype, parts, forward):
    """forward: the step kernel writes the neighbours' halo rows; otherwise a
    halo copy before every step."""
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver
    from hipims_b200.strips import StripSolver

    d = S.urban_catchment(192, dx=2.0, seed=8, rain_mm_h=120.0)
    c = S.catchment_from(d)
    one = FusedSolver(c, dtype=dtype, device=cuda, origin=(0, 0))  # the strips' tile grid
    st = StripSolver(c, parts, dtype=dtype, device=cuda, forward_halos=forward)
    for _ in range(3):
        one.step(20)
        st.step(20)
        a, b = one.state(), st.state()
        for f in ("h", "qx", "qy", "h_max"):
            assert torch.equal(a[f], b[f]), f
        c1 = one.controls()[0]
        for cs in st.controls():
            assert (cs.t, cs.dt, cs.step) == (c1.t, c1.dt, c1.step)
    vol = sum(cs.volume for cs in st.controls())
    assert vol == pytest.approx(one.controls()[0].volume, rel=1e-12)


def _peer_rank_main(rank, world, port, q):
    """One strip per process, both on GPU 0, gloo for the host-side
    collectives; the step kernels write each other's halo rows through CUDA
    IPC mappings.  No kernel waits on another: the clock all_reduce between
    steps orders them."""
    import torch.distributed as dist

    from hipims_b200 import scenarios as S
    from hipims_b200.strips import DistributedStrips

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        dev = torch.device("cuda", 0)
        d = S.urban_catchment(160, dx=2.0, seed=11, rain_mm_h=120.0)
        ds = DistributedStrips(S.catchment_from(d), rank, world, dtype=torch.float32,
                               device=dev, peer=True)
        ds.step(30)
        torch.cuda.synchronize(dev)
        st = ds.fs.state(0)
        c = ds.fs.controls()[0]
        q.put((rank, {f: st[f].cpu().numpy().copy() for f in ("h", "qx", "qy", "h_max")},
               (c.t, c.dt, c.step)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_peer_strips_on_one_device_reproduce_the_undivided_run(cuda):
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_peer_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, fields, clock = q.get(timeout=300)
        res[rank] = (fields, clock)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    d = S.urban_catchment(160, dx=2.0, seed=11, rain_mm_h=120.0)
    one = FusedSolver(S.catchment_from(d), dtype=torch.float32, device=cuda, origin=(0, 0))
    one.step(30)
    want = one.state(0)
    c1 = one.controls()[0]
    for f in ("h", "qx", "qy", "h_max"):
        got = np.concatenate([res[r][0][f] for r in range(world)], axis=0)
        np.testing.assert_array_equal(got, want[f].cpu().numpy(), err_msg=f)
    for r in range(world):
        assert res[r][1] == (c1.t, c1.dt, c1.step)
