"""The coupling RPC contract (CHANS-HiPIMS/CHANS-HiPIMS_server.py:269-341)
over loopback msgpack-RPC, with a fake simulation backend on the CPU and the
fused solver on the GPU."""
import threading
import time

import numpy as np
import pytest

from hipims_b200.coupling import HiPIMSService, RPCClient, serve_in_thread


class FakeBackend:
    """t advances in 0.7 s steps; the 'depth' at agent k is t * (k + 1)."""

    def __init__(self, n=5, delay=0.0):
        self.t = 0.0
        self.n = n
        self.delay = delay
        self.steps = 0

    def current_time(self):
        return self.t

    def advance_to(self, target):
        while self.t < target:
            time.sleep(self.delay)
            self.t += 0.7
            self.steps += 1

    def gather(self):
        return [self.t * (k + 1) for k in range(self.n)]

    def reset(self):
        self.t = 0.0


@pytest.fixture()
def server():
    svc = HiPIMSService(FakeBackend(delay=0.001))
    srv, stop = serve_in_thread(svc, port=0)
    yield svc, srv.server_address[1]
    stop()


def test_request_data_advances_and_returns_latest(server):
    svc, port = server
    c = RPCClient(port=port)
    out = c.call("request_data", 120)
    t = svc.backend.t
    assert t >= 120 and t < 120.7 + 1e-9
    assert out == pytest.approx([t * (k + 1) for k in range(5)])
    assert svc.current_time == int(t)
    assert c.call("echo", [1, "a"]) == [1, "a"]
    # a request for a time already reached does not advance
    steps = svc.backend.steps
    assert c.call("request_data", 100) == pytest.approx(out)
    assert svc.backend.steps == steps
    c.close()


def test_set_target_in_the_past_raises_wrong_time(server):
    svc, port = server
    c = RPCClient(port=port)
    c.call("request_data", 60)
    with pytest.raises(RuntimeError, match="Wrong Time"):
        c.call("set_target", 10)
    c.call("set_target", 90, True)
    assert c.call("get_latest_data") == pytest.approx(svc.backend.gather())
    assert svc.backend.t >= 90
    c.call("reset_simulation")
    assert svc.current_time == 0 and svc.target_time == 0
    c.close()


def test_concurrent_clients_wait_without_spinning(server):
    svc, port = server
    results = []

    def worker():
        c = RPCClient(port=port)
        results.append(c.call("request_data", 30))
        c.close()

    ths = [threading.Thread(target=worker) for _ in range(4)]
    for th in ths:
        th.start()
    for th in ths:
        th.join(30)
    assert len(results) == 4
    for r in results:
        assert r == pytest.approx(results[0]) or r[0] >= results[0][0]


def test_unknown_method_is_an_error(server):
    _, port = server
    c = RPCClient(port=port)
    with pytest.raises(RuntimeError, match="no method"):
        c.call("drop_tables")
    c.close()


@pytest.mark.gpu
def test_rpc_over_fused_solver_matches_direct_gather(cuda):
    import torch

    from hipims_b200 import scenarios as S
    from hipims_b200.coupling import FusedBackend
    from hipims_b200.fused import FusedSolver
    from hipims_b200.scenarios import catchment_from

    d = S.urban_catchment(96, seed=5, rain_mm_h=300.0)
    pos = np.argwhere(d["mask"] > 0)
    ids = np.sort(np.random.default_rng(1).choice(len(pos), 200, replace=False))
    fs = FusedSolver(catchment_from(d), dtype=torch.float32, device=cuda)
    svc = HiPIMSService(FusedBackend(fs, pos[ids, 0], pos[ids, 1]))
    srv, stop = serve_in_thread(svc, port=0)
    try:
        c = RPCClient(port=srv.server_address[1])
        out = np.asarray(c.call("request_data", 60))
        c.close()
    finally:
        stop()
    assert fs.controls()[0].t >= 60
    ref = fs.compacted()["h"][ids]
    np.testing.assert_array_equal(out, ref)
