"""Coupling to the FLAMEGPU household model over msgpack-RPC.

Keeps the contract of the reference's HiPIMS RPC server
(CHANS-HiPIMS/CHANS-HiPIMS_server.py:269-341), which the FLAMEGPU client calls
through rpclib every 120 ABM iterations
(CHANS-FLAMEGPU/CHANS-FLAMEGPU/CHANS_ABM/src/model/functions.c:63-100):

  request_data(time)            advance to `time` if ahead, return the depths at
                                the agent cells (list of float, compacted order)
  set_target(target, sync=True) raise "Wrong Time" if target < current time
  get_latest_data()             depths of the latest step
  sync_to_target_time()         run the solver until the target in a thread
  reset_simulation()            target = current = 0
  echo(x)                       x

Differences from the reference, none visible to the client: the server uses
the standard library and `msgpack` (mprpc/gevent are not needed); callers
wait on a threading.Event instead of spinning on `running_simulation`; the
depths are gathered on the device (hb_gather) and copied to the host once,
instead of `h[idx_target_ABM1].cpu()` after every step.
"""
from __future__ import annotations

import socketserver
import threading
from typing import Any, Callable, Protocol

import msgpack
import numpy as np
import torch

from . import ops
from .fused import FusedSolver

REQUEST, RESPONSE, NOTIFY = 0, 1, 2


class Backend(Protocol):
    def current_time(self) -> float: ...
    def advance_to(self, target: float) -> None: ...
    def gather(self) -> list: ...
    def reset(self) -> None: ...


class FusedBackend:
    """A FusedSolver instance plus the agent cells to report.

    agent_rows / agent_cols: raster positions of the agent cells, in the
    order the reference reports them (ascending compacted id = row-major order
    of the valid cells, `CHANS-HiPIMS_server.py:140-153`).  The reference
    server runs the 1st-order scheme (its `'secondOrder': False`): build the
    solver with `FusedSolver(..., order=1)` to match it.
    """

    def __init__(self, solver: FusedSolver, agent_rows, agent_cols, instance: int = 0,
                 velocities: bool = False, chunk: int = 64):
        self.fs = solver
        self.k = instance
        self.velocities = velocities
        self.chunk = chunk
        self.offsets = solver.cell_offsets(instance, np.asarray(agent_rows),
                                           np.asarray(agent_cols))
        self._t0 = solver.controls()[instance].t

    def current_time(self) -> float:
        return float(self.fs.controls()[self.k].t)

    def advance_to(self, target: float) -> None:
        if self.current_time() < target:
            self.fs.run_until(target, chunk=self.chunk)

    def gather(self) -> list:
        h, qx, qy = self.fs.current(self.k)
        if self.velocities:
            gh, gu, gv = ops.gather(self.offsets, h, qx, qy, velocities=True)
            out = torch.stack([gh, gu, gv], dim=1)
        else:
            out = ops.gather(self.offsets, h)
        return out.double().cpu().numpy().tolist()

    def reset(self) -> None:
        pass


class HiPIMSService:
    """The RPC methods of the reference server, over a simulation backend."""

    def __init__(self, backend: Backend):
        self.backend = backend
        self.target_time = 0
        self.current_time = 0
        self._idle = threading.Event()
        self._idle.set()
        self._lock = threading.Lock()
        self._error: BaseException | None = None
        self._results: list = backend.gather()

    # -- helpers --------------------------------------------------------
    def _wait_idle(self, timeout: float | None = None) -> None:
        if not self._idle.wait(timeout):
            raise TimeoutError("simulation still running")
        if self._error is not None:
            err, self._error = self._error, None
            raise RuntimeError(f"simulation failed: {err}")

    def _run_loop(self) -> None:
        try:
            self.backend.advance_to(float(self.target_time))
            self.current_time = int(self.backend.current_time())
            self._results = self.backend.gather()
        except BaseException as e:  # reported to the next caller
            self._error = e
        finally:
            self._idle.set()

    # -- RPC methods (CHANS-HiPIMS_server.py:287-335) --------------------
    def get_latest_data(self):
        self._wait_idle()
        return self._results

    def sync_to_target_time(self):
        with self._lock:
            self._wait_idle()
            self._idle.clear()
            threading.Thread(target=self._run_loop, daemon=True).start()

    def set_target(self, target_time, sync=True):
        target_time = int(target_time)
        if target_time < self.current_time:
            raise Exception("Wrong Time")
        self.target_time = target_time
        if sync:
            self.sync_to_target_time()

    def request_data(self, time):
        time = int(time)
        if time > self.current_time:
            self.set_target(time)
        self._wait_idle()
        return list(self.get_latest_data())

    def reset_simulation(self):
        self._wait_idle()
        self.target_time = 0
        self.current_time = 0
        self.backend.reset()

    def echo(self, x):
        return x

    METHODS = ("request_data", "set_target", "get_latest_data", "sync_to_target_time",
               "reset_simulation", "echo")

    def dispatch(self, method: str, params: list) -> Any:
        if method not in self.METHODS:
            raise AttributeError(f"no method {method!r}")
        return getattr(self, method)(*params)


class _Handler(socketserver.BaseRequestHandler):
    def handle(self) -> None:
        service: HiPIMSService = self.server.service  # type: ignore[attr-defined]
        unpacker = msgpack.Unpacker(raw=False, strict_map_key=False)
        sock = self.request
        while True:
            data = sock.recv(1 << 16)
            if not data:
                return
            unpacker.feed(data)
            for msg in unpacker:
                if not isinstance(msg, (list, tuple)) or not msg:
                    continue
                if msg[0] == REQUEST and len(msg) == 4:
                    _, msgid, method, params = msg
                    try:
                        result, error = service.dispatch(method, list(params)), None
                    except Exception as e:  # noqa: BLE001 - sent to the client
                        result, error = None, str(e)
                    sock.sendall(msgpack.packb([RESPONSE, msgid, error, result],
                                               use_bin_type=True))
                elif msg[0] == NOTIFY and len(msg) == 3:
                    try:
                        service.dispatch(msg[1], list(msg[2]))
                    except Exception:  # noqa: BLE001 - notifications have no reply
                        pass


class RPCServer(socketserver.ThreadingTCPServer):
    """msgpack-RPC server of a HiPIMSService (default 127.0.0.1:6060 as the
    reference, CHANS-HiPIMS_server.py:338-341)."""

    allow_reuse_address = True
    daemon_threads = True

    def __init__(self, service: HiPIMSService, host: str = "127.0.0.1", port: int = 6060):
        super().__init__((host, port), _Handler)
        self.service = service


class RPCClient:
    """Minimal msgpack-RPC client (the calls rpclib::client makes)."""

    def __init__(self, host: str = "127.0.0.1", port: int = 6060, timeout: float = 60.0):
        import socket

        self.sock = socket.create_connection((host, port), timeout=timeout)
        self.unpacker = msgpack.Unpacker(raw=False, strict_map_key=False)
        self.msgid = 0

    def call(self, method: str, *params) -> Any:
        self.msgid += 1
        self.sock.sendall(msgpack.packb([REQUEST, self.msgid, method, list(params)],
                                        use_bin_type=True))
        while True:
            for msg in self.unpacker:
                if msg[0] == RESPONSE and msg[1] == self.msgid:
                    if msg[2] is not None:
                        raise RuntimeError(msg[2])
                    return msg[3]
            data = self.sock.recv(1 << 16)
            if not data:
                raise ConnectionError("server closed the connection")
            self.unpacker.feed(data)

    def close(self) -> None:
        self.sock.close()


def serve_in_thread(service: HiPIMSService, port: int = 0,
                    host: str = "127.0.0.1") -> tuple[RPCServer, Callable[[], None]]:
    """Start a server on a background thread; returns (server, stop)."""
    srv = RPCServer(service, host, port)
    th = threading.Thread(target=srv.serve_forever, daemon=True)
    th.start()

    def stop() -> None:
        srv.shutdown()
        srv.server_close()

    return srv, stop
