"""The launch-shape autotuner: candidate choice, the JSON cache, the spin-up
before timing (host logic on CPU with a fake timer), and one real tuning run
on the GPU."""
import numpy as np
import pytest
import torch

from hipims_b200 import autotune
from hipims_b200.fused import Catchment


def _catchments(n=2, side=48):
    out = []
    for k in range(n):
        mask = np.ones((side + 8 * k, side), np.int32)
        mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = 50
        z = np.zeros(mask.shape)
        h = np.full(mask.shape, 0.1)
        out.append(Catchment(mask=mask, z=z, h=h, rain=np.array([[0.0, 1e-5], [1e6, 1e-5]])))
    return out


@pytest.fixture
def fake_gpu(monkeypatch, tmp_path):
    monkeypatch.setenv("HIPIMS_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda device=None: "FakeGPU")
    return tmp_path / "tune.json"


def test_tune_picks_fastest_and_caches(fake_gpu, monkeypatch):
    times = {((32, 64), 4): 1.15, ((32, 64), 3): 1.20, ((64, 32), 4): 1.53,
             ((32, 32), 5): 1.33, ((32, 32), 6): 1.05}
    calls = []

    def fake_time(cs, dtype, device, cfg, steps=6, warmup=autotune.SPINUP_STEPS):
        calls.append((tuple(cfg["tile"]), cfg["minb"], warmup))
        return times[(tuple(cfg["tile"]), cfg["minb"])]

    monkeypatch.setattr(autotune, "time_config", fake_time)
    cs = _catchments()
    best = autotune.tune(cs, torch.float32, "cpu", steps=4)
    assert best["tile"] == (32, 32) and best["minb"] == 6
    assert len(calls) == len(autotune.DEFAULT_CANDIDATES)
    assert fake_gpu.exists()
    # a second call reads the cache and times nothing
    calls.clear()
    again = autotune.tune(cs, torch.float32, "cpu", steps=4)
    assert calls == [] and again["tile"] == (32, 32) and again["minb"] == 6
    # another batch shape is another key
    autotune.tune(_catchments(3), torch.float32, "cpu", steps=4)
    assert len(calls) == len(autotune.DEFAULT_CANDIDATES)


def test_tune_key_carries_the_spinup(fake_gpu):
    key = autotune.batch_key(_catchments(), torch.float32, "cpu")
    assert key.startswith("FakeGPU|float32|n=2|")
    assert key.endswith(f"|spinup={autotune.SPINUP_STEPS}")


def test_candidates_are_timed_after_a_spinup():
    # the first steps of a dry start do not represent a run: the default
    # warm-up of a candidate's timing is the spin-up
    import inspect

    sig = inspect.signature(autotune.time_config)
    assert sig.parameters["warmup"].default == autotune.SPINUP_STEPS >= 8


def test_fp64_has_one_shape(fake_gpu):
    assert autotune.tune(_catchments(), torch.float64, "cpu") == {"tile": (32, 32)}


def test_cells_per_lane():
    assert [autotune.cells_per_lane(c) for c in autotune.DEFAULT_CANDIDATES] == [2, 2, 1, 1, 1]


@pytest.mark.gpu
def test_tune_on_gpu(cuda, tmp_path, monkeypatch):
    from hipims_b200.fused import FusedSolver

    monkeypatch.setenv("HIPIMS_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    cs = _catchments()
    best = autotune.tune(cs, torch.float32, cuda, steps=2)
    shapes = {(tuple(c["tile"]), c["minb"]) for c in autotune.DEFAULT_CANDIDATES}
    assert (tuple(best["tile"]), best["minb"]) in shapes
    assert len(best["tried"]) == len(autotune.DEFAULT_CANDIDATES)
    assert all(ms > 0 for _, ms in best["tried"])
    fs = FusedSolver(cs, dtype=torch.float32, device=cuda, tile=best["tile"], minb=best["minb"])
    fs.step(4)
    fs.check()
    for k in range(len(cs)):
        h = fs.state(k)["h"].cpu().numpy()
        assert np.all(np.isfinite(h)) and h.min() >= 0.0
