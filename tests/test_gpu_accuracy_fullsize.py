"""FP32 against FP64 on the full 2048 x 2048 urban storm (config 2), the FP64
run's time-step schedule replayed, with the stated tolerance of the FP32
product:

  * max |h32 - h64| <= 1e-4 m at every one of the first 48 steps;
  * at most 0.1 % of the 4.2 M cells beyond 1e-5 m at every one of 256 steps
    (p99.9 of |h32 - h64| <= 1e-5 m);
  * the FP64 volume balance of the FP32 run closes to 1e-7 of the rain.

Printed beside them: the horizon up to which the scheme itself resolves
1e-5 m (the FP64 run with its bed scaled by 1 + 1e-15 stays within 1e-5 m of
the unperturbed one) and the first step at which FP32 departs by more than
1e-4 m.  The north-star form of the tolerance (1e-4 m in the max norm up to
that horizon, 124 steps here) is not met: draining films on bumps lose ~1e-5
of their outflow per step to FP32 rounding of the cell's free surface
against its edge bed (ulp of a 0.05 m offset), and the reference scheme's
own negative-depth oscillation in such cells then lets the two runs part
(first departure beyond 1e-4 m near step 64).

The three runs advance in lockstep on the device; nothing is copied back per
step but a few scalars."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

STEPS = 256
MAX_STEPS = 48      # steps over which the max-norm tolerance holds
TOL_MAX = 1e-4
TOL_TAIL = 1e-5     # p99.9 bound
TAIL_FRACTION = 1e-3
SENS_LIMIT = 1e-5


def test_fp32_tracks_fp64_on_the_2048_storm(cuda):
    from hipims_b200 import scenarios as S
    from hipims_b200.fused import FusedSolver
    from hipims_b200.scenarios import catchment_from

    d = S.urban_catchment(2048, dx=2.0, seed=0)
    f64 = FusedSolver(catchment_from(d), dtype=torch.float64, device=cuda, tile=(32, 32))
    dts = []
    for _ in range(STEPS):
        f64.step(1)
        dts.append(f64.controls()[0].dt)
    del f64
    dts = np.asarray(dts)
    ref = FusedSolver(catchment_from(d), dtype=torch.float64, device=cuda, tile=(32, 32))
    zp = np.asarray(d["z"], dtype=np.float64) * (1.0 + 1e-15)
    per = FusedSolver(catchment_from(d, z=zp, dt_replay=dts), dtype=torch.float64, device=cuda,
                      tile=(32, 32))
    f32 = FusedSolver(catchment_from(d, dt_replay=dts), dtype=torch.float32, device=cuda)
    valid = torch.as_tensor(f32.inst[0].valid, device=cuda)
    n_valid = int(valid.sum())
    allowed = int(TAIL_FRACTION * n_valid)  # cells beyond the p99.9 bound
    sens, err, over = [], [], []
    for _ in range(STEPS):
        ref.step(1)
        per.step(1)
        f32.step(1)
        h = ref.state(0)["h"]
        dp = torch.where(valid, (per.state(0)["h"] - h).abs(), torch.zeros_like(h))
        d32 = torch.where(valid, (f32.state(0)["h"].double() - h).abs(), torch.zeros_like(h))
        sens.append(dp.max())
        err.append(d32.max())
        over.append((d32 > TOL_TAIL).sum())
    sens = torch.stack(sens).cpu().numpy()
    err = torch.stack(err).cpu().numpy()
    over = torch.stack(over).cpu().numpy()
    horizon = int(np.argmax(sens > SENS_LIMIT)) if (sens > SENS_LIMIT).any() else STEPS
    first = int(np.argmax(err > TOL_MAX)) + 1 if (err > TOL_MAX).any() else None
    print(f"FP64 self-sensitivity <= {SENS_LIMIT} m for {horizon} steps; FP32 max |dh| over "
          f"the first {MAX_STEPS} steps {err[:MAX_STEPS].max():.3e} m, first step beyond "
          f"{TOL_MAX} m: {first}, over all {STEPS} steps {err.max():.3e} m; cells beyond "
          f"{TOL_TAIL} m at most {over.max()} of {n_valid}")
    assert err[:MAX_STEPS].max() <= TOL_MAX
    assert over.max() <= allowed
    c = f32.controls()[0]
    bal = abs(c.volume - c.volume0 - c.rain_volume + c.outflow_volume) / c.rain_volume
    assert bal < 1e-7, bal
