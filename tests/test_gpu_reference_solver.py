"""The reference's own solver class, unmodified, on this library's drop-in
modules.

HP/SWE_CUDA.py (staged byte for byte into baseline/_ref/pythonHipims by
baseline/install_ref_py.py) is executed with the 13 extension modules it
imports at load resolved to chans-hipims-flamegpu_b200/<name>.py.  Its
`Godunov` object then runs the loop of CHANS-HiPIMS_server.py:246-256 (flux,
station rain, friction + update + time step; infiltration where the case has
it, as HP/CatchFlood_main.py:164-170 orders it) and is compared with:
  * the golden fixtures made from the reference's own kernels built for the
    host (tests/golden/*.npz), at the tolerances of test_gpu_godunov.py;
  * the oracle on the 256 x 256 dam break, 1000 steps (config 1);
  * the restated solver (hipims_b200.solver.Godunov) on the same ops.
"""
import glob
import os

import numpy as np
import pytest
import torch

import make_golden as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
# as in test_gpu_godunov.py: the bumpy wet/dry mixed-boundary and infiltration
# cases amplify CUDA-vs-glibc pow differences (1e-16) through the scheme's
# thresholds
GOLDEN_ATOL = {"mixed_bc_o2.npz": 1e-4, "urban24_infil_o2.npz": 1e-5}


@pytest.fixture(scope="module")
def RefGodunov(cuda):
    from baseline import ref_loop

    if not ref_loop.available():
        pytest.skip("the reference solver is not staged (python baseline/install_ref_py.py)")
    return ref_loop.load_swe_cuda(ref_loop.b200_modules()).Godunov


def run_reference_loop(cls, d, order, dev, steps, t_end=np.inf, export_step=1e30, outpath=None,
                       dtype=torch.float64):
    g = cls(dev, d["dx"], d["cfl"], export_step, secondOrder=(order == 2),
            firstTimeStep=d["first_dt"], tensorType=dtype)
    if outpath is not None:
        g.setOutPutPath(outpath)
    T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64))
    mask = torch.as_tensor(np.asarray(d["mask"]))
    wl = d.get("wl") if d.get("wl") is not None else np.asarray(d["z"]) + np.asarray(d["h"])
    g.init__fluidField_tensor(mask, T(d["h"]), T(d["qx"]), T(d["qy"]), T(wl), T(d["z"]), dev)
    g.set__frictionField_tensor(torch.as_tensor(np.atleast_1d(d["manning"]), device=dev), dev)
    if d.get("landuse") is not None:
        g.set_landuse(mask, torch.as_tensor(np.asarray(d["landuse"])), dev)
    bl = {}
    for k, key in (("given_depth", "H_GIVEN"), ("given_wl", "WL_GIVEN"), ("given_q", "Q_GIVEN")):
        if d.get(k) is not None:
            bl[key] = np.asarray(d[k])
    g.set_boundary_tensor(bl, dev)
    rm = d.get("rain_mask")
    rm = np.zeros(np.asarray(d["mask"]).shape, np.int16) if rm is None else rm
    g.set_distributed_rainfall_station_Mask(mask, torch.as_tensor(np.asarray(rm)), dev)
    rain = d.get("rain")
    rain = np.array([[0.0, 0.0], [1e9, 0.0]]) if rain is None else np.asarray(rain)
    inf = d.get("infiltration")
    if inf is not None:
        P = lambda a: torch.as_tensor(np.atleast_1d(np.asarray(a, np.float64)), device=dev)
        g.set__infiltrationField_tensor(P(inf["ks"]), P(inf["psi"]), P(inf["dtheta"]), dev)
    n = 0
    while n < steps and g.t.item() < t_end:
        g.addFlux()
        g.addStation_PrecipitationSource(rain, dev)
        if inf is not None:
            g.addInfiltrationSource()
        g.time_friction_euler_update_cuda(dev)
        n += 1
    return g, n


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_reference_solver_on_b200_modules_matches_golden(cuda, RefGodunov, path, tmp_path):
    d, order, exp = G.load_case(path)
    g, n = run_reference_loop(RefGodunov, d, order, cuda, d["steps"], d["t_end"],
                              d["export_step"], outpath=str(tmp_path))
    assert n == int(exp["steps"])
    atol = GOLDEN_ATOL.get(os.path.basename(path), 1e-10)
    assert g.t.item() == pytest.approx(float(exp["t"]), rel=max(atol, 1e-12))
    fields = [("h", g._h_internal), ("qx", g._qx_internal), ("qy", g._qy_internal),
              ("h_max", g._h_max)]
    if "cum" in exp:
        fields.append(("cum", g._cumulativeWaterDepth))
    for k, x in fields:
        np.testing.assert_allclose(x.cpu().numpy(), exp[k], rtol=0, atol=atol, err_msg=k)
    if np.isfinite(d["export_step"]) and d["export_step"] < 1e20 and g._export_n > 0:
        # the reference's own exportField wrote its .pt files
        assert any(f.startswith("h_") for f in os.listdir(str(tmp_path)))


def test_reference_solver_dam_break_1000_steps(cuda, RefGodunov):
    from hipims_b200 import scenarios as S

    d = S.dam_break(256)
    sim = O.Sim(d, order=2)
    sim.run(1000)
    g, n = run_reference_loop(RefGodunov, d, 2, cuda, 1000)
    assert n == 1000
    st = sim.state()
    err = {k: np.abs(x.cpu().numpy() - st[k]).max()
           for k, x in (("h", g._h_internal), ("qx", g._qx_internal), ("qy", g._qy_internal))}
    print("reference Godunov on B200 ops vs oracle after 1000 steps:", err)
    assert g.t.item() == pytest.approx(st["t"], rel=1e-9)
    assert max(err.values()) < 1e-7


@pytest.mark.parametrize("order", [1, 2])
def test_reference_solver_equals_restated_solver(cuda, RefGodunov, order):
    """The reference class and hipims_b200.solver.Godunov, on the same ops and
    the mixed-boundary case, step for step: the same clock and fields."""
    from test_gpu_godunov import run_godunov

    d = G.mixed_bc_case(17, order)
    a, na = run_reference_loop(RefGodunov, d, order, cuda, 40)
    b, nb = run_godunov(d, order, cuda, 40)
    assert na == nb == 40
    assert a.t.item() == pytest.approx(b.t.item(), rel=1e-13)
    for f in ("_h_internal", "_qx_internal", "_qy_internal", "_h_max"):
        np.testing.assert_allclose(getattr(a, f).cpu().numpy(), getattr(b, f).cpu().numpy(),
                                   rtol=0, atol=1e-12, err_msg=f)


@pytest.mark.parametrize("size", [2, 3])
def test_reference_parallel_solver_on_b200_modules(cuda, size):
    """The reference's multi-GPU solver class, unmodified, with its ranks on
    this library's drop-in modules and on the reference's own kernels built
    for sm_100a: the same clock and fields on every rank, and rank strips
    that meet in their overlap rows (1st order, the class's scheme: its
    neighbour table has the 1st-order five rows)."""
    from baseline import ref_gpu, ref_loop
    from hipims_b200 import scenarios as S

    if not ref_loop.available() or not ref_gpu.available():
        pytest.skip("the reference solver or its sm_100a kernels are not staged")
    d = S.urban_catchment(120, dx=2.0, seed=5, rain_mm_h=150.0)
    # a 1 cm sheet everywhere (a rank without wet cells keeps its last time
    # step, HP/Parallel_SWE_CUDA.py:492-494, which the MIN reduction then
    # holds for all) and a pond that spreads across the strip edges
    h0 = np.full(np.asarray(d["mask"]).shape, 0.01)
    h0[20:50, 30:70] = 0.4
    d["h"] = np.where(np.asarray(d["mask"]) > 0, h0, 0.0)
    d["qx"] = np.zeros_like(d["h"])
    d["qy"] = np.zeros_like(d["h"])
    steps = 60
    ours, splits = ref_loop.run_parallel_loop(
        ref_loop.load_parallel_swe(ref_loop.b200_modules()).Parallel_SWE, d, cuda, steps, size)
    theirs, _ = ref_loop.run_parallel_loop(
        ref_loop.load_parallel_swe(ref_loop.reference_kernel_modules()).Parallel_SWE, d, cuda,
        steps, size)
    for a, b in zip(ours, theirs):
        assert a.t.item() == pytest.approx(b.t.item(), rel=1e-12)
        for f in ("_h_internal", "_qx_internal", "_qy_internal", "_h_max"):
            np.testing.assert_allclose(getattr(a, f).cpu().numpy(), getattr(b, f).cpu().numpy(),
                                       rtol=0, atol=1e-9, err_msg=f)
    # the clock advanced well past the first steps, the pond's wave crossed a
    # strip edge, and after the last exchange is received every cell held by
    # two ranks has one value
    assert ours[0].t.item() > 100 * d["first_dt"]
    moving = [int((g._qy_internal.abs() > 1e-3).sum()) for g in ours]
    assert sum(1 for m in moving if m > 0) >= 2, moving
    mask = np.asarray(d["mask"])
    seen = {}
    for r, g in enumerate(ours):
        g.update_overlap_receive()
        a, b = ref_loop.rank_rows(splits, r, size, mask.shape[0])
        rows, cols = np.nonzero(mask[a:b] > 0)
        h = g._h_internal.cpu().numpy()
        for k, (y, x) in enumerate(zip(rows + a, cols)):
            if (y, x) in seen:
                assert seen[(y, x)] == h[k], (r, y, x)
            else:
                seen[(y, x)] = h[k]
    assert len(seen) == int((mask > 0).sum())
