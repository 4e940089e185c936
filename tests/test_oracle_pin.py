"""Pin the CPU oracle: the restatement must reproduce the reference's own
kernels (compiled for the host) bit for bit, on the committed golden fixtures
and, when oracle/_ref is built, on fresh cases."""
import glob
import os

import numpy as np
import pytest

import make_golden as G
from oracle import oracle as O

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
FIELDS = ("h", "qx", "qy", "wl", "h_max")


def test_golden_fixtures_exist():
    names = {os.path.basename(p) for p in GOLDEN}
    for n in ("dam_break48_o2.npz", "channel_o2.npz", "mixed_bc_o2.npz", "mixed_bc_o1.npz"):
        assert n in names


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_matches_golden(path):
    d, order, exp = G.load_case(path)
    sim = O.Sim(d, order=order, backend="oracle", export_step=d["export_step"])
    n = sim.run(d["steps"], d["t_end"])
    st = sim.state()
    assert n == int(exp["steps"])
    assert st["t"] == float(exp["t"]) and st["dt"] == float(exp["dt"])
    assert sim.g.exports == int(exp["exports"])
    for k in FIELDS + (("cum",) if "cum" in exp else ()):
        np.testing.assert_array_equal(st[k], exp[k], err_msg=k)


needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_matches_reference_build(order, seed):
    d = G.mixed_bc_case(100 + seed, order)
    a = O.Sim(d, order=order, backend="oracle", export_step=d["export_step"])
    b = O.Sim(d, order=order, backend="ref", export_step=d["export_step"])
    a.run(40)
    b.run(40)
    sa, sb = a.state(), b.state()
    assert sa["t"] == sb["t"]
    for k in FIELDS:
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=k)


@needs_ref
def test_single_kernels_match_reference_build():
    """Each kernel alone, on one random state, against the reference kernel."""
    import ctypes

    d = G.mixed_bc_case(7, 2)
    a = O.Sim(d, order=2)
    R = O.ref_lib()
    N = a.N
    rng = np.random.default_rng(0)
    wet = np.arange(N, dtype=np.int32)
    for order, sym in ((2, "ref_flux2"), (1, "ref_flux1")):
        out_o = [np.zeros(N) for _ in range(3)]
        out_r = [np.zeros(N) for _ in range(3)]
        O.flux(order, wet, *out_o, a.h, a.wl, a.z, a.qx, a.qy, a.index, a.normal, a.gd, a.gw,
               a.gq, 0.5, 0.3, 0.01)
        dx, t, dt = (ctypes.c_double(v) for v in (0.5, 0.3, 0.01))
        P = lambda x: x.ctypes.data
        getattr(R, sym)(N, N, a.gd.shape[1], a.gd.shape[0], a.gw.shape[1], a.gw.shape[0],
                        a.gq.shape[1], a.gq.shape[0], ctypes.c_void_p(P(wet)),
                        *(ctypes.c_void_p(P(x)) for x in (a.h, a.wl, a.z, a.qx, a.qy, a.index,
                                                          a.normal, a.gd, a.gw, a.gq)),
                        ctypes.byref(dx), ctypes.byref(t), ctypes.byref(dt),
                        *(ctypes.c_void_p(P(x)) for x in out_r))
        for x, y in zip(out_o, out_r):
            np.testing.assert_array_equal(x, y)
    assert rng is not None


def test_topology_pin_backcase():
    """HP/backCase.ipynb prints torch.Size([5, 5625]) for its 27 x 227 raster."""
    from hipims_b200 import scenarios as S

    c = S.channel()
    assert c["mask"].shape == (27, 227)
    idx = O.build_index(c["mask"].astype(np.int32))
    assert idx.size == 5 * 5625


def test_physics_lake_at_rest():
    """Flat free surface over a bumpy bed, closed walls: stays at rest."""
    from hipims_b200 import scenarios as S

    d = S.dam_break(32, ring_code=30)
    rng = np.random.default_rng(3)
    z = rng.uniform(0.0, 0.5, d["mask"].shape)
    d["z"] = z
    d["h"] = np.where(d["mask"] > 0, 1.0 - z, 0.0)
    d["wl"] = d["z"] + d["h"]
    sim = O.Sim(d, order=2)
    sim.run(200)
    st = sim.state()
    assert np.abs(st["qx"]).max() < 1e-12 and np.abs(st["qy"]).max() < 1e-12
    assert np.abs(st["h"] + sim.z - 1.0).max() < 1e-12


def test_physics_mass_conservation_walls():
    from hipims_b200 import scenarios as S

    d = S.dam_break(32, ring_code=40)
    sim = O.Sim(d, order=2)
    v0 = sim.h.sum()
    sim.run(300)
    assert abs(sim.h.sum() - v0) / v0 < 1e-12


def test_physics_rain_in_closed_box():
    from hipims_b200 import scenarios as S

    d = S.dam_break(16, ring_code=30)
    d["h"] = np.where(d["mask"] > 0, 0.1, 0.0)
    d["rain"] = np.array([[0.0, 1e-3], [1000.0, 1e-3]])
    d["rain_mask"] = np.zeros(d["mask"].shape, np.int16)
    sim = O.Sim(d, order=2)
    v0 = sim.h.sum()
    t0 = sim.t
    total = 0.0
    for _ in range(50):
        total += 1e-3 * sim.dt * sim.N
        sim.step()
    assert abs((sim.h.sum() - v0) - total) / total < 1e-10
    assert sim.t > t0


@needs_ref
def test_oracle_infiltration_step_matches_reference_build():
    """The step with Green-Ampt infiltration (flux, rain, infiltration,
    friction: HP/CatchFlood_main.py:164-170) bit for bit against the
    reference's kernels built for the host, on two soil zones."""
    from hipims_b200 import scenarios as S

    d = S.urban_catchment(40, dx=2.0, seed=2)
    d["infiltration"] = dict(ks=[2.0e-6, 5.0e-6], psi=[0.11, 0.2], dtheta=[0.3, 0.45])
    a, b = O.Sim(d, order=2), O.Sim(d, order=2, backend="ref")
    a.run(150)
    b.run(150)
    sa, sb = a.state(), b.state()
    for f in ("h", "qx", "qy", "cum"):
        np.testing.assert_array_equal(sa[f], sb[f])
    assert sa["cum"].max() > 1e-3


def random_case(seed: int, order: int) -> dict:
    """A small catchment of random shape: a smoothed-noise no-data mask (holes,
    one-cell channels, ragged edges), 0-5 boxes of random boundary types on its
    ring, a random bed, wet/dry mix and discharges, two Manning zones, rain,
    and boundary tables with columns for every id a box can take (a missing
    column is read past the row by the reference, which is undefined)."""
    from hipims_b200.topology import boundary_codes

    rng = np.random.default_rng(seed)
    ny, nx = int(rng.integers(3, 30)), int(rng.integers(3, 30))
    f = rng.normal(size=(ny + 2, nx + 2))
    for _ in range(2):
        f = (f + np.roll(f, 1, 0) + np.roll(f, -1, 0) + np.roll(f, 1, 1) + np.roll(f, -1, 1)) / 5
    nodata = f < np.quantile(f, rng.uniform(0.0, 0.45))
    nodata[0, :] = nodata[-1, :] = nodata[:, 0] = nodata[:, -1] = True
    if (~nodata).sum() < 2:
        nodata[1:-1, 1:-1] = False
    types = [3, 4, 5, 6, 7, 8] + ([9] if order == 1 else [])
    boxes = []
    for _ in range(int(rng.integers(0, 6))):
        r0, c0 = int(rng.integers(0, ny + 2)), int(rng.integers(0, nx + 2))
        boxes.append((r0, r0 + int(rng.integers(1, 8)), c0, c0 + int(rng.integers(1, 8)),
                      int(rng.choice(types))))
    mask = boundary_codes(nodata, default_bc=int(rng.choice([30, 40, 50])), boxes=boxes)
    z = rng.uniform(0.0, 0.5, mask.shape)
    h = np.where(rng.uniform(size=mask.shape) < 0.6, rng.uniform(0.0, 0.5, mask.shape), 0.0)
    qx = rng.normal(0.0, 0.05, mask.shape) * (h > 0)
    qy = rng.normal(0.0, 0.05, mask.shape) * (h > 0)
    h[nodata] = qx[nodata] = qy[nodata] = 0.0
    times = np.array([[0.0], [100.0]])
    return dict(mask=mask, z=z, h=h, qx=qx, qy=qy, wl=z + h,
                landuse=(rng.uniform(size=mask.shape) < 0.5).astype(np.uint8),
                manning=[0.02, 0.06], dx=float(rng.uniform(0.5, 2.0)), cfl=0.5, first_dt=1.0e-3,
                rain=np.array([[0.0, 1e-4], [2.0, 3e-4], [10.0, 0.0]]),
                given_depth=np.hstack([times, rng.uniform(0.1, 0.5, (2, 8))]),
                given_wl=np.hstack([times, rng.uniform(0.3, 0.8, (2, 8))]),
                given_q=np.hstack([times, rng.normal(0.0, 0.05, (2, 16))]))


@needs_ref
@pytest.mark.parametrize("order", [1, 2])
def test_oracle_matches_reference_build_on_random_shapes(order):
    """30 random catchments per order, 15 steps each, bit for bit (seeds 0-199
    of the same generator, both orders, were checked the same way when the
    test was written)."""
    for seed in range(30):
        d = random_case(1000 + seed, order)
        a = O.Sim(d, order=order, backend="oracle", export_step=0.5)
        b = O.Sim(d, order=order, backend="ref", export_step=0.5)
        a.run(15)
        b.run(15)
        sa, sb = a.state(), b.state()
        assert sa["t"] == sb["t"], seed
        for k in FIELDS:
            np.testing.assert_array_equal(sa[k], sb[k], err_msg=f"seed {seed} {k}")


def _radial_dam_break(n: int = 64) -> dict:
    """A column of water (radius n/5, 1 m over 0.1 m) in the middle of an
    n x n flat frictionless box with slip walls."""
    from hipims_b200.topology import boundary_codes

    nodata = np.ones((n + 2, n + 2), dtype=bool)
    nodata[1:-1, 1:-1] = False
    mask = boundary_codes(nodata, default_bc=40)
    r, c = np.meshgrid(np.arange(n + 2) - (n + 1) / 2, np.arange(n + 2) - (n + 1) / 2,
                       indexing="ij")
    h = np.where(r ** 2 + c ** 2 < (n / 5) ** 2, 1.0, 0.1)
    h[nodata] = 0.0
    z = np.zeros_like(h)
    return dict(mask=mask, z=z, h=h, qx=np.zeros_like(h), qy=np.zeros_like(h), wl=z + h,
                manning=[0.0], dx=1.0, cfl=0.5, first_dt=1.0e-3)


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("backend", ["oracle", "ref"])
def test_physics_radial_dam_break_symmetry(order, backend):
    """Mirror in x and in y and the swap of the axes leave a radial dam break
    unchanged to round-off (the y axis of the rasters points south, so under
    the swap qx(r, c) = -qy(c, r))."""
    if backend == "ref" and not O.ref_available():
        pytest.skip("oracle/_ref not built")
    n = 64
    s = O.Sim(_radial_dam_break(n), order=order, backend=backend)
    s.run(60)
    H, QX, QY = (a.reshape(n, n) for a in (s.h, s.qx, s.qy))
    assert H.max() < 0.9  # the column has collapsed
    tol = 1e-13
    assert np.abs(H - H[:, ::-1]).max() < tol and np.abs(QX + QX[:, ::-1]).max() < tol
    assert np.abs(H - H[::-1, :]).max() < tol and np.abs(QY + QY[::-1, :]).max() < tol
    assert np.abs(H - H.T).max() < tol and np.abs(QX + QY.T).max() < tol


def _stoker(x, t, hl, hr, x0):
    """Stoker's solution of the frictionless wet/wet dam break: rarefaction,
    constant middle state (h_m, u_m) and a shock into the still water."""
    from scipy.optimize import brentq

    g = 9.81
    cl = np.sqrt(g * hl)

    def momentum_jump(cm):
        hm = cm * cm / g
        um = 2.0 * (cl - cm)
        s = hm * um / (hm - hr)
        return s * hm * um - (hm * um * um + 0.5 * g * (hm * hm - hr * hr))

    cm = brentq(momentum_jump, np.sqrt(g * hr) * (1 + 1e-9), cl * (1 - 1e-9))
    hm, um = cm * cm / g, 2.0 * (cl - cm)
    s = hm * um / (hm - hr)
    xi = (x - x0) / t
    h = np.where(xi < -cl, hl, np.where(xi < um - cm, ((2 * cl - xi) / 3) ** 2 / g,
                                        np.where(xi < s, hm, hr)))
    return h, hm, s


def _dam_break_1d(n: int, order: int, t_end: float, hl: float = 1.0, hr: float = 0.1):
    from hipims_b200.topology import boundary_codes

    nodata = np.ones((3, n + 2), dtype=bool)
    nodata[1, 1:-1] = False
    mask = boundary_codes(nodata, default_bc=50)
    x = np.arange(n + 2) - 0.5
    h = np.where(x[None, :] < n / 2, hl, hr) * np.ones((3, 1))
    h[nodata] = 0.0
    z = np.zeros_like(h)
    d = dict(mask=mask, z=z, h=h, qx=np.zeros_like(h), qy=np.zeros_like(h), wl=z + h,
             manning=[0.0], dx=1.0, cfl=0.5, first_dt=1.0e-3)
    sim = O.Sim(d, order=order, export_step=t_end)  # the export clip lands on t_end
    sim.run(100000, t_end)
    xc = np.arange(1, n + 1) - 0.5
    return sim, xc, _stoker(xc, sim.t, hl, hr, n / 2)


@pytest.mark.parametrize("order,l1", [(1, 0.004), (2, 0.0015)])
def test_physics_stoker_dam_break(order, l1):
    """The frictionless 1-D dam break (1 m over 0.1 m) against Stoker's
    solution: mean depth error, shock position within a cell, qy = 0, and the
    error shrinking with the grid."""
    sim, xc, (exact, hm, s) = _dam_break_1d(400, order, 20.0)
    assert sim.t == 20.0
    err = np.abs(sim.h - exact)
    assert err.mean() < l1, err.mean()
    mid = 0.5 * (hm + 0.1)
    j = np.where((sim.h[:-1] >= mid) & (sim.h[1:] < mid))[0][-1]
    shock = xc[j] + (sim.h[j] - mid) / (sim.h[j] - sim.h[j + 1])
    assert abs(shock - (200.0 + s * 20.0)) < 1.0
    assert not np.any(sim.qy)
    coarse = _dam_break_1d(200, order, 10.0)
    fine = _dam_break_1d(800, order, 40.0)
    e_coarse = np.abs(coarse[0].h - coarse[2][0]).mean()
    e_fine = np.abs(fine[0].h - fine[2][0]).mean()
    assert e_fine < 0.7 * e_coarse, (e_coarse, e_fine)
