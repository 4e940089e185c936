"""GPU parity of the compat ops (the reference's op surface) against the
pinned CPU oracle, through the C ABI.  FP64: the same arithmetic in the same
order, so agreement to a few ulp (tolerance rtol 1e-12); FP32: rtol 1e-5."""
import numpy as np
import pytest
import torch

import make_golden as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = {torch.float64: dict(rtol=1e-12, atol=1e-14), torch.float32: dict(rtol=1e-5, atol=2e-6)}
# FP32 flux: a handful of minmod / dry-threshold decisions may flip on random
# states; the flipped cells still agree to 1e-4 (the magnitude of one face's
# dt/dx * flux here).
FLUX32 = dict(rtol=1e-4, atol=1e-4)


def _state(seed, order=2):
    d = G.mixed_bc_case(seed, order)
    return d, O.Sim(d, order=order)


def _t(a, dtype, dev):
    return torch.as_tensor(np.asarray(a), device=dev).to(dtype).contiguous()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("order", [2, 1])
def test_flux_matches_oracle(cuda, dtype, order):
    from hipims_b200 import ops

    d, s = _state(21 + order, order)
    N = s.N
    rng = np.random.default_rng(order)
    wet = np.sort(rng.choice(N, size=N * 3 // 4, replace=False)).astype(np.int32)
    outs = [rng.normal(0, 1e-3, N) for _ in range(3)]
    exp = [o.copy() for o in outs]
    dx, t, dt = 0.5, 0.6, 0.01
    O.flux(order, wet, *exp, s.h, s.wl, s.z, s.qx, s.qy, s.index, s.normal, s.gd, s.gw, s.gq,
           dx, t, dt)
    T = lambda a: _t(a, dtype, cuda)
    got = [T(o) for o in outs]
    op = ops.flux_2nd_order if order == 2 else ops.flux_1st_order
    op(torch.as_tensor(wet, device=cuda), *got, T(s.h), T(s.wl), T(s.z), T(s.qx), T(s.qy),
       torch.as_tensor(s.index, device=cuda), T(s.normal.reshape(4, 2)), T(s.gd), T(s.gw),
       T(s.gq), T([dx]), T([t]), T([dt]))
    for g_, e in zip(got, exp):
        a = g_.double().cpu().numpy()
        if dtype == torch.float64:
            np.testing.assert_allclose(a, e, **TOL[dtype])
        else:
            np.testing.assert_allclose(a, e, **FLUX32)
            assert np.mean(np.abs(a - e) <= 2e-6 + 1e-5 * np.abs(e)) > 0.99


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_friction_timestep_rain_mask_euler(cuda, dtype):
    from hipims_b200 import ops

    d, s = _state(31)
    N = s.N
    rng = np.random.default_rng(5)
    T = lambda a: _t(a, dtype, cuda)
    hu, qxu, qyu = rng.normal(0, 0.01, N), rng.normal(0, 0.01, N), rng.normal(0, 0.01, N)
    zu = np.zeros(N)
    lst = np.arange(N, dtype=np.int32)
    # friction + update
    e = [x.copy() for x in (hu, qxu, qyu, zu, s.h, s.wl, s.qx, s.qy, s.z)]
    O.friction_update(lst, *e[:4], s.landuse, *e[4:], s.manning, 0.02)
    g = [T(x) for x in (hu, qxu, qyu, zu, s.h, s.wl, s.qx, s.qy, s.z)]
    ops.friction_update(torch.as_tensor(lst, device=cuda), *g[:4],
                        torch.as_tensor(s.landuse, device=cuda), *g[4:], T(s.manning), T([0.02]))
    for a, b in zip(g, e):
        np.testing.assert_allclose(a.double().cpu().numpy(), b, **TOL[dtype])
    # timestep
    acc_e, hm_e = np.full(N, 60.0), s.h_max.copy() * 0.5
    O.timestep(lst, acc_e, hm_e, e[4], e[6], e[7], 0.5, 0.5)
    acc_g, hm_g = T(np.full(N, 60.0)), T(s.h_max * 0.5)
    ops.update_timestep(torch.as_tensor(lst, device=cuda), acc_g, hm_g, g[4], g[6], g[7],
                        T([0.5]), T([0.5]), T([0.0]), T([0.02]))
    np.testing.assert_allclose(acc_g.double().cpu().numpy(), acc_e, rtol=1e-6 if dtype ==
                               torch.float32 else 1e-12)
    np.testing.assert_allclose(hm_g.double().cpu().numpy(), hm_e, **TOL[dtype])
    assert float(ops.device_min(acc_g)) == pytest.approx(acc_e.min(), rel=1e-6)
    # station rain
    rm = rng.integers(0, 3, N).astype(np.int16)
    data = np.array([1e-4, 2e-4, 3e-4])
    r_e = hu.copy()
    O.rain_station(r_e, rm, data, 0.5)
    r_g = T(hu)
    ops.station_rain(r_g, torch.as_tensor(rm, device=cuda), T(data), T([0.5]))
    np.testing.assert_allclose(r_g.double().cpu().numpy(), r_e, **TOL[dtype])
    # flux mask (including the cell-0 rule) at t > 0 and t == 0
    for tt in (0.0, 1.0):
        m_e = np.zeros(N, np.uint8)
        O.flux_mask(m_e, s.h, s.index, tt)
        m_g = torch.zeros(N, dtype=torch.bool, device=cuda)
        ops.flux_mask(m_g, T(s.h), torch.as_tensor(s.index, device=cuda), T([tt]))
        np.testing.assert_array_equal(m_g.cpu().numpy().astype(np.uint8), m_e)
    # euler update
    e2 = [x.copy() for x in (s.h, s.wl, s.z, s.qx, s.qy)]
    O.euler_update(lst, hu, qxu, qyu, zu, *e2)
    g2 = [T(x) for x in (s.h, s.wl, s.z, s.qx, s.qy)]
    ops.euler_update(torch.as_tensor(lst, device=cuda), T(hu), T(qxu), T(qyu), T(zu), *g2)
    for a, b in zip(g2, e2):
        np.testing.assert_allclose(a.double().cpu().numpy(), b, **TOL[dtype])


def test_infiltration_matches_oracle(cuda):
    from hipims_b200 import ops

    d, s = _state(41)
    N = s.N
    lst = np.arange(N, dtype=np.int32)
    hu = np.zeros(N)
    cum = np.random.default_rng(1).uniform(0, 0.01, N)
    ks, psi, dth = np.array([1e-6, 5e-6]), np.array([0.1, 0.2]), np.array([0.3, 0.4])
    hu_e, cum_e = hu.copy(), cum.copy()
    O.infiltration(lst, hu_e, s.landuse, s.h, ks, psi, dth, cum_e, 10.0)
    T = lambda a: _t(a, torch.float64, cuda)
    hu_g, cum_g = T(hu), T(cum)
    ops.infiltration(torch.as_tensor(lst, device=cuda), hu_g,
                     torch.as_tensor(s.landuse, device=cuda), T(s.h), T(ks), T(psi), T(dth),
                     cum_g, T([10.0]))
    np.testing.assert_allclose(hu_g.cpu().numpy(), hu_e, rtol=1e-12, atol=1e-16)
    np.testing.assert_allclose(cum_g.cpu().numpy(), cum_e, rtol=1e-12, atol=1e-16)


def test_device_min_large(cuda):
    from hipims_b200 import ops

    x = torch.rand(3_000_001, dtype=torch.float64, device=cuda) + 1.0
    x[1_234_567] = 0.25
    assert float(ops.device_min(x)) == 0.25
    assert float(ops.device_min(x)) == 0.25  # counter reset between calls
