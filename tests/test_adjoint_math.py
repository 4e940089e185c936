"""Reverse-mode face and cell functions of the adjoint (csrc/hb_adjoint.cuh),
compiled for the CPU, against central finite differences of their forward
functions on random states away from the scheme's kinks."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "chans-hipims-flamegpu_b200", "csrc")


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("adj") / "libadjcheck.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", CSRC,
                    os.path.join(HERE, "adjoint_check.cpp"), "-o", out], check=True)
    L = ctypes.CDLL(out)
    P, D, I = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
    L.face_fwd_c.argtypes = [I, P, I, I, I, P]
    L.face_vjp_c.argtypes = [I, P, I, I, I, P, P]
    L.cell_fwd_c.argtypes = [P, P, D, D, P]
    L.cell_vjp_c.argtypes = [P, P, D, D, P, P, P, P]
    return L


def _p(a):
    return a.ctypes.data


def face_out(L, d, x, vL, vR, ns):
    o = np.zeros(5)
    L.face_fwd_c(d, _p(x), vL, vR, ns, _p(o))
    return o


def _fd_ok(f, x, i, eps):
    """Central difference with a kink check (two step sizes must agree)."""
    def cd(e):
        xp, xm = x.copy(), x.copy()
        xp[i] += e
        xm[i] -= e
        return (f(xp) - f(xm)) / (2 * e)
    def one_sided(e):
        xp = x.copy()
        xp[i] += e
        return (f(xp) - f(x)) / e
    a, b = cd(eps), cd(eps / 4)
    # A kink exactly at x (a dry cell at h = 0) passes the two central
    # differences but not the comparison of the two one-sided ones.
    ok = (np.allclose(a, b, rtol=1e-4, atol=1e-9)
          and np.allclose(one_sided(eps), one_sided(-eps), rtol=1e-3, atol=1e-6))
    return b, ok


def _state(rng, wet=True):
    x = np.zeros(16)
    for k in range(4):
        h = rng.uniform(0.05, 0.6) if wet else rng.choice([0.0, rng.uniform(0.05, 0.6)])
        x[4 * k: 4 * k + 4] = [h, rng.normal(0, 0.15), rng.normal(0, 0.15),
                               rng.uniform(0.0, 0.3)]
    return x


@pytest.mark.parametrize("direction", [0, 1])
@pytest.mark.parametrize("seed", range(12))
def test_face_vjp_matches_finite_differences(lib, direction, seed):
    rng = np.random.default_rng(seed)
    x = _state(rng, wet=seed % 3 != 0)
    vL, vR, ns = int(seed % 4 != 1), int(seed % 5 != 2), int(seed % 6 == 5)
    ob = rng.normal(0, 1, 5)
    xb = np.zeros(12)
    lib.face_vjp_c(direction, _p(x), vL, vR, ns, _p(ob), _p(xb))
    f = lambda xx: float(face_out(lib, direction, xx, vL, vR, ns) @ ob)
    checked = 0
    for cell in range(4):
        for comp in range(3):
            i = 4 * cell + comp
            fd, ok = _fd_ok(f, x, i, 1e-6)
            if not ok:
                continue  # a discrete decision switches within the stencil
            checked += 1
            assert xb[3 * cell + comp] == pytest.approx(fd, rel=1e-5, abs=1e-7), (cell, comp)
    assert checked >= 6


@pytest.mark.parametrize("seed", range(20))
def test_cell_vjp_matches_finite_differences(lib, seed):
    rng = np.random.default_rng(100 + seed)
    u = np.array([rng.uniform(0.001, 0.5), rng.normal(0, 0.3), rng.normal(0, 0.3)])
    r = np.array([rng.normal(0, 0.01), rng.normal(0, 0.02), rng.normal(0, 0.02)])
    if seed % 5 == 0:  # thin film: limiter and near-dry branches
        u[0] = rng.uniform(1e-4, 3e-3)
    n, dt = rng.uniform(0.02, 0.1), rng.uniform(0.05, 0.5)
    ob = rng.normal(0, 1, 3)
    ub, rb, nb = np.zeros(3), np.zeros(3), ctypes.c_double()
    lib.cell_vjp_c(_p(u), _p(r), n, dt, _p(ob), _p(ub), _p(rb), ctypes.byref(nb))

    def out(uu, rr, nn):
        o = np.zeros(3)
        lib.cell_fwd_c(_p(uu), _p(rr), nn, dt, _p(o))
        return float(o @ ob)

    # Steps of 1e-5: the reference friction form 1 - sqrt(1 + 4x) cancels,
    # so smaller steps measure rounding noise rather than the derivative.
    for i in range(3):
        fd, ok = _fd_ok(lambda v: out(v, r, n), u, i, 1e-5)
        if ok:
            assert ub[i] == pytest.approx(fd, rel=1e-5, abs=1e-8)
        fd, ok = _fd_ok(lambda v: out(u, v, n), r, i, 1e-5)
        if ok:
            assert rb[i] == pytest.approx(fd, rel=1e-5, abs=1e-8)
    fd, ok = _fd_ok(lambda v: out(u, r, v[0]), np.array([n]), 0, 1e-5)
    if ok:
        assert nb.value == pytest.approx(fd, rel=1e-5, abs=1e-8)
