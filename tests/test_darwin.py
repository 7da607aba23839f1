"""Darwin model (src/EMField.mm:447-651, 1138-1361): the oracle's
Helmholtz split on a manufactured current, and the GPU solve against the
oracle on the same currents."""
import numpy as np
import pytest

from gample_b200 import capi
from oracle import lib as L
from tests.helpers import condition


def _gradient_current(ngx, ngy, ngb, dx, dy, f):
    """jx, jy (reference extents) = the face differences of a periodic node
    field f (ngy, ngx), ghost faces filled periodically."""
    nx, ny = ngx + 2 * ngb, ngy + 2 * ngb
    jx = np.zeros((ny + 1, nx + 2), np.float32)
    jy = np.zeros((ny + 2, nx + 1), np.float32)
    gx = ((np.roll(f, -1, axis=1) - f) / dx).astype(np.float32)   # face between node i and i+1
    gy = ((np.roll(f, -1, axis=0) - f) / dy).astype(np.float32)
    for j in range(ngy):
        for i in range(ngx):
            jx[j + ngb, i + ngb + 1] = gx[j, i]
            jy[j + ngb + 1, i + ngb] = gy[j, i]
        jx[j + ngb, ngb] = gx[j, ngx - 1]
    for i in range(ngx):
        jy[ngb, i + ngb] = gy[ngy - 1, i]
    return jx, jy


def test_oracle_darwin_splits_a_gradient_current():
    """J = grad f (doubly periodic): psi = f - mean(f) and A = 0."""
    ngx, ngy, ngb, dx, dy = 24, 16, 1, 0.01, 0.012
    xs, ys = np.meshgrid(np.arange(ngx) / ngx, np.arange(ngy) / ngy)
    f = 3e9 * np.sin(2 * np.pi * xs) * np.cos(4 * np.pi * ys) + 1e9 * np.cos(2 * np.pi * ys)
    jx, jy = _gradient_current(ngx, ngy, ngb, dx, dy, f)
    d = L.Darwin(ngx, ngy, ngb, True, True, np.float32(dx), np.float32(dy))
    out = d.solve(jx, jy, 1e-12)
    want = f - f.mean()
    assert np.max(np.abs(out["psi"] - want)) < 1e-5 * np.max(np.abs(want))
    a_scale = 4 * np.pi / 2.99792458e10 * np.max(np.abs(jx)) * (ngx * dx) ** 2
    assert np.max(np.abs(out["Ax"])) < 1e-5 * a_scale
    assert np.max(np.abs(out["Ay"])) < 1e-5 * a_scale


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["periodic", "neumann", "config3"])
def test_darwin_matches_oracle(gpu, case):
    """config3: the Darwin configuration's set-up at 128^2 (doubly periodic,
    order 5, electron drift 0.1 v_te sin(2 pi x / L) along y from the
    build-added SinusoidalDriftVel key: a transverse current)."""
    if case == "periodic":
        cond = condition(ngx=32, ngy=32, order=1, ppc=16, em=2, cur_dens=1, vxe=4e7)
    elif case == "config3":
        cond = condition(ngx=128, ngy=128, order=5, ppc=16, em=2, cur_dens=1)
        vte = np.sqrt(2 * 1.3806503e-16 * 10.0 * 11604.0 / 9.10938188e-28)
        cond["ParamForParticle"][0]["SinusoidalDriftVel"] = [0.0, 0.1 * vte, 0.0]
    else:
        cond = condition(ngx=33, ngy=24, order=3, ppc=16, xbc="Dirichlet", ybc="periodic", em=2, cur_dens=1,
                         vxe=4e7)
    dt = cond["ParamForTimeIntegration"]["TimeStep"]
    sim = capi.Sim(cond)
    sim.initialize()
    sim.run(2)
    jx, jy = sim.field("jx"), sim.field("jy")
    it, err = sim.solve_darwin(dt)
    assert all(e <= 1e-8 for e in err), err
    dx = np.float32(cond["ParamForField"]["GridSizeOfX"])
    dy = np.float32(cond["ParamForField"]["GridSizeOfY"])
    o = L.Darwin(sim.ngx, sim.ngy, sim.ngb, case != "neumann", True, dx, dy)
    # the GPU's A_last after two cycles is unknown to the oracle: compare the
    # potentials, and the fields of the next solve from a shared A_last
    want = o.solve(jx, jy, dt)
    for k in ("psi", "Ax", "Ay"):
        got = sim.field(k)
        s = np.max(np.abs(want[k]))
        assert s > 0
        assert np.max(np.abs(got - want[k])) < 2e-6 * s, k
    sim.run(1)  # its own Darwin solve leaves A_last = the current A
    o.lastAx, o.lastAy = sim.field("Ax").copy(), sim.field("Ay").copy()
    jx, jy = sim.field("jx"), sim.field("jy")
    sim.solve_darwin(dt)
    want = o.solve(jx, jy, dt)
    for k in ("Ax", "Ay"):
        s = np.max(np.abs(want[k]))
        assert np.max(np.abs(sim.field(k) - want[k])) < 2e-6 * s, k
    for k in ("delEx", "delEy", "delBz"):
        got, w = sim.field(k), want[k]
        s = np.max(np.abs(w))
        assert s > 0
        assert np.max(np.abs(got - w)) < 2e-3 * s, k
    sim.close()
