"""Long-run physics of the GPU step: the Langmuir oscillation at the plasma
frequency (Bohm-Gross) and total-energy conservation, against analytic
references (the reference repository holds no golden data for either)."""
import math

import numpy as np
import pytest

from gample_b200 import capi
from tests.helpers import EC, ME, MXE, condition

N0 = 5e10
WPE = math.sqrt(4 * math.pi * N0 * EC ** 2 / ME)


def _lattice(ngx, ngy, ngb, side):
    """side x side particles per cell on a regular sub-lattice (quiet start)."""
    o = (np.arange(side) + 0.5) / side
    cx, cy = np.meshgrid(np.arange(ngx), np.arange(ngy))
    ox, oy = np.meshgrid(o, o)
    x = (cx[..., None, None] + ox[None, None]).ravel() + ngb
    y = (cy[..., None, None] + oy[None, None]).ravel() + ngb
    return x.astype(np.float32), y.astype(np.float32)


@pytest.mark.gpu
def test_langmuir_oscillation_at_the_plasma_frequency(gpu):
    ngx, ngy, side = 64, 4, 4
    lam_d = math.sqrt(10 * 1.6021764262e-12 / (4 * math.pi * N0 * EC ** 2))
    dx = 0.5 * lam_d
    dt = 0.1 / WPE
    steps = 630  # ten plasma periods
    cond = condition(ngx=ngx, ngy=ngy, order=3, ppc=side * side, dx=dx, dt=dt, te=1.0, ti=0.01, density=N0,
                     end=steps)
    sim = capi.Sim(cond)
    x, y = _lattice(ngx, ngy, 1, side)
    k = 2 * math.pi / (ngx * dx)
    v0 = 2e6
    for s in range(2):
        p = np.zeros(len(x), capi.PARTICLE_DTYPE)
        p["x"], p["y"] = x, y
        if s == 0:
            p["vx"] = (v0 * np.sin(k * (x.astype(np.float64) - 1) * dx)).astype(np.float32)
        sim.set_particles(s, p)
    sim.initialize()
    ex = []
    for _ in range(steps):
        sim.run(1)
        ex.append(sim.last_solve().probe[1])  # Ex at (ngx/4, ngy/2): the wave's antinode
    ex = np.array(ex)
    # mean period from the zero crossings (linear interpolation)
    sgn = np.sign(ex)
    idx = np.where(sgn[:-1] * sgn[1:] < 0)[0]
    t = idx + ex[idx] / (ex[idx] - ex[idx + 1])
    half = np.diff(t)
    omega = math.pi / (np.mean(half) * dt)
    # Bohm-Gross at Te = 1 eV: w^2 = wpe^2 (1 + 3 k^2 lambda_D(1 eV)^2)
    lam1 = lam_d / math.sqrt(10)
    want = WPE * math.sqrt(1 + 3 * (k * lam1) ** 2)
    assert len(idx) >= 18
    assert abs(omega / want - 1) < 0.02, (omega / WPE, want / WPE)
    sim.close()


@pytest.mark.gpu
def test_total_energy_is_conserved(gpu):
    lam_d = math.sqrt(10 * 1.6021764262e-12 / (4 * math.pi * N0 * EC ** 2))
    dt = 0.05 / WPE
    cond = condition(ngx=48, ngy=48, order=3, ppc=64, dx=0.5 * lam_d, dt=dt, te=10.0, ti=1.0, density=N0, end=400)
    sim = capi.Sim(cond)
    sim.initialize()
    tot = []
    for c in range(400):
        sim.run(1)
        ke = sim.last_flow(0).kinetic_energy + sim.last_flow(1).kinetic_energy
        tot.append(ke + sim.last_solve().field_energy_cgs)
    tot = np.array(tot)
    drift = abs(tot[-1] - tot[0]) / tot[0]
    assert drift < 0.01, drift
    sim.close()

