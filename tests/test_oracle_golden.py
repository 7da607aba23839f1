"""The CPU oracle against the reference's own recorded outputs and published
known answers (no GPU needed).

Pins: the reference's timeseries traces of data/single_darwin.json and
data/uniform_darwin.json (10 cycles each: loader RNG, 5th-order deposit and
gather, Boris push, ghost folding, Poisson CSR, phi reconstruction, gradient,
CSV probe), splitmix64 / PCG32 published test vectors, and scipy's direct
solve of the Poisson system.
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import config as ocfg
from oracle import lib as L
from tests.helpers import GOLDEN, condition, read_trace


def run_oracle_trace(cfg, ncycles):
    sim = L.OracleSim(cfg, real64=False)
    sim.load_initial()
    sim.reset_charge()
    for s in range(sim.ns):
        sim.deposit(s)
    sim.solve_poisson(0.0)
    rows = []
    t = comp = 0.0
    dt = cfg["time"]["TimeStep"]
    for cyc in range(1, ncycles + 1):
        y = dt - comp
        tt = t + y
        comp = (tt - t) - y
        t = tt
        st, _ = sim.cycle(cyc)
        rows.append([cyc, t] + [float(np.float32(v)) for v in st.probe])
    return np.array(rows)


@pytest.mark.parametrize("name", ["single_darwin", "uniform_darwin"])
def test_oracle_reproduces_reference_trace(name):
    cfg = ocfg.parse(os.path.join(GOLDEN, name + ".json"))
    _, ref = read_trace(os.path.join(GOLDEN, name + "_test_timeseries.csv"))
    got = run_oracle_trace(cfg, len(ref))
    np.testing.assert_array_equal(got[:, 0], ref[:, 0])
    np.testing.assert_allclose(got[:, 1], ref[:, 1], rtol=1e-6)
    for col in (2, 3, 4):
        # Tolerance: 2e-4 relative plus 3e-4 of the trace's range. The floor
        # covers FP32 position rounding (one electron at x ~ 22 cells has an
        # ulp of 2e-6 cells against a 0.1-cell step, i.e. 2e-5 of the dipole
        # per step; Ey1 of that dipole is the most sensitive column) and the
        # FP32 charge noise (uniform_darwin's cycle 1 is pure rounding, ~2e-7
        # of the range). The traces swing through their whole range, so an
        # error in the method shows up at O(1).
        scale = np.max(np.abs(ref[:, col]))
        err = np.abs(got[:, col] - ref[:, col])
        assert np.all(err <= 2e-4 * np.abs(ref[:, col]) + 3e-4 * scale), (col, err, ref[:, col])


def test_csv_text_format_matches_reference():
    # src/XmlLogger.h:89-93 and the ostream time format of src/XmlLogger.h:37
    cfg = ocfg.parse(os.path.join(GOLDEN, "single_darwin.json"))
    got = run_oracle_trace(cfg, 1)
    line = f"1,{L.fmt_time(got[0, 1])},{L.fmt_sci(got[0, 2])},{L.fmt_sci(got[0, 3])},{L.fmt_sci(got[0, 4])}"
    with open(os.path.join(GOLDEN, "single_darwin_test_timeseries.csv")) as f:
        f.readline()
        assert f.readline().strip() == line


def test_splitmix64_published_vectors():
    # Vigna's splitmix64 reference output for seed 1234567.
    got = L.splitmix64_stream(1234567, 5)
    assert list(map(int, got)) == [6457827717110365317, 3203168211198807973, 9817491932198370423,
                                   4593380528125082431, 16408922859458223821]


def test_pcg32_published_vectors():
    # pcg32 demo: pcg32_srandom_r(42, 54) then six outputs.
    mult = 6364136223846793005
    mask = (1 << 64) - 1
    inc = ((54 << 1) | 1) & mask
    state = (0 * mult + inc) & mask
    state = (state + 42) & mask
    state = (state * mult + inc) & mask
    got = L.pcg32_raw(state, inc, 6)
    assert [hex(int(v)) for v in got] == ["0xa15c02b7", "0x7b47f409", "0xba1d3330", "0x83d2f293",
                                          "0xbfa4784b", "0xcbed606e"]


def test_loader_is_neutral():
    # Each ion sits on its electron (src/Collision.mm:147-151): rho vanishes
    # before the first push (FP64 deposit: exactly).
    cfg = ocfg.parse(condition(ngx=16, ngy=16, order=3, ppc=4))
    sim = L.OracleSim(cfg, real64=True)
    sim.load_initial()
    sim.reset_charge()
    for s in range(2):
        sim.deposit(s)
    e = sim.particles(0)
    i = sim.particles(1)
    np.testing.assert_array_equal(e["x"], i["x"])
    np.testing.assert_array_equal(e["y"], i["y"])
    # cancels to FP64 summation rounding (species are summed one after the other)
    scale = abs(sim.species_consts(0)["scale"])
    assert np.max(np.abs(sim.field("rho"))) < 1e-13 * scale * 4


def _laplacian(nx, ny, dx, dy, perx, pery):
    ex = sp.diags([np.ones(nx - 1), -2 * np.ones(nx), np.ones(nx - 1)], [-1, 0, 1], format="lil")
    ey = sp.diags([np.ones(ny - 1), -2 * np.ones(ny), np.ones(ny - 1)], [-1, 0, 1], format="lil")
    if perx:
        ex[0, nx - 1] = ex[nx - 1, 0] = 1
    if pery:
        ey[0, ny - 1] = ey[ny - 1, 0] = 1
    return (sp.kron(sp.eye(ny), ex) / dx ** 2 + sp.kron(ey, sp.eye(nx)) / dy ** 2).tocsr()


def test_poisson_oracle_against_scipy():
    # Dirichlet x (phi = 200 V / 0 V) and periodic y, as data/org.json.
    c = condition(ngx=24, ngy=16, order=1, ppc=2, xbc="Dirichlet", ybc="periodic", phi_xmin=200.0)
    cfg = ocfg.parse(c)
    sim = L.OracleSim(cfg, real64=True)
    rng = np.random.default_rng(0)
    rho = rng.standard_normal(sim.shape("rho")) * 1e-3
    sim.set_field("rho", rho)
    st = sim.solve_poisson(0.0, tol=1e-13)
    sol = sim.poisson_solution()
    rho = sim.field("rho")  # after ghost folding (src/EMField.mm:751-850)
    nkx1, nky1 = 24 - 1, 16
    dxx = float(np.float32(0.005))  # the field stores dx as float (src/EMField.mm:65)
    A = _laplacian(nkx1, nky1, dxx, dxx, False, True)
    b = -4 * np.pi * rho[0:nky1, 1:1 + nkx1].ravel().astype(np.float64)
    vt = 200 * 1e8 / 2.99792458e10
    b = b.reshape(nky1, nkx1)
    b[:, 0] += -vt / dxx ** 2
    ref = spla.spsolve(A, b.ravel())
    assert st.error < 1e-12
    np.testing.assert_allclose(sol, ref, rtol=1e-9, atol=1e-12 * np.max(np.abs(ref)))


def test_compaction_quirk_documented():
    # src/Particle.mm:908-966 pulls one live particle too many when the tail
    # scan runs out of live particles; the build counts every flagged
    # particle exactly once.
    cfg = ocfg.parse(condition(ngx=8, ngy=8, order=1, ppc=1))
    sim = L.OracleSim(cfg, real64=False)
    x = np.arange(3, dtype=np.float64) + 1.5
    z = np.zeros(3)
    sim.set_particles(0, x, x, z, z, z, piflag=[0, 1, 1])
    fs = sim.reduce(0, faithful=True)
    assert sim.pnum(0) == 0 and fs.pulled == 3      # the live particle is lost
    sim.set_particles(0, x, x, z, z, z, piflag=[0, 1, 1])
    fs = sim.reduce(0, faithful=False)
    assert sim.pnum(0) == 1 and fs.pulled == 2
    assert list(fs.pinum) == [-2, 0, 0, 0]          # electrons: charge-sign units


def test_shape_factors():
    for order in (1, 3, 5):
        for h in np.linspace(0.0, 0.999, 37):
            wb = L.shape_build(order, h).astype(np.float64)
            wr = L.shape_ref(order, h, f64=True)
            np.testing.assert_allclose(wb, wr, atol=2e-7)
            assert abs(wb.sum() - 1.0) < 4e-7
