"""Edge cases of the step through the C ABI (GPU): an empty species, a
particle count that fills no chunk or warp evenly, a store filled beyond its
capacity, and a step after which every particle has left the domain."""
import numpy as np
import pytest

from gample_b200 import capi
from oracle import config as ocfg
from oracle import lib as L
from tests.helpers import condition

pytestmark = pytest.mark.gpu


def _records(x, y, vx, vy, vz):
    a = np.zeros(len(x), capi.PARTICLE_DTYPE)
    a["x"], a["y"], a["vx"], a["vy"], a["vz"] = x, y, vx, vy, vz
    return a


def test_empty_species_runs_and_deposits_nothing(gpu):
    cond = condition(ngx=32, ngy=24, order=3, ppc=4, xbc="Dirichlet", ybc="periodic", deposit_mode=1, end=3)
    sim = capi.Sim(cond)
    sim.initialize()
    sim.set_particles(0, np.zeros(0, capi.PARTICLE_DTYPE))
    assert sim.count(0) == 0
    sim.reset_charge()
    sim.integrate_charge(0)
    assert np.all(sim.field("rho") == 0.0)
    sim.run(3)  # push, compaction and sort of an empty store
    assert sim.count(0) == 0
    assert len(sim.particles(0)) == 0
    assert np.all(np.isfinite(sim.field("Ex")))
    sim.close()


@pytest.mark.parametrize("n", [1, 31, 1001, 2049])
def test_ragged_particle_counts_match_the_oracle(gpu, n):
    """Counts that end inside a warp or a 2048-particle chunk: the
    deterministic deposit is bit-exact and the push agrees to 1e-5."""
    ngx, ngy, order = 24, 16, 3
    cond = condition(ngx=ngx, ngy=ngy, order=order, ppc=2, xbc="periodic", ybc="periodic", deposit_mode=1,
                     bz_tesla=0.02, dt=2e-11)
    sim = capi.Sim(cond)
    ora = L.OracleSim(ocfg.parse(cond))
    rng = np.random.default_rng(n)
    ngb = order // 2
    x = (ngb + rng.uniform(0, ngx, n)).astype(np.float32)
    y = (ngb + rng.uniform(0, ngy, n)).astype(np.float32)
    v = rng.normal(0.0, 3e7, (3, n)).astype(np.float32)
    for s in range(2):
        sim.set_particles(s, _records(x, y, v[0], v[1], v[2]))
        ora.set_particles(s, x, y, v[0], v[1], v[2], f32=True)
    assert sim.count(0) == n
    # deterministic deposit of species 0: exact fixed-point sums
    sim.reset_charge()
    sim.integrate_charge(0)
    raw = sim.particles_raw(0)
    ix = (raw["cell"] & 0xFFFF).astype(np.int32)
    iy = (raw["cell"] >> 16).astype(np.int32)
    acc = L.det_deposit_rho(order, ngx, ngy, ngb, ix, iy, raw["ox"], raw["oy"])
    scale = np.float64(np.float32(ora.species_consts(0)["scale"]))
    # species sums added into a zeroed field, as the library combines them (+0.0 where empty)
    expect = (np.zeros(acc.shape) + acc.astype(np.float64) * (scale * 2.0 ** -40)).astype(np.float32)
    assert np.array_equal(sim.field("rho").view(np.uint32), expect.view(np.uint32))
    # one push in the same smooth random fields on both sides (the push keeps
    # the upload order, so particles compare one to one)
    for name in ("Ex", "Ey", "Bz"):
        shape = ora.shape(name)
        jj, ii = np.meshgrid(np.arange(shape[0]), np.arange(shape[1]), indexing="ij")
        amp = 500.0 if name == "Bz" else 30.0
        f = amp * (np.sin(0.3 * ii + 0.2 * jj) + 0.5 * np.cos(0.17 * ii - 0.4 * jj)) + (amp if name == "Bz" else 0.0)
        ora.set_field(name, f)
        sim.set_field(name, ora.field(name).astype(np.float32))
    ora.push(0)
    sim.update(0, cond["ParamForTimeIntegration"]["TimeStep"], fused_deposit=False)
    g, r = sim.particles(0), ora.particles(0, f32=True)
    assert len(g) == n and len(r["x"]) == n
    assert np.array_equal(g["piflag"], r["piflag"])
    vth = float(np.sqrt(np.mean(r["vx"].astype(np.float64) ** 2)))
    for c in ("vx", "vy", "vz"):
        a, b = g[c].astype(np.float64), r[c].astype(np.float64)
        assert np.all(np.abs(a - b) <= 1e-5 * (np.abs(b) + vth)), c
    for c, period in (("x", ngx), ("y", ngy)):
        d = np.abs(g[c].astype(np.float64) - r[c].astype(np.float64))
        d = np.minimum(d, period - d)  # periodic wrap on either side
        assert np.all(d <= 1e-4), c
    sim.close()


@pytest.mark.parametrize("n", [5, 200_003])
def test_upload_in_random_order_is_sorted_by_tile(gpu, n):
    """Uploaded particles are in no particular order; initialize() sorts them
    through the staged record scatter (32-byte records in the spare buffers
    of both species): the same particles come back, ordered by 8x8 tile, then
    row and column inside the tile. An upload between cycles is sorted by the
    next cycle (24-byte records in the species' own spare buffer)."""
    cond = condition(ngx=40, ngy=24, order=1, ppc=2, xbc="periodic", ybc="Dirichlet", pnum_max=250_000,
                     dt=1e-18)
    sim = capi.Sim(cond)
    rng = np.random.default_rng(n)
    x = rng.uniform(0, 40, n).astype(np.float32)
    y = rng.uniform(0.5, 23.5, n).astype(np.float32)
    v = rng.normal(0.0, 1e5, (3, n)).astype(np.float32)
    for s in range(2):
        sim.set_particles(s, _records(x, y, v[0], v[1], v[2]))
    before = [sim.particles_raw(s) for s in range(2)]
    sim.initialize()
    cols = ("cell", "ox", "oy", "vx", "vy", "vz")
    for s in range(2):
        after = sim.particles_raw(s)
        assert len(after["cell"]) == n
        ix, iy = after["cell"] & 0xFFFF, after["cell"] >> 16
        key = (((iy // 8).astype(np.int64) * 4096 + ix // 8) * 8 + iy % 8) * 8 + ix % 8
        assert np.all(np.diff(key) >= 0)
        as_bits = lambda d: np.stack([d[c].view(np.uint32) for c in cols])
        a, b = as_bits(before[s]), as_bits(after)
        np.testing.assert_array_equal(a[:, np.lexsort(a[::-1])], b[:, np.lexsort(b[::-1])])
    # particles at rest and a 1e-18 s step: the cycle's push keeps every cell
    z = np.zeros(n, np.float32)
    sim.set_particles(0, _records(x, y, z, z, z))
    sim.run(1)
    after = sim.particles_raw(0)
    assert len(after["cell"]) == n
    ix, iy = after["cell"] & 0xFFFF, after["cell"] >> 16
    key = (((iy // 8).astype(np.int64) * 4096 + ix // 8) * 8 + iy % 8) * 8 + ix % 8
    assert np.all(np.diff(key) >= 0)
    np.testing.assert_array_equal(np.sort(after["cell"]), np.sort(before[0]["cell"]))
    sim.close()


def _tile_key(cell):
    ix, iy = (cell & 0xFFFF).astype(np.int64), (cell >> 16).astype(np.int64)
    return (((iy // 8) * 4096 + ix // 8) * 8 + iy % 8) * 8 + ix % 8


@pytest.mark.parametrize("n", [7, 300_001])
@pytest.mark.parametrize("path", [1, 2])
def test_resort_of_nearly_sorted_particles_with_strays(gpu, n, path):
    """The periodic re-sort's input: particles in tile order that have since
    drifted by up to three cells, with 2 % strays anywhere on the grid (holes
    refilled from the end of the store, re-injected particles) and a ragged
    last block. The block-local re-sort (path 1) and the staged record
    scatter (path 2) both return the same particles in tile order."""
    ngx, ngy = 96, 72
    cond = condition(ngx=ngx, ngy=ngy, order=1, ppc=2, xbc="periodic", ybc="periodic",
                     pnum_max=max(n, 2 * ngx * ngy) + 10)
    sim = capi.Sim(cond)
    rng = np.random.default_rng(n + path)
    x = rng.uniform(0, ngx, n)
    y = rng.uniform(0, ngy, n)
    order = np.lexsort((np.floor(x) % 8, np.floor(y) % 8, np.floor(x) // 8, np.floor(y) // 8))
    x, y = x[order], y[order]
    x = (x + rng.uniform(-3, 3, n)) % ngx
    y = (y + rng.uniform(-3, 3, n)) % ngy
    stray = rng.random(n) < 0.02
    x[stray] = rng.uniform(0, ngx, np.count_nonzero(stray))
    y[stray] = rng.uniform(0, ngy, np.count_nonzero(stray))
    v = rng.normal(0.0, 1e5, (3, n)).astype(np.float32)
    xf, yf = x.astype(np.float32), y.astype(np.float32)
    xf[xf >= ngx], yf[yf >= ngy] = 0.0, 0.0  # rounded up onto the far edge
    recs = _records(xf, yf, v[0], v[1], v[2])
    for s in range(2):
        sim.set_particles(s, recs)
    cols = ("cell", "ox", "oy", "vx", "vy", "vz")
    as_bits = lambda d: np.stack([d[c].view(np.uint32) for c in cols])
    for s in range(2):
        before = sim.particles_raw(s)
        assert np.any(np.diff(_tile_key(before["cell"])) < 0) or n < 10
        sim.sort(s, path)
        after = sim.particles_raw(s)
        assert len(after["cell"]) == n
        assert np.all(np.diff(_tile_key(after["cell"])) >= 0)
        a, b = as_bits(before), as_bits(after)
        np.testing.assert_array_equal(a[:, np.lexsort(a[::-1])], b[:, np.lexsort(b[::-1])])
    sim.close()


def test_upload_beyond_the_capacity_is_an_error(gpu):
    cond = condition(ngx=16, ngy=16, order=1, ppc=2, pnum_max=1000)
    sim = capi.Sim(cond)
    n = 1001
    a = _records(np.full(n, 4.5, np.float32), np.full(n, 4.5, np.float32), np.zeros(n, np.float32),
                 np.zeros(n, np.float32), np.zeros(n, np.float32))
    with pytest.raises(capi.GampleError) as e:
        sim.set_particles(0, a)
    assert "pNumMax" in str(e.value) or "pNum" in str(e.value)
    # the simulation is still usable after the rejected call
    sim.set_particles(0, a[:1000])
    assert sim.count(0) == 1000
    sim.close()


def test_every_particle_leaving_the_domain_empties_the_store(gpu):
    """Absorbing x walls and velocities of many cells per step toward Xmin:
    after one push and the compaction the store is empty, the wall count
    equals the particle count, as in the oracle."""
    ngx, ngy = 24, 16
    cond = condition(ngx=ngx, ngy=ngy, order=1, ppc=2, xbc="Dirichlet", ybc="periodic", pbc_x="Delete",
                     pbc_y="periodic", dt=5e-11)
    sim = capi.Sim(cond)
    ora = L.OracleSim(ocfg.parse(cond))
    rng = np.random.default_rng(7)
    n = 777
    x = rng.uniform(1, ngx - 1, n).astype(np.float32)
    y = rng.uniform(0, ngy, n).astype(np.float32)
    dx = cond["ParamForField"]["GridSizeOfX"]
    vx = np.full(n, -3.0 * ngx * dx / cond["ParamForTimeIntegration"]["TimeStep"], np.float32)
    z = np.zeros(n, np.float32)
    sim.set_particles(0, _records(x, y, vx, z, z))
    ora.set_particles(0, x, y, vx, z, z, f32=True)
    ora.push(0)
    fo = ora.reduce(0)
    sim.update(0, cond["ParamForTimeIntegration"]["TimeStep"], fused_deposit=False)
    fg = sim.reduce(0)
    assert sim.count(0) == 0 == ora.pnum(0)
    assert fg.particle_number == fo.pnum == 0
    assert list(fg.pinum) == list(fo.pinum)
    assert len(sim.particles(0)) == 0
    sim.close()
