"""The CUDA path against the oracle at the benchmark configurations.

  * config 1 in full: 128 x 128 doubly periodic, CIC, 64 particles per cell
    per species (2.1 M particles), Bz at w_ce / w_pe = 0.5, dt * w_pe = 0.1,
    Poisson to 1e-8. Twenty cycles side by side: particle counts, the CSV
    probe and the field energy every cycle; phi, E and the whole particle
    multiset (matched one to one) at the end. Then the full 200 steps:
    the kinetic, field and total energy histories agree statistically.
  * config-2 geometry (512 x 512, order 3, Dirichlet x with absorbing walls,
    periodic y, Bz 0.02 T, dt * w_pe = 0.05): one push + fused deposit of
    the atomic mode at 64 particles per cell (cell-sorted chunks cover a few
    cells, so the gather goes through the per-cell polynomial tables and the
    deposit through the lane-private windows) compared particle by particle;
    four whole cycles at 8 particles per cell with a re-sort every second
    cycle, compaction and flux-Maxwellian re-injection, compared cycle by
    cycle; the 512 x 512 multigrid solve measured against the oracle's CSR
    system and its tight FP64 solve.

Tolerances: push 1e-5 relative (velocities against |v| + v_th, positions
against the displacement), deposit 2e-7 of the peak charge (atomic mode),
Poisson relative residual <= 1e-8, E within 1e-4 of a 1e-12 FP64 solve; over
twenty cycles the two runs part by FP32 rounding only, so the probe, field
energy and particle states must agree to 1e-4 of their scales.
"""
import numpy as np
import pytest

from gample_b200 import capi
from oracle import config as ocfg
from oracle import lib as L
from tests.helpers import config1, config2, multiset_match, rel_inf, to_aos

pytestmark = pytest.mark.gpu


def _sync_initial(sim, ora):
    """initialize() on the device (initial deposit + solve, src/main.mm:136-141)
    and the same on the oracle."""
    sim.initialize()
    ora.load_initial()
    ora.reset_charge()
    for s in range(2):
        ora.deposit(s)
    ora.solve_poisson(0.0)


def _vth(p):
    return float(np.sqrt(np.mean(np.asarray(p["vx"], np.float64) ** 2)))


# ------------------------------------------------------------------ config 1
def _within_fp32_spread(label, err_gpu, err_fp32, floor=1e-6):
    """Over many cycles two FP32 runs part through the particles' chaotic
    motion. The CUDA path must stay as close to the FP64 oracle as the FP32
    oracle (the reference's arithmetic) does: within 3 times its distance."""
    print(f"{label}: CUDA vs FP64 oracle {err_gpu:.2e}, FP32 oracle vs FP64 oracle {err_fp32:.2e}")
    assert err_gpu <= 3.0 * err_fp32 + floor, (label, err_gpu, err_fp32)


def test_config1_twenty_cycles_match_oracle(gpu):
    cond = config1(end=20)
    sim = capi.Sim(cond)
    ora = L.OracleSim(ocfg.parse(cond))
    ora64 = L.OracleSim(ocfg.parse(cond), real64=True)
    _sync_initial(sim, ora)
    ora64.load_initial()
    ora64.reset_charge()
    for s in range(2):
        ora64.deposit(s)
    ora64.solve_poisson(0.0)
    probes = {"g": [], "o": [], "d": []}
    ee = {"g": [], "o": [], "d": []}
    for cyc in range(20):
        sim.run(1)
        st_o, _ = ora.cycle(cyc + 1, faithful=False)
        st_d, _ = ora64.cycle(cyc + 1, faithful=False)
        st = sim.last_solve()
        for s in range(2):
            assert sim.count(s) == ora.pnum(s) == ora64.pnum(s) == 128 * 128 * 64
        assert st.error <= 1e-8
        for k, v in (("g", st), ("o", st_o), ("d", st_d)):
            probes[k].append(list(v.probe))
        ee["g"].append(st.electric_energy)
        ee["o"].append(st_o.energy)
        ee["d"].append(st_d.energy)
    p = {k: np.array(v) for k, v in probes.items()}
    for c in range(3):
        scale = np.max(np.abs(p["d"][:, c]))
        e_g = np.max(np.abs(p["g"][:, c] - p["d"][:, c])) / scale
        e_o = np.max(np.abs(p["o"][:, c] - p["d"][:, c])) / scale
        _within_fp32_spread(f"config1 probe {c}", e_g, e_o)
        assert e_g < 1e-3
    # field energy against its largest value (the first solve's is exactly 0
    # in FP64: the load puts every ion on an electron)
    e = {k: np.array(v) for k, v in ee.items()}
    emax = np.max(e["d"])
    _within_fp32_spread("config1 field energy", np.max(np.abs(e["g"] - e["d"])) / emax,
                        np.max(np.abs(e["o"] - e["d"])) / emax)
    # fields of the last solve
    for name in ("Ex", "Ey", "phi"):
        _within_fp32_spread(f"config1 {name}", rel_inf(sim.field(name), ora64.field(name)),
                            rel_inf(ora.field(name), ora64.field(name)))
    # the whole particle multiset, matched one to one
    for s in range(2):
        g, o, d = sim.particles(s), ora.particles(s, f32=True), ora64.particles(s)
        assert np.all(g["piflag"] == 0)
        vth = _vth(d)
        sc = (1.0, 1.0, vth, vth, vth)
        dg, bij_g = multiset_match(g, d, sc, (128.0, 128.0))
        # the FP32 oracle drifts further: its nearest neighbour may be
        # another particle, so only the CUDA path must match one to one
        do, _ = multiset_match(o, d, sc, (128.0, 128.0))
        print(f"config1 species {s}: one-to-one {bij_g}")
        assert bij_g, s
        _within_fp32_spread(f"config1 species {s} particles (cells / v_th)", dg, do)
        assert dg < 1e-3


@pytest.mark.slow
def test_config1_full_run_energy_history_matches_oracle(gpu):
    """200 steps (the configuration's length): trajectories decorrelate
    (FP32 rounding grows through the particles' chaotic motion), so the
    comparison is statistical: kinetic energy per species and field energy
    averaged over the last 100 steps agree within a few per cent, and both
    runs conserve total energy to the same degree."""
    cond = config1(end=200)
    sim = capi.Sim(cond)
    ora = L.OracleSim(ocfg.parse(cond))
    _sync_initial(sim, ora)
    hist = {"g": [], "o": []}
    for cyc in range(200):
        sim.run(1)
        st_o, fs_o = ora.cycle(cyc + 1, faithful=False)
        st = sim.last_solve()
        ke_g = sum(sim.last_flow(s).kinetic_energy for s in range(2))
        ke_o = sum(f.ke for f in fs_o)
        # CGS field energy: the logged sum E^2 dx dy / 2 over 4 pi
        hist["g"].append((ke_g, st.electric_energy / (4 * np.pi)))
        hist["o"].append((ke_o, st_o.energy / (4 * np.pi)))
    g, o = np.array(hist["g"]), np.array(hist["o"])
    assert abs(g[100:, 0].mean() / o[100:, 0].mean() - 1) < 0.01
    assert abs(g[100:, 1].mean() / o[100:, 1].mean() - 1) < 0.05
    tot_g, tot_o = g.sum(axis=1), o.sum(axis=1)
    drift_g = abs(tot_g[-1] / tot_g[0] - 1)
    drift_o = abs(tot_o[-1] / tot_o[0] - 1)
    print(f"config1 200 steps: KE ratio {g[100:, 0].mean() / o[100:, 0].mean():.4f}, field energy ratio "
          f"{g[100:, 1].mean() / o[100:, 1].mean():.4f}, total-energy drift {drift_g:.2e} (oracle {drift_o:.2e})")
    assert drift_g < 0.01 and drift_o < 0.01, (drift_g, drift_o)


# ------------------------------------------------------------------ config 2
def _tile_order(x, y):
    ix, iy = np.floor(x).astype(np.int64), np.floor(y).astype(np.int64)
    return np.lexsort((ix % 8, iy % 8, ix // 8, iy // 8))


def test_config2_push_and_fused_deposit_at_64ppc_match_oracle(gpu):
    cond = config2(ppc=64, reflux=False)
    sim = capi.Sim(cond)
    ora = L.OracleSim(ocfg.parse(cond))
    ora.load_initial()
    rng = np.random.default_rng(512)
    for name in ("Ex", "Ey"):
        ora.set_field(name, rng.standard_normal(ora.shape(name)) * 30.0)
        sim.set_field(name, ora.field(name).astype(np.float32))
    dt = cond["ParamForTimeIntegration"]["TimeStep"]
    ngx = ngy = 512
    for s in range(2):
        o = ora.particles(s, f32=True)
        perm = _tile_order(o["x"], o["y"])
        o = {c: o[c][perm] for c in ("x", "y", "vx", "vy", "vz")}
        ora.set_particles(s, o["x"], o["y"], o["vx"], o["vy"], o["vz"], f32=True)
        sim.set_particles(s, to_aos(o["x"], o["y"], o["vx"], o["vy"], o["vz"]))
        ora.push(s)
        sim.reset_charge()
        sim.update(s, dt, fused_deposit=True)
        g, r = sim.particles(s), ora.particles(s, f32=True)
        xr, yr = r["x"].astype(np.float64), r["y"].astype(np.float64)
        near_wall = np.abs(xr - np.round(xr)) < 1e-4
        assert not np.any((g["piflag"] != r["piflag"]) & ~near_wall)
        if s == 0:
            assert np.count_nonzero(r["piflag"]) > 0  # electrons reach the walls
        live = (g["piflag"] == 0) & (r["piflag"] == 0)
        vth = _vth({"vx": r["vx"][live]})
        for c in ("vx", "vy", "vz"):
            a, b = g[c][live].astype(np.float64), r[c][live].astype(np.float64)
            assert np.all(np.abs(a - b) <= 1e-5 * (np.abs(b) + vth)), c
        cst = ora.species_consts(s)
        for c, k, period in (("x", "constX", None), ("y", "constY", ngy)):
            x0 = o[c][live].astype(np.float64)
            dg = g[c][live].astype(np.float64) - x0
            dr = r[c][live].astype(np.float64) - x0
            if period:
                dg = (dg - dr + period / 2) % period - period / 2 + dr
            ulp = np.spacing((np.abs(r[c][live]) + (period or 0)).astype(np.float32)).astype(np.float64)
            assert np.all(np.abs(dg - dr) <= 4 * ulp + 1e-5 * (np.abs(dr) + vth * cst[k])), c
        # The fused deposit of the pushed particles against an exact deposit of
        # the same states. The states must be taken as cell + offset: a float
        # position near x = 512 carries 3e-5 cells of rounding, which would
        # move the reference sum by more than the deposit's own error.
        raw = sim.particles_raw(s)
        ok = raw["cell"] >= 0
        ix = (raw["cell"][ok] & 0xFFFF).astype(np.int32)
        iy = (raw["cell"][ok] >> 16).astype(np.int32)
        acc = L.det_deposit_rho(3, ngx, ngy, 1, ix, iy, raw["ox"][ok], raw["oy"][ok])  # 2^-40 fixed point
        exact = acc.astype(np.float64) * (np.float64(np.float32(cst["scale"])) * 2.0 ** -40)
        err = rel_inf(sim.field("rho"), exact)
        print(f"config2 64 ppc species {s}: fused deposit error {err:.2e} of the peak charge")
        assert err < 2e-7, s


def _flux_maxwellian_moments(p, vth, label):
    """Velocity moments of flux-Maxwellian re-injected particles: vx =
    v_th sqrt(-ln r) (a flux-weighted half Maxwellian), vy, vz Gaussian
    with variance v_th^2 / 2; bounds at 6 standard errors."""
    n = len(p["vx"])
    assert n > 200, label
    vx, vy, vz = (np.asarray(p[c], np.float64) / vth for c in ("vx", "vy", "vz"))
    se = 6.0 / np.sqrt(n)
    assert np.all(vx > 0), label
    assert abs(vx.mean() - np.sqrt(np.pi) / 2) < se * np.sqrt(1 - np.pi / 4), label
    assert abs((vx ** 2).mean() - 1.0) < se * 1.0, label
    for v in (vy, vz):
        assert abs(v.mean()) < se * np.sqrt(0.5), label
        assert abs((v ** 2).mean() - 0.5) < se * np.sqrt(0.5), label


def test_config2_cycles_with_resort_compaction_reflux_match_oracle(gpu):
    cond = config2(ppc=8, end=4)
    cond["ParamForComputing"]["SortInterval"] = 2
    sim = capi.Sim(cond)
    ora = L.OracleSim(ocfg.parse(cond))
    _sync_initial(sim, ora)
    dt = cond["ParamForTimeIntegration"]["TimeStep"]
    injected = {0: [], 1: []}
    vth_src = [np.sqrt(2 * 1.3806503e-16 * t * 11604.0 / m) for t, m in ((10.0, 9.10938188e-28),
                                                                         (0.1, 1836 * 131.29 * 9.10938188e-28))]
    for cyc in range(4):
        n_before = [ora.pnum(s) for s in range(2)]
        sim.run(1)
        st_o, fs_o = ora.cycle(cyc + 1, faithful=False)
        st = sim.last_solve()
        assert st.error <= 1e-8
        for s in range(2):
            fg = sim.last_flow(s)
            assert list(fg.pinum) == list(fs_o[s].pinum), (cyc, s)
            assert fg.pulled == fs_o[s].pulled, (cyc, s)
            assert sim.count(s) == ora.pnum(s), (cyc, s)
            addn = fs_o[s].pulled
            assert ora.pnum(s) == n_before[s]  # every absorbed particle comes back
            if s == 0:
                assert addn > 0
            if addn:
                # the newest particles: the same RNG slots on both sides
                g, o = sim.particles(s)[-addn:], ora.particles(s, f32=True)
                o = {c: o[c][-addn:] for c in ("x", "y", "vx", "vy", "vz")}
                for c in ("vx", "vy", "vz"):
                    np.testing.assert_allclose(g[c], o[c], rtol=2e-6, atol=2e-6 * vth_src[s])
                for c in ("x", "y"):
                    np.testing.assert_allclose(g[c], o[c], rtol=2e-6, atol=1e-5)
                injected[s].append(g)
        # The CSV probe (phi, Ex, Ey at one node) against the field's own
        # scale. The first cycle solves the charge of the load, where every
        # ion sits on an electron: rho is rounding noise on both sides, so
        # the comparison starts with the second cycle.
        for c, name in enumerate(("phi", "Ex", "Ey")):
            scale = np.max(np.abs(ora.field(name)))
            err = abs(st.probe[c] - st_o.probe[c]) / scale
            print(f"config2 cycle {cyc} probe {name}: error {err:.2e} of the field's peak")
            if cyc > 0:
                assert err <= 1e-4, (cyc, name, st.probe[c], st_o.probe[c])
    # electrons only: the cold ions (Ti = 0.1 eV) hardly reach a wall in four steps
    _flux_maxwellian_moments(np.concatenate(injected[0]), vth_src[0], "electrons")
    # the 512 x 512 multigrid: residual on the oracle's CSR system and E
    # against the oracle's tight FP64 solve of the same folded charge
    rho = sim.field("rho")
    st = sim.solve_poisson(dt)
    assert st.error <= 1e-8
    ora64 = L.OracleSim(ocfg.parse(cond), real64=True)
    ora64.set_field("rho", sim.field("rho"))
    res = ora64.poisson_residual(sim.field("sol").ravel())
    assert res <= 1.05e-8, res
    ora64.set_field("rho", rho)
    ora64.solve_poisson(dt, tol=1e-12)
    for name in ("Ex", "Ey", "phi"):
        assert rel_inf(sim.field(name), ora64.field(name)) < 1e-4, name
