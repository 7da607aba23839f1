"""Components of the step that the trace and parity tests do not reach,
each against the oracle or the reference's own file format:

  * the hollow-cathode shift of phi (src/EMField.mm:1063-1077);
  * the electric energy, its increment and the Joule sum of the Poisson
    diagnostics (src/EMField.mm:1096-1116);
  * the XML log: section and key names of src/Particle.mm:990-1001,
    src/EMField.mm:1119-1126 and src/main.mm:167-248, read the way the
    reference's tools/parseXML.py reads them, with values against the oracle;
  * B from a file (InitializeTypeOfB From1dXFile, src/EMField.mm:175-197,
    658-687) written by the reference's tools/makeBfld.py, and a push in
    that non-uniform Bz against the oracle;
  * non-finite uploaded records come back as invalid in the flow statistics;
  * the build-added sinusoidal drift of the initial load (the transverse
    current of the Darwin configuration).
"""
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from gample_b200 import capi
from oracle import config as ocfg
from oracle import lib as L
from tests.helpers import GOLDEN, condition, rel_inf, to_aos

pytestmark = pytest.mark.gpu

ERG_TO_EV = 1 / 1.6021764262e-12


def _sync_initial(sim, ora):
    sim.initialize()
    ora.load_initial()
    ora.reset_charge()
    for s in range(2):
        ora.deposit(s)
    return ora.solve_poisson(0.0)


# --------------------------------------------------------- hollow cathode
@pytest.mark.parametrize("pos_cells", [10, 23])
def test_hollow_cathode_phi_shift_matches_oracle(gpu, pos_cells):
    ngx, ngy, dx = 48, 24, 0.005
    cond = condition(ngx=ngx, ngy=ngy, order=3, ppc=4, xbc="Dirichlet", ybc="periodic", phi_xmin=200.0, dx=dx)
    cathode = pos_cells * dx + 0.3 * dx
    cond["BoundaryConditionForField"].append({"RegionName": "hollow-cathode", "Value": cathode})
    sim = capi.Sim(cond)
    ora = L.OracleSim(ocfg.parse(cond), real64=True)
    rng = np.random.default_rng(pos_cells)
    rho = (rng.standard_normal(sim.shape("rho")) * 1e-2 + 5e-3).astype(np.float32)
    sim.set_field("rho", rho)
    st = sim.solve_poisson(0.0)
    ora.set_field("rho", rho)
    st_o = ora.solve_poisson(0.0, tol=1e-13)
    assert st.error <= 1e-8
    assert st_o.mean_cathode != 0.0
    # a 1e-8 residual bounds the solution error through the condition number
    assert abs(st.mean_cathode - st_o.mean_cathode) <= 1e-4 * abs(st_o.mean_cathode)
    for name in ("phi", "Ex", "Ey"):
        assert rel_inf(sim.field(name), ora.field(name)) < 1e-4, name
    # the shift is the reference's linear ramp: phi minus the unshifted fill
    ora_plain = L.OracleSim(ocfg.parse(condition(ngx=ngx, ngy=ngy, order=3, ppc=4, xbc="Dirichlet",
                                                 ybc="periodic", phi_xmin=200.0, dx=dx)), real64=True)
    ora_plain.set_field("rho", rho)
    ora_plain.solve_poisson(0.0, tol=1e-13)
    ramp = ora_plain.field("phi") - sim.field("phi")
    i = np.arange(ramp.shape[1])
    want = (st_o.mean_cathode / 299.792458) * ((i - 1 - 2) * dx) / cathode
    assert np.max(np.abs(ramp - want[None, :])) <= 1e-4 * np.max(np.abs(ora.field("phi")))


# ----------------------------------------------- energy, increment, Joule
def test_energy_increment_and_joule_match_oracle(gpu):
    cond = condition(ngx=48, ngy=32, order=3, ppc=12, xbc="Dirichlet", ybc="periodic", phi_xmin=50.0,
                     cur_dens=1, vxe=3e7, te=10.0, dt=1e-11, end=4)
    sim = capi.Sim(cond)
    ora = L.OracleSim(ocfg.parse(cond))
    st_o = _sync_initial(sim, ora)
    prev_o = st_o.energy
    for cyc in range(4):
        sim.run(1)
        st_o, _ = ora.cycle(cyc + 1, faithful=False)
        st = sim.last_solve()
        assert abs(st.electric_energy - st_o.energy) <= 1e-4 * st_o.energy
        inc_o = st_o.energy - prev_o
        assert abs(st.electric_energy_increment - inc_o) <= 1e-4 * st_o.energy
        assert st_o.joule != 0.0
        # the Joule sum cancels: bound its error by the sum of |E| |j|
        dx, dy = cond["ParamForField"]["GridSizeOfX"], cond["ParamForField"]["GridSizeOfY"]
        dt = cond["ParamForTimeIntegration"]["TimeStep"]
        bound = dt * dx * dy * (np.sum(np.abs(ora.field("Ex") * ora.field("jx"))) +
                                np.sum(np.abs(ora.field("Ey") * ora.field("jy"))))
        assert abs(st.joule_heating - st_o.joule) <= 1e-4 * bound
        # the physical (CGS) field energy carries the reference's missing 1/(4 pi)
        assert abs(st.field_energy_cgs * 4 * np.pi - st.electric_energy) <= 1e-9 * st.electric_energy
        prev_o = st_o.energy


# --------------------------------------------------------------- XML log
def _parse_xml(path, section, tag):
    """tools/parseXML.py:parseXML restated: the values of <tag> in the
    <Section Name=section> of every <Cycle>."""
    root = ET.parse(path).getroot()
    ids, vals = [], []
    for cyc in root.findall("Cycle"):
        ids.append(int(cyc.get("ID")))
        sec = next((s for s in cyc.findall("Section") if s.get("Name") == section), None)
        elem = sec.find(tag) if sec is not None else None
        vals.append(float(elem.text) if elem is not None and elem.text else None)
    return ids, vals


def test_xml_log_sections_keys_and_values(gpu, tmp_path):
    src = [{"ParticleName": "electron", "GenerateType": "hollow-cathode", "SrcSetMethod": "BoundaryCurrentAtXmax",
            "GeneratePosX": [0.15, 0.15], "GenerateTemp": 5}]
    cond = condition(ngx=40, ngy=16, order=3, ppc=8, xbc="Dirichlet", ybc="periodic", phi_xmin=20.0, te=20.0,
                     sources=src, dt=1e-11, end=3)
    log = str(tmp_path / "xmltest")
    sim = capi.Sim(cond, log_name=log, reference_order=True)
    ora = L.OracleSim(ocfg.parse(cond))
    _sync_initial(sim, ora)
    rows = []
    for cyc in range(3):
        sim.run(1)
        st_o, fs_o = ora.cycle(cyc + 1, faithful=False)
        rows.append((st_o, [(f.pnum, f.pulled, list(f.pinum), f.ke) for f in fs_o]))
    sim.close()
    path = log + "_log.xml"
    root = ET.parse(path).getroot()
    assert root.tag == "SimulationLog"
    cycles = root.findall("Cycle")
    assert [int(c.get("ID")) for c in cycles] == [1, 2, 3]
    names = {s.get("Name") for s in cycles[0].findall("Section")}
    for want in ("solvePoisson", "flowout_electron", "flowout_ion_Xe1", "hollowCathode", "elapsedTime",
                 "memoryUsage"):
        assert want in names, want
    keys = {s.get("Name"): {e.tag for e in s} for s in cycles[0].findall("Section")}
    assert keys["solvePoisson"] == {"iteration", "error", "meanCathode", "totalElectricEnergy", "totalEEincrement",
                                    "jouleHeating"}
    assert keys["flowout_electron"] >= {"particleNumber", "pulledPtclNum", "Xmin", "Xmax", "Ymin", "Ymax",
                                        "totalKineticEnergy", "totalKEincrement"}
    assert keys["hollowCathode"] == {"addn_neglected", "addn_injected"}
    assert keys["elapsedTime"] >= {"integCDens_electron", "integCDens_ion_Xe1", "solvePoisson", "update_electron",
                                   "update_ion_Xe1", "reduce_electron", "reduce_ion_Xe1", "artificialIonization",
                                   "hollowCathode"}
    assert keys["memoryUsage"] == {"physicalFootprint", "residentSetSize"}
    # values, read like tools/parseXML.py
    for s, name in enumerate(("electron", "ion_Xe1")):
        _, pn = _parse_xml(path, "flowout_" + name, "particleNumber")
        _, pulled = _parse_xml(path, "flowout_" + name, "pulledPtclNum")
        _, ke = _parse_xml(path, "flowout_" + name, "totalKineticEnergy")
        for k, (st_o, fl) in enumerate(rows):
            assert pn[k] == fl[s][0] and pulled[k] == fl[s][1], (name, k)
            for w, wall in enumerate(("Xmin", "Xmax", "Ymin", "Ymax")):
                assert _parse_xml(path, "flowout_" + name, wall)[1][k] == fl[s][2][w]
            assert abs(ke[k] - fl[s][3] * ERG_TO_EV) <= 1e-5 * fl[s][3] * ERG_TO_EV
    _, ee = _parse_xml(path, "solvePoisson", "totalElectricEnergy")
    _, err = _parse_xml(path, "solvePoisson", "error")
    for k, (st_o, _) in enumerate(rows):
        assert abs(ee[k] - st_o.energy * ERG_TO_EV) <= 1e-4 * st_o.energy * ERG_TO_EV
        assert err[k] <= 1e-8
    _, t_us = _parse_xml(path, "elapsedTime", "update_electron")
    assert all(v is not None and v >= 0 for v in t_us)
    _, rss = _parse_xml(path, "memoryUsage", "residentSetSize")
    _, foot = _parse_xml(path, "memoryUsage", "physicalFootprint")
    assert all(r > 0 and f >= r for r, f in zip(rss, foot))


# ------------------------------------------------------------ From1dXFile
def _read_1d(path):
    """EMField.mm:658-687: int32 n, float32 d, then n + 1 float32."""
    with open(path, "rb") as f:
        buf = f.read()
    n = int(np.frombuffer(buf[:4], np.int32)[0])
    return np.frombuffer(buf[8:8 + 4 * (n + 1)], np.float32)


def test_b_from_1d_file_and_push_match_oracle(gpu):
    ngx, ngy = 48, 16
    cond = condition(ngx=ngx, ngy=ngy, order=3, ppc=16, xbc="Dirichlet", ybc="periodic", pbc_x="Delete", te=10.0,
                     dt=2e-11, dx=0.005)
    f = cond["ParamForField"]
    f["InitializeTypeOfB"] = "From1dXFile"
    for c in ("x", "y", "z"):
        f["FilePathOfB" + c] = os.path.join(GOLDEN, f"B{c}_1dx.bin")
    sim = capi.Sim(cond)
    nx, ny = ngx + 2, ngy + 2
    bz_in = _read_1d(os.path.join(GOLDEN, "Bz_1dx.bin"))
    assert len(bz_in) == nx + 2
    want = np.broadcast_to((bz_in.astype(np.float64) * 1e4).astype(np.float32)[None, :], (ny + 2, nx + 2))
    assert np.array_equal(sim.field("Bz"), want)
    # a push in this Bz (per-particle Bz gather) against the oracle
    ora = L.OracleSim(ocfg.parse(dict(cond, ParamForField=dict(f, InitializeTypeOfB="Uniform",
                                                               AmplitudeOfB=[0.0, 0.0, 0.0]))))
    ora.load_initial()
    ora.set_field("Bz", want)
    rng = np.random.default_rng(7)
    for name in ("Ex", "Ey"):
        ora.set_field(name, rng.standard_normal(ora.shape(name)) * 10.0)
        sim.set_field(name, ora.field(name).astype(np.float32))
    for s in range(2):
        o = ora.particles(s, f32=True)
        sim.set_particles(s, to_aos(o["x"], o["y"], o["vx"], o["vy"], o["vz"]))
        ora.push(s)
        sim.update(s, 2e-11, fused_deposit=False)
        g, r = sim.particles(s), ora.particles(s, f32=True)
        live = (g["piflag"] == 0) & (r["piflag"] == 0)
        assert np.count_nonzero(live) > 0.95 * len(g)
        vth = float(np.sqrt(np.mean(r["vx"][live].astype(np.float64) ** 2)))
        for c in ("vx", "vy", "vz"):
            a, b = g[c][live].astype(np.float64), r[c][live].astype(np.float64)
            assert np.all(np.abs(a - b) <= 1e-5 * (np.abs(b) + vth)), c


# --------------------------------------------------- non-finite uploads
def test_non_finite_uploads_are_counted_invalid(gpu):
    cond = condition(ngx=32, ngy=16, order=3, ppc=8, xbc="Dirichlet", ybc="periodic", dt=1e-11)
    sim = capi.Sim(cond)
    recs = sim.particles(0)
    n = len(recs)
    bad = {}
    bad[3] = ("x", np.nan)
    bad[17] = ("y", np.inf)
    bad[40] = ("vx", np.inf)
    bad[41] = ("vy", -np.inf)
    bad[99] = ("vz", np.nan)
    bad[120] = ("x", 1e30)  # far outside the arrays
    bad[121] = ("y", -5.0)
    for k, (c, v) in bad.items():
        recs[c][k] = v
    sim.set_particles(0, recs)
    sim.update(0, 1e-11, fused_deposit=False)
    fs = sim.reduce(0)
    wall = sum(fs.pinum) * -1  # electrons count -1 per particle
    assert fs.invalid == len(bad)
    assert fs.particle_number == n - len(bad) - wall
    assert fs.pulled == len(bad) + wall
    g = sim.particles(0)
    assert len(g) == fs.particle_number
    assert np.all(np.isfinite(g["x"])) and np.all(np.isfinite(g["vx"])) and np.all(np.isfinite(g["vz"]))


# ------------------------------------------------- sinusoidal initial drift
def test_sinusoidal_initial_drift_profile(gpu):
    """ParamForParticle SinusoidalDriftVel (build addition): the initial
    load's electron velocities get a drift a * sin(2 pi (x - Xmin) / Lx) per
    component on top of the reference's Maxwellian; the ions keep theirs.
    The binned mean vy follows the profile within 5 standard errors, and the
    loader without the key is unchanged (bit-exact against the oracle)."""
    ngx, ngy = 64, 16
    cond = condition(ngx=ngx, ngy=ngy, order=1, ppc=64, xbc="periodic", ybc="periodic")
    plain = capi.Sim(cond)
    plain.initialize()
    ref = [plain.particles(s) for s in range(2)]
    plain.close()
    vte = float(np.sqrt(np.mean(ref[0]["vx"].astype(np.float64) ** 2)))
    amp = 0.1 * vte
    cond["ParamForParticle"][0]["SinusoidalDriftVel"] = [0.0, amp, 0.0]
    sim = capi.Sim(cond)
    sim.initialize()
    e, i = sim.particles(0), sim.particles(1)
    ngb = sim.ngb
    sim.close()
    key = ["x", "y", "vx", "vz"]
    np.testing.assert_array_equal(np.sort(e, order=key)[key], np.sort(ref[0], order=key)[key])
    np.testing.assert_array_equal(np.sort(i, order=key), np.sort(ref[1], order=key))
    bins = np.floor((e["x"].astype(np.float64) - ngb) / ngx * 16).astype(int)
    for b in range(16):
        sel = bins == b
        vy = e["vy"][sel].astype(np.float64)
        xm = (b + 0.5) / 16
        want = amp * np.sin(2 * np.pi * xm)
        se = np.std(vy) / np.sqrt(len(vy))
        # the profile varies across a bin: its mean is sin at the centre times sinc
        want *= np.sinc(1 / 16)
        assert abs(vy.mean() - want) < 5 * se + 0.002 * amp, (b, vy.mean(), want, se)
