"""Velocity moments (src/Moment.mm), the binary field/moment/phase-space
outputs and the restart files (src/FileIO.mm)."""
import os

import numpy as np
import pytest

from gample_b200 import capi
from oracle import config as ocfg
from oracle import lib as L
from tests.helpers import ME, MXE, condition, read_field_file, with_changes

C_LIGHT = 2.99792458e10


# ---------------------------------------------------------------- oracle side (CPU)
def test_oracle_moments_of_a_maxwellian():
    """n and P = n k T of a loaded Maxwellian, and the reference's FP32
    summation agrees with the FP64 one."""
    cond = condition(ngx=16, ngy=16, order=3, ppc=64, te=10.0)
    ora = L.OracleSim(ocfg.parse(cond))
    ora.load_initial()
    ref = ora.moments(0, build=False)
    bld = ora.moments(0, build=True)
    inner = (slice(4, -4), slice(4, -4))
    dens = 5e10
    assert abs(np.mean(bld["n"][inner]) / dens - 1) < 0.02
    kT = 10.0 * 1.6021764262e-12
    # P_xx = n m <(v - u)^2> = n k T for each direction of a Maxwellian
    assert abs(np.mean(bld["Pxx"][inner]) / (dens * kT) - 1) < 0.05
    assert abs(np.mean(bld["Pzz"][inner]) / (dens * kT) - 1) < 0.05
    for k in ("n", "Pxx", "Pyy"):
        s = np.max(np.abs(bld[k]))
        assert np.max(np.abs(ref[k] - bld[k])) < 1e-5 * s, k


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("order", [1, 3, 5])
def test_moments_match_oracle(gpu, order):
    cond = condition(ngx=40, ngy=28, order=order, ppc=16, xbc="Dirichlet", ybc="periodic", bz_tesla=0.02,
                     vxe=3e7, end=3)
    sim = capi.Sim(cond)
    sim.initialize()
    sim.run(3)
    ora = L.OracleSim(ocfg.parse(cond))
    for s in range(2):
        g = sim.particles(s)
        ora.set_particles(s, g["x"], g["y"], g["vx"], g["vy"], g["vz"])
        got = sim.moments(s)
        want = ora.moments(s, build=True)
        n_max = np.max(want["n"])
        assert np.max(np.abs(got["n"] - want["n"])) < 1e-5 * n_max
        dense = want["n"] > 0.2 * n_max
        for k in ("ux", "uy", "uz"):
            vs = np.sqrt(np.max(want["Pxx"]) / n_max / (ME if s == 0 else MXE))
            assert np.max(np.abs(got[k] - want[k])[dense]) < 1e-4 * vs, (s, k)
        for k in ("Pxx", "Pxy", "Pxz", "Pyy", "Pyz", "Pzz"):
            ps = np.max(np.abs(want["Pxx"]))
            assert np.max(np.abs(got[k] - want[k])[dense]) < 1e-4 * ps, (s, k)
    sim.close()


@pytest.mark.gpu
def test_binary_outputs_and_restart(gpu, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    os.mkdir("bin")
    cond = condition(ngx=32, ngy=24, order=3, ppc=8, xbc="Dirichlet", ybc="periodic", em=2, cur_dens=1, end=4)
    cond["ParamForTimeIntegration"].update(FieldOutput=2, ParticleOutput=1, ProgressOutput=2, ProjectName="out")
    sim = capi.Sim(cond, log_name="out_test")
    sim.initialize()
    sim.run(4)
    for c in (0, 2, 4):
        assert os.path.exists(f"bin/out_EMField_{c:08d}.bin")
        for name in ("electron", "ion_Xe1"):
            assert os.path.exists(f"bin/out_Moments_{name}_{c:08d}.bin")
    mesh, rec = read_field_file("bin/out_EMField_00000004.bin")
    assert (mesh["ngx"], mesh["ngy"], mesh["ngb"]) == (32, 24, 1)
    assert list(rec) == ["rho", "phi", "Ex", "Ey", "Bz", "jx", "jy", "delEx", "delEy", "delBz"]
    # the last output was written after cycle 4's solve; phi and E are unchanged since
    sv = np.float32(1 / (1e8 / C_LIGHT))
    np.testing.assert_array_equal(rec["phi"][1], sim.field("phi").astype(np.float32) * sv)
    gv = np.float32(1 / (1e6 / C_LIGHT))
    np.testing.assert_array_equal(rec["Ex"][1], sim.field("Ex") * gv)
    np.testing.assert_array_equal(rec["Ey"][1], sim.field("Ey") * gv)
    # moments file of the final state: the moments computed now (FP32
    # shared-memory sums in atomic order: equal to a few ulp)
    mesh, mrec = read_field_file("bin/out_Moments_electron_00000004.bin")
    mom = sim.moments(0)
    np.testing.assert_allclose(mrec["electron_n"][1], mom["n"], rtol=2e-6, atol=0)
    pmax = np.max(np.abs(mom["Pxx"]))
    np.testing.assert_allclose(mrec["electron_Pxx"][1], mom["Pxx"] * np.float32(0.1), rtol=0, atol=1e-5 * pmax)
    # phase space: one record (cycle, x, y, vx, vy, vz) per cycle for particles 0..19
    ps = np.fromfile("bin/out_PhaseSpace_electron_0.bin", dtype=np.dtype(
        [("cycle", "<i4"), ("x", "<f4"), ("y", "<f4"), ("vx", "<f4"), ("vy", "<f4"), ("vz", "<f4")]))
    assert list(ps["cycle"]) == [1, 2, 3, 4]
    # restart files: the particle records after cycle 4
    saved = [sim.particles(s) for s in range(2)]
    for s, name in enumerate(("electron", "ion_Xe1")):
        raw = np.fromfile(f"bin/out_ProgressData_{name}_00000004.bin", dtype=saved[s].dtype)
        np.testing.assert_array_equal(raw, saved[s])
    sim.close()
    # a run restarted from cycle 4 starts from exactly those particles
    cond2 = with_changes(cond)
    cond2["ParamForTimeIntegration"].update(Start=4, End=6, RestartName="out", ProjectName="re")
    sim2 = capi.Sim(cond2, log_name="re_test")
    sim2.initialize()
    key = ["x", "y", "vx", "vy", "vz", "piflag"]  # initialize() re-sorts the loaded particles by cell
    for s in range(2):
        np.testing.assert_array_equal(np.sort(sim2.particles(s), order=key), np.sort(saved[s], order=key))
    sim2.run(2)
    assert sim2.cycle_number() == (6, pytest.approx(6 * cond["ParamForTimeIntegration"]["TimeStep"]))
    sim2.close()
