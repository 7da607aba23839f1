"""Condition-file builders and comparison helpers shared by the tests."""
import copy
import json
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")

EC = 4.803204197e-10
ME = 9.10938188e-28
MXE = 1836 * 131.29 * ME


def condition(ngx=32, ngy=24, order=3, ppc=8, xbc="periodic", ybc="periodic", pbc_x=None, pbc_y=None,
              dx=0.005, dy=None, dt=5e-12, te=10.0, ti=0.1, bz_tesla=0.0, boris=2, density=5e10, end=5,
              tol=1e-8, maxiter=200, deposit_mode=0, cur_dens=0, em=1, sources=None, vxe=0.0,
              phi_xmin=0.0, phi_xmax=0.0, pnum_max=None, log_output=1):
    """Two-species (electron, Xe+) condition in the reference's schema."""
    dy = dx if dy is None else dy
    if pbc_x is None:
        pbc_x = "periodic" if xbc == "periodic" else "Delete"
    if pbc_y is None:
        pbc_y = "periodic" if ybc == "periodic" else "Delete"
    n = ppc * ngx * ngy
    cond = {
        "FlagForEquation": {"Particle": 2, "EMField": em, "MCCollision": 0},
        "ParamForTimeIntegration": {"Start": 0, "End": end, "TimeStep": dt, "LogOutput": log_output,
                                    "ParticleOutput": 0, "FieldOutput": 0, "ProgressOutput": 0,
                                    "ProjectName": "test", "RestartName": "test"},
        "ParamForComputing": {"MaximumParticleNumber": pnum_max or (2 * n + 1024), "ThreadGroupSize": 256,
                              "MaxiterForPoisson": maxiter, "ToleranceForPoisson": tol,
                              "DepositMode": deposit_mode},
        "ParamForField": {"NumberOfGridX": ngx, "NumberOfGridY": ngy, "GridSizeOfX": dx, "GridSizeOfY": dy,
                          "InitializeTypeOfE": "Uniform", "AmplitudeOfE": [0.0, 0.0, 0.0],
                          "InitializeTypeOfB": "Uniform", "AmplitudeOfB": [0.0, 0.0, bz_tesla * 1e4],
                          "WeightingOrder": order, "BorisOrder": boris, "FlagForCurDens": cur_dens},
        "ParamForParticle": [
            {"ParticleName": "electron", "pNumSetMethod": "PtclNumPerCell", "pNumValue": ppc, "Charge": -EC,
             "Mass": ME, "WeightSetMethod": "InitialNumDens", "WeightValue": density,
             "GenerateType": "uniform-Gaussian", "InitialTemp": te, "InitialVel": [vxe, 0.0, 0.0]},
            {"ParticleName": "ion_Xe1", "pNumSetMethod": "PtclNumPerCell", "pNumValue": ppc, "Charge": EC,
             "Mass": MXE, "WeightSetMethod": "InitialNumDens", "WeightValue": density,
             "GenerateType": "uniform-Gaussian", "InitialTemp": ti},
        ],
        "SourceForParticle": sources or [],
        "BoundaryConditionForParticle": [
            {"RegionName": "Xmin", "BCType": pbc_x}, {"RegionName": "Xmax", "BCType": pbc_x},
            {"RegionName": "Ymin", "BCType": pbc_y}, {"RegionName": "Ymax", "BCType": pbc_y}],
        "BoundaryConditionForField": [
            {"RegionName": "Xmin", "BCType": xbc, "Value": phi_xmin},
            {"RegionName": "Xmax", "BCType": xbc, "Value": phi_xmax},
            {"RegionName": "Ymin", "BCType": ybc}, {"RegionName": "Ymax", "BCType": ybc}],
    }
    return cond


def with_changes(cond, **kw):
    c = copy.deepcopy(cond)
    for k, v in kw.items():
        sec, key = k.split("__")
        c[sec][key] = v
    return c


def load_golden(name):
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        return json.load(f)


def read_trace(path):
    rows = []
    with open(path) as f:
        header = f.readline().strip().split(",")
        for line in f:
            parts = line.strip().split(",")
            if len(parts) == len(header):
                rows.append([float(x) for x in parts])
    return header, np.array(rows)


def to_aos(x, y, vx, vy, vz, piflag=None):
    from gample_b200.capi import PARTICLE_DTYPE
    a = np.zeros(len(x), PARTICLE_DTYPE)
    a["x"], a["y"], a["vx"], a["vy"], a["vz"] = x, y, vx, vy, vz
    if piflag is not None:
        a["piflag"] = piflag
    return a


def rel_inf(a, b, scale=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = np.max(np.abs(b)) if scale is None else scale
    return float(np.max(np.abs(a - b)) / s) if s > 0 else float(np.max(np.abs(a - b)))


def read_field_file(path):
    """Records of a field/moment file (src/FileIO.mm:109-136, 228-248):
    header ngx, ngy, ngb (int32), dx, dy (float32), then per record a 32-byte
    name, an int32 type id and a float32 array whose shape follows the type
    (0 node, 1 x-shifted, 2 y-shifted, 3 both, 4 potential)."""
    with open(path, "rb") as f:
        buf = f.read()
    ngx, ngy, ngb = np.frombuffer(buf[:12], np.int32)
    dx, dy = np.frombuffer(buf[12:20], np.float32)
    off = 20
    records = {}
    while off < len(buf):
        name = buf[off:off + 32].split(b"\0", 1)[0].decode()
        tid = int(np.frombuffer(buf[off + 32:off + 36], np.int32)[0])
        nx, ny = ngx + 2 * ngb, ngy + 2 * ngb
        ex = {0: (0, 0), 1: (1, 0), 2: (0, 1), 3: (1, 1), 4: (2, 2)}[tid]
        shape = (ny + 1 + ex[1], nx + 1 + ex[0])
        n = shape[0] * shape[1]
        records[name] = (tid, np.frombuffer(buf[off + 36:off + 36 + 4 * n], np.float32).reshape(shape))
        off += 36 + 4 * n
    return {"ngx": int(ngx), "ngy": int(ngy), "ngb": int(ngb), "dx": float(dx), "dy": float(dy)}, records


C_LIGHT = 2.99792458e10
EV_ERG = 1.6021764262e-12


def plasma_scales(density=5e10, te_ev=10.0):
    """Debye length (cm) and electron plasma frequency (rad/s) of an
    electron population (CGS)."""
    import math
    lam_d = math.sqrt(te_ev * EV_ERG / (4 * math.pi * density * EC ** 2))
    wpe = math.sqrt(4 * math.pi * density * EC ** 2 / ME)
    return lam_d, wpe


def config1(end=200, ppc=64, ngx=128, ngy=128, **kw):
    """Plain ES-PIC on a doubly periodic grid: dx = 0.5 Debye length, CIC
    weighting, Boris push in a uniform Bz with w_ce / w_pe = 0.5,
    dt * w_pe = 0.1, Te = 10 eV, Ti = 0.1 eV, 64 particles per cell per
    species, Poisson to 1e-8 relative residual."""
    lam_d, wpe = plasma_scales()
    bz_gauss = 0.5 * wpe * ME * C_LIGHT / EC
    args = dict(ngx=ngx, ngy=ngy, order=1, ppc=ppc, xbc="periodic", ybc="periodic", dx=0.5 * lam_d,
                dt=0.1 / wpe, te=10.0, ti=0.1, bz_tesla=bz_gauss / 1e4, boris=2, density=5e10, end=end, tol=1e-8,
                maxiter=200)
    args.update(kw)
    return condition(**args)


def config2(ppc=8, ngx=512, ngy=512, end=1000, reflux=True, **kw):
    """3rd-order ES-PIC: Dirichlet x walls (phi = 0) with absorbing
    particles, periodic y, Bz = 0.02 T, dt * w_pe = 0.05, dx = 0.5 Debye
    length, Te = 10 eV, Ti = 0.1 eV, every absorbed particle re-injected at
    x = 0 from a flux Maxwellian (GenerateType fluxMaxwellianAtXmin)."""
    lam_d, wpe = plasma_scales()
    sources = None
    if reflux:
        sources = [{"ParticleName": name, "GenerateType": "fluxMaxwellianAtXmin",
                    "SrcSetMethod": "AbsorbedParticleNumber", "GenerateTemp": t}
                   for name, t in (("electron", 10.0), ("ion_Xe1", 0.1))]
    args = dict(ngx=ngx, ngy=ngy, order=3, ppc=ppc, xbc="Dirichlet", ybc="periodic", pbc_x="Delete",
                pbc_y="periodic", dx=0.5 * lam_d, dt=0.05 / wpe, te=10.0, ti=0.1, bz_tesla=0.02, boris=2,
                density=5e10, end=end, tol=1e-8, maxiter=100, sources=sources,
                pnum_max=int(2 * ppc * ngx * ngy * 1.05) + 4096)
    args.update(kw)
    return condition(**args)


def multiset_match(a, b, scales, periods):
    """Match two particle sets (dicts or record arrays with x, y, vx, vy, vz)
    one to one by nearest neighbour in scaled coordinates (positions over
    `scales[0:2]`, velocities over `scales[2:5]`; `periods` gives the
    periodic length of each position coordinate or None). Returns the largest
    matched distance and whether the matching is a bijection."""
    from scipy.spatial import cKDTree
    big = 1e6

    def pts(p):
        cols = []
        for i, c in enumerate(("x", "y", "vx", "vy", "vz")):
            v = np.asarray(p[c], np.float64) / scales[i]
            if i < 2 and periods[i] is not None:
                v = np.mod(v, periods[i] / scales[i])
            else:
                v = v + big / 2
            cols.append(v)
        return np.stack(cols, axis=1)

    box = [periods[i] / scales[i] if i < 2 and periods[i] is not None else 4 * big for i in range(5)]
    tree = cKDTree(pts(b), boxsize=box)
    d, idx = tree.query(pts(a), k=1)
    return float(np.max(d)) if len(d) else 0.0, bool(np.unique(idx).size == len(idx) == len(b["x"]))
