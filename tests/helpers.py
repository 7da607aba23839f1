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
