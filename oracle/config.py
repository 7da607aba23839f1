"""Restatement of gample's JSON condition parser (test infrastructure only).

Mirrors src/Init.mm:27-301 (parse) and :304-394 (per-section defaults),
src/EMField.mm:199-234 (field boundary strings), src/Particle.mm:459-514
(particle boundary strings) and src/Collision.mm:220-233, 368-377 (generator
type strings). Only tests/, smoke() and bench.py's CPU baseline use it; the
product parses the same schema in C++.
"""
from __future__ import annotations

import json
import math
import struct

EC = 4.803204197e-10          # src/Constant.h:4
C_LIGHT = 2.99792458e10       # src/Constant.h:5
EV_TO_K = 11604.0             # src/Constant.h:13
JTOSJ = 1 / (10 / C_LIGHT * 1e4)  # src/Constant.h:22

DEFAULTS = {  # src/Init.mm:304-394
    "FlagForEquation": {"Particle": 0, "EMField": 0, "MCCollision": 0},
    "ParamForTimeIntegration": {"Start": 0, "End": 0, "TimeStep": 0, "LogOutput": 0, "ParticleOutput": 0,
                                "FieldOutput": 0, "ProgressOutput": 0, "ProjectName": "undefined",
                                "RestartName": "undefined"},
    "ParamForComputing": {"MaximumParticleNumber": 0.08, "ThreadGroupSize": 256, "IntegrationChunkSize": 256,
                          "AggregationThreshold": 0.1, "ChebyshevDegree": 5, "AMGCycleType": 1,
                          "MaxiterForPoisson": 200, "ToleranceForPoisson": 1e-7},
    "ParamForParticle": {"ParticleName": "undefined", "pNumSetMethod": "undefined", "pNumValue": 0, "Charge": 0,
                         "Mass": -1, "WeightSetMethod": "undefined", "WeightValue": 0, "GenerateType": "undefined",
                         "InitialPosX": [-1, -1], "InitialPosY": [-1, -1], "InitialVel": [0, 0, 0],
                         "InitialTemp": 0},
    "BoundaryCondition": {"RegionName": "undefined", "BCType": "undefined", "Value": 0},
    "SourceForParticle": {"ParticleName": "undefined", "GenerateType": "undefined", "SrcSetMethod": "undefined",
                          "SrcVal": 0, "GeneratePosX": [-1, -1], "GeneratePosY": [-1, -1],
                          "GenerateVel": [0, 0, 0], "GenerateTemp": 0, "GenVelForElectron": [0, 0, 0],
                          "GenTempForElectron": 0},
    "ParamForField": {"NumberOfGridX": 0, "NumberOfGridY": 0, "GridSizeOfX": 0, "GridSizeOfY": 0,
                      "InitializeTypeOfE": "undefined", "AmplitudeOfE": [0, 0, 0], "FilePathOfEx": "undefined",
                      "FilePathOfEy": "undefined", "FilePathOfEz": "undefined", "InitializeTypeOfB": "undefined",
                      "AmplitudeOfB": [0, 0, 0], "FilePathOfBx": "undefined", "FilePathOfBy": "undefined",
                      "FilePathOfBz": "undefined", "WeightingOrder": 5, "BorisOrder": 2, "FlagForCurDens": 0,
                      "PtclPosOffset": 0},
}

FIELD_BC = {"periodic": 0, "Dirichlet": 1, "Neumann": 2}
PARTICLE_BC = {"periodic": 0, "Delete": 1, "Reflect": 2}
LOAD_GEN = {"uniform-Gaussian": 0, "Xsinusoidal-Gaussian": 1, "Ysinusoidal-Gaussian": 2, "quietStart": 4,
            "Xgaussian-Gaussian": 5, "Ygaussian-Gaussian": 6}
# Source generator codes; 7 (flux-Maxwellian re-injection at Xmin) is the
# build's addition for the absorbing-wall workload and has no reference code.
SOURCE_GEN = {"uniformIonization": 0, "XsinusoidalIonization": 1, "YsinusoidalIonization": 2,
              "hollow-cathode": 3, "fluxMaxwellianAtXmin": 7}
WALLS = ("Xmin", "Xmax", "Ymin", "Ymax")


class ConfigError(ValueError):
    """Raised where the reference's parser returns nil."""


def _int(v):
    """NSNumber/NSString integerValue: truncation toward zero."""
    if isinstance(v, bool):
        return int(v)
    if isinstance(v, (int, float)):
        return int(v) if math.isfinite(v) else 0
    if isinstance(v, str):
        s = v.strip()
        digits = ""
        for i, ch in enumerate(s):
            if ch.isdigit() or (i == 0 and ch in "+-"):
                digits += ch
            else:
                break
        try:
            return int(digits)
        except ValueError:
            return 0
    return 0


def _dbl(v):
    if isinstance(v, bool):
        return float(v)
    if isinstance(v, (int, float)):
        return float(v)
    if isinstance(v, str):
        try:
            return float(v)
        except ValueError:
            return 0.0
    return 0.0


def _f32(x):
    """Round to float32 (src/Init.h:27-36 stores these members as float)."""
    return struct.unpack("f", struct.pack("f", x))[0]


def _vec(v):
    return [_dbl(x) for x in v] if isinstance(v, list) else []


def _merged(section_defaults, d):
    m = dict(section_defaults)
    m.update(d)
    return m


def parse(path_or_dict):
    """Parse a condition file exactly as src/Init.mm:27-301 does."""
    if isinstance(path_or_dict, dict):
        root = path_or_dict
    else:
        with open(path_or_dict) as f:
            root = json.load(f)
    if not isinstance(root, dict):
        raise ConfigError("top level is not an object")
    out = {}
    flag = root.get("FlagForEquation")
    if not isinstance(flag, dict):
        raise ConfigError("FlagForEquation")
    m = _merged(DEFAULTS["FlagForEquation"], flag)
    out["flag"] = {k: _int(m[k]) for k in ("Particle", "EMField", "MCCollision")}

    t = root.get("ParamForTimeIntegration")
    if not isinstance(t, dict):
        raise ConfigError("ParamForTimeIntegration")
    m = _merged(DEFAULTS["ParamForTimeIntegration"], t)
    out["time"] = {"Start": _int(m["Start"]), "End": _int(m["End"]), "TimeStep": _dbl(m["TimeStep"]),
                   "LogOutput": _int(m["LogOutput"]), "ParticleOutput": _int(m["ParticleOutput"]),
                   "FieldOutput": _int(m["FieldOutput"]), "ProgressOutput": _int(m["ProgressOutput"]),
                   "ProjectName": m["ProjectName"], "RestartName": m["RestartName"]}

    c = root.get("ParamForComputing")
    if not isinstance(c, dict):
        raise ConfigError("ParamForComputing")
    m = _merged(DEFAULTS["ParamForComputing"], c)
    out["comp"] = {"pNumMax": _int(m["MaximumParticleNumber"]) & 0xFFFFFFFF,
                   "threadGroupSize": _int(m["ThreadGroupSize"]),
                   "integrationChunkSize": _int(m["IntegrationChunkSize"]),
                   "aggrThreshold": _f32(_dbl(m["AggregationThreshold"])), "chebDegree": _int(m["ChebyshevDegree"]),
                   "amgCycleType": _int(m["AMGCycleType"]), "maxiter": _int(m["MaxiterForPoisson"]),
                   "tolerance": _f32(_dbl(m["ToleranceForPoisson"])),
                   # build addition: master seed of the RNG streams (the reference fixes 0)
                   "masterSeed": int(c.get("MasterSeed", 0))}

    fd = root.get("ParamForField")
    if not isinstance(fd, dict):
        raise ConfigError("ParamForField")
    m = _merged(DEFAULTS["ParamForField"], fd)
    fld = {"ngx": _int(m["NumberOfGridX"]), "ngy": _int(m["NumberOfGridY"]), "dx": _dbl(m["GridSizeOfX"]),
           "dy": _dbl(m["GridSizeOfY"]), "InitTypeE": m["InitializeTypeOfE"], "ampE": _vec(m["AmplitudeOfE"]),
           "InitTypeB": m["InitializeTypeOfB"], "ampB": _vec(m["AmplitudeOfB"]),
           "FilePathBx": m["FilePathOfBx"], "FilePathBy": m["FilePathOfBy"], "FilePathBz": m["FilePathOfBz"],
           "weightOrder": _int(m["WeightingOrder"]), "BorisOrder": _int(m["BorisOrder"]),
           "checkCurDens": _int(m["FlagForCurDens"]), "diff_ngb": _int(m["PtclPosOffset"])}
    fld["ngb"] = int(fld["weightOrder"] / 2)  # src/Init.mm:140 (C integer division)
    out["field"] = fld

    fbc = root.get("BoundaryConditionForField")
    if not isinstance(fbc, list):
        raise ConfigError("BoundaryConditionForField")
    out["fieldBCs"] = []
    for e in fbc:
        if not isinstance(e, dict):
            continue
        m = _merged(DEFAULTS["BoundaryCondition"], e)
        out["fieldBCs"].append({"position": m["RegionName"], "type": m["BCType"], "val": _dbl(m["Value"])})

    parts = root.get("ParamForParticle")
    if not isinstance(parts, list):
        raise ConfigError("ParamForParticle")
    out["particles"] = []
    ngx, ngy = fld["ngx"], fld["ngy"]
    for e in parts:
        if not isinstance(e, dict):
            continue
        m = _merged(DEFAULTS["ParamForParticle"], e)
        if m["pNumSetMethod"] == "InitialParticleNumber":
            pnum = _int(m["pNumValue"])
        elif m["pNumSetMethod"] == "PtclNumPerCell":
            pnum = _int(m["pNumValue"]) * ngx * ngy
        else:
            raise ConfigError("pNumSet failed.")
        pnum &= 0xFFFFFFFF
        if m["WeightSetMethod"] == "WeightValue":
            w = _dbl(m["WeightValue"])
        elif m["WeightSetMethod"] == "InitialNumDens":
            ppc = float(pnum) / float(ngx * ngy)
            w = _dbl(m["WeightValue"]) * fld["dx"] * fld["dy"] / ppc
        else:
            raise ConfigError("WeightSet failed.")
        out["particles"].append({"pName": m["ParticleName"], "pNum": pnum, "q": _dbl(m["Charge"]),
                                 "m": _dbl(m["Mass"]), "w": w, "genType": m["GenerateType"],
                                 "genX": _vec(m["InitialPosX"]), "genY": _vec(m["InitialPosY"]),
                                 "genU": _vec(m["InitialVel"]), "genT": _dbl(m["InitialTemp"]) * EV_TO_K})

    srcs = root.get("SourceForParticle")
    if not isinstance(srcs, list):
        raise ConfigError("SourceForParticle")
    out["sources"] = []
    for e in srcs:
        if not isinstance(e, dict):
            continue
        m = _merged(DEFAULTS["SourceForParticle"], e)
        meth = m["SrcSetMethod"]
        val = _dbl(m.get("SrcValue", 0))
        if meth == "Source[1/cm/s]":
            src = val
        elif meth == "CurrentDensity[A/m2]":
            src = val * JTOSJ * ngy * fld["dy"] / EC
        elif meth == "BoundaryCurrentAtXmin":
            src = 0
        elif meth == "BoundaryCurrentAtXmax":
            src = 1
        elif meth == "BoundaryCurrentAtYmin":
            src = 2
        elif meth == "BoundaryCurrentAtYmax":
            src = 3
        elif meth == "AbsorbedParticleNumber":  # build addition (fluxMaxwellianAtXmin)
            src = 0
        else:
            raise ConfigError("SrcSet failed.")
        out["sources"].append({"pName": m["ParticleName"], "genType": m["GenerateType"], "src": float(src),
                               "genX": _vec(m["GeneratePosX"]), "genY": _vec(m["GeneratePosY"]),
                               "genU": _vec(m["GenerateVel"]), "genT": _dbl(m["GenerateTemp"]) * EV_TO_K,
                               "genU_ele": _vec(m["GenVelForElectron"]),
                               "genT_ele": _dbl(m["GenTempForElectron"]) * EV_TO_K})

    pbc = root.get("BoundaryConditionForParticle")
    if not isinstance(pbc, list):
        raise ConfigError("BoundaryConditionForParticle")
    out["particleBCs"] = []
    for e in pbc:
        if not isinstance(e, dict):
            continue
        out["particleBCs"].append({"position": e.get("RegionName"), "type": e.get("BCType")})
    return out


def field_bc_codes(cfg):
    """Per wall (Xmin, Xmax, Ymin, Ymax): code, value; and cathode position."""
    codes, vals, cathode = [-1] * 4, [0.0] * 4, -1.0
    for bc in cfg["fieldBCs"]:
        if bc["position"] in WALLS:
            w = WALLS.index(bc["position"])
            codes[w] = FIELD_BC.get(bc["type"], -1)
            vals[w] = bc["val"]
        elif bc["position"] == "hollow-cathode":
            cathode = bc["val"]
    return codes, vals, cathode


def particle_bc_codes(cfg):
    codes = [-1] * 4
    for bc in cfg["particleBCs"]:
        if bc["position"] in WALLS:
            codes[WALLS.index(bc["position"])] = PARTICLE_BC.get(bc["type"], -1)
    return codes


def _pad(v, n, fill):
    v = list(v) + [fill] * n
    return v[:n]


def to_struct(cfg, lib_module):
    """Fill an or_config ctypes struct (oracle/lib.py) from a parsed config."""
    C = lib_module.OrConfig()
    f = cfg["field"]
    C.n_species = cfg["flag"]["Particle"]
    C.em_field = cfg["flag"]["EMField"]
    C.mc_collision = cfg["flag"]["MCCollision"]
    t = cfg["time"]
    C.start, C.end, C.dt = t["Start"], t["End"], t["TimeStep"]
    C.log_output, C.particle_output = t["LogOutput"], t["ParticleOutput"]
    C.field_output, C.progress_output = t["FieldOutput"], t["ProgressOutput"]
    C.pnum_max = cfg["comp"]["pNumMax"]
    C.maxiter = cfg["comp"]["maxiter"]
    C.tol = cfg["comp"]["tolerance"]
    C.master_seed = cfg["comp"].get("masterSeed", 0)
    C.ngx, C.ngy, C.ngb, C.dx, C.dy = f["ngx"], f["ngy"], f["ngb"], f["dx"], f["dy"]
    C.ampE[:] = _pad(f["ampE"], 3, 0.0)
    C.ampB[:] = _pad(f["ampB"], 3, 0.0)
    C.initE_uniform = int(f["InitTypeE"] == "Uniform")
    C.initB_uniform = int(f["InitTypeB"] == "Uniform")
    C.weight_order, C.boris_order, C.cur_dens = f["weightOrder"], f["BorisOrder"], f["checkCurDens"]
    codes, vals, cathode = field_bc_codes(cfg)
    C.fbc[:] = codes
    C.fbc_val[:] = vals
    C.cathode_pos = cathode
    C.pbc[:] = particle_bc_codes(cfg)
    for s, p in enumerate(cfg["particles"][: lib_module.OR_MAX_SPECIES]):
        sp = C.sp[s]
        sp.name = p["pName"].encode()[:31]
        sp.pnum = p["pNum"]
        sp.q, sp.m, sp.w = p["q"], p["m"], p["w"]
        sp.gen_type = LOAD_GEN.get(p["genType"], -1)
        sp.genX[:] = _pad(p["genX"], 2, -1.0)
        sp.genY[:] = _pad(p["genY"], 2, -1.0)
        sp.genU[:] = _pad(p["genU"], 3, 0.0)
        sp.genT = p["genT"]
    C.n_sources = min(len(cfg["sources"]), lib_module.OR_MAX_SOURCES)
    for i, s in enumerate(cfg["sources"][: lib_module.OR_MAX_SOURCES]):
        so = C.src[i]
        so.pname = s["pName"].encode()[:31]
        so.gen_type = SOURCE_GEN.get(s["genType"], -1)
        so.src = s["src"]
        so.genX[:] = _pad(s["genX"], 2, -1.0)
        so.genY[:] = _pad(s["genY"], 2, -1.0)
        so.genU[:] = _pad(s["genU"], 3, 0.0)
        so.genU_ele[:] = _pad(s["genU_ele"], 3, 0.0)
        so.genT, so.genT_ele = s["genT"], s["genT_ele"]
    return C
