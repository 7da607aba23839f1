"""ctypes bindings of the CPU oracle (test infrastructure only).

Loads oracle/liboracle.so (built by oracle/Makefile). Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import config as cfgmod

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
OR_MAX_SPECIES = 4
OR_MAX_SOURCES = 4


class OrSpecies(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("pnum", C.c_uint), ("q", C.c_double), ("m", C.c_double),
                ("w", C.c_double), ("gen_type", C.c_int), ("genX", C.c_double * 2), ("genY", C.c_double * 2),
                ("genU", C.c_double * 3), ("genT", C.c_double)]


class OrSource(C.Structure):
    _fields_ = [("pname", C.c_char * 32), ("gen_type", C.c_int), ("src", C.c_double), ("genX", C.c_double * 2),
                ("genY", C.c_double * 2), ("genU", C.c_double * 3), ("genU_ele", C.c_double * 3),
                ("genT", C.c_double), ("genT_ele", C.c_double)]


class OrConfig(C.Structure):
    _fields_ = [("n_species", C.c_int), ("em_field", C.c_int), ("mc_collision", C.c_int), ("start", C.c_int),
                ("end", C.c_int), ("dt", C.c_double), ("log_output", C.c_int), ("particle_output", C.c_int),
                ("field_output", C.c_int), ("progress_output", C.c_int), ("pnum_max", C.c_uint),
                ("maxiter", C.c_int), ("tol", C.c_double), ("ngx", C.c_int), ("ngy", C.c_int), ("ngb", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("ampE", C.c_double * 3), ("ampB", C.c_double * 3),
                ("initE_uniform", C.c_int), ("initB_uniform", C.c_int), ("weight_order", C.c_int),
                ("boris_order", C.c_int), ("cur_dens", C.c_int), ("fbc", C.c_int * 4), ("fbc_val", C.c_double * 4),
                ("cathode_pos", C.c_double), ("pbc", C.c_int * 4), ("sp", OrSpecies * OR_MAX_SPECIES),
                ("n_sources", C.c_int), ("src", OrSource * OR_MAX_SOURCES), ("master_seed", C.c_uint64)]


class OrSolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("error", C.c_double), ("mean_cathode", C.c_double),
                ("energy", C.c_double), ("joule", C.c_double), ("probe", C.c_double * 3)]


class OrFlowStats(C.Structure):
    _fields_ = [("pinum", C.c_int * 4), ("pulled", C.c_int), ("pnum", C.c_uint), ("ke", C.c_double)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, i, d, u = C.c_void_p, C.c_int, C.c_double, C.c_uint
        dp, fp, ip = C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int)
        sig = {
            "or_sim_create": (vp, [C.POINTER(OrConfig), i]),
            "or_sim_free": (None, [vp]),
            "or_sim_load_initial": (i, [vp]),
            "or_sim_reset_charge": (None, [vp]),
            "or_sim_deposit": (None, [vp, i]),
            "or_sim_solve_poisson": (None, [vp, d, d, C.POINTER(OrSolveStats)]),
            "or_sim_push": (None, [vp, i, d]),
            "or_sim_reduce": (None, [vp, i, i, C.POINTER(OrFlowStats)]),
            "or_sim_ionize": (i, [vp, d, ip]),
            "or_sim_hollow_cathode": (i, [vp, d, ip]),
            "or_sim_reflux": (i, [vp, d, ip]),
            "or_sim_cycle": (i, [vp, i, i, C.POINTER(OrSolveStats), C.POINTER(OrFlowStats)]),
            "or_sim_pnum": (u, [vp, i]),
            "or_sim_set_pnum": (None, [vp, i, u]),
            "or_sim_get_particles": (None, [vp, i, dp, dp, dp, dp, dp, ip]),
            "or_sim_set_particles": (None, [vp, i, u, dp, dp, dp, dp, dp, ip]),
            "or_sim_get_particles_f32": (None, [vp, i, fp, fp, fp, fp, fp, ip]),
            "or_sim_set_particles_f32": (None, [vp, i, u, fp, fp, fp, fp, fp, ip]),
            "or_sim_get_field": (None, [vp, i, dp]),
            "or_sim_set_field": (None, [vp, i, dp]),
            "or_sim_species_consts": (None, [vp, i, fp, fp, fp, fp, fp]),
            "or_sim_poisson_size": (i, [vp]),
            "or_sim_poisson_residual": (d, [vp, dp]),
            "or_sim_get_poisson_solution": (None, [vp, dp]),
            "or_sim_moments": (None, [vp, i, i, C.c_void_p]),
            "or_darwin": (None, [i, i, i, i, i, C.c_float, C.c_float, d] + [C.c_void_p] * 10),
            "or_det_deposit_rho": (None, [i, i, i, i, i, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p]),
            "or_det_deposit_j": (None, [i, i, i, i, i] + [C.c_void_p] * 8),
            "or_shape_build": (None, [i, C.c_float, fp]),
            "or_shape_ref_f32": (None, [i, C.c_float, fp]),
            "or_shape_ref_f64": (None, [i, d, dp]),
            "or_pcg_stream": (None, [C.c_uint64, C.c_uint64, i, i, C.POINTER(C.c_uint32)]),
            "or_minstd_uniform": (d, [i, dp]),
            "or_splitmix64_stream": (None, [C.c_uint64, i, C.POINTER(C.c_uint64)]),
            "or_pcg32_raw": (None, [C.c_uint64, C.c_uint64, i, C.POINTER(C.c_uint32)]),
            "or_num_threads": (i, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


FIELD_IDS = {"rho": 0, "Ex": 1, "Ey": 2, "Bz": 3, "jx": 4, "jy": 5, "phi": 6}


class OracleSim:
    """One simulation (Particle + EMField + Collision objects) on the CPU."""

    def __init__(self, cfg, real64=False):
        if not isinstance(cfg, dict) or "field" not in cfg:
            cfg = cfgmod.parse(cfg)
        self.cfg = cfg
        import sys
        self.struct = cfgmod.to_struct(cfg, sys.modules[__name__])
        self.h = lib().or_sim_create(C.byref(self.struct), int(real64))
        f = cfg["field"]
        self.ngx, self.ngy, self.ngb = f["ngx"], f["ngy"], f["ngb"]
        self.nx, self.ny = self.ngx + 2 * self.ngb, self.ngy + 2 * self.ngb
        self.ns = cfg["flag"]["Particle"]
        self.dt = cfg["time"]["TimeStep"]

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().or_sim_free(h)
            self.h = None

    def shape(self, which):
        nx, ny = self.nx, self.ny
        return {"rho": (ny + 1, nx + 1), "Ex": (ny + 1, nx + 2), "Ey": (ny + 2, nx + 1), "Bz": (ny + 2, nx + 2),
                "jx": (ny + 1, nx + 2), "jy": (ny + 2, nx + 1), "phi": (ny + 3, nx + 3)}[which]

    def load_initial(self):
        rc = lib().or_sim_load_initial(self.h)
        if rc != 0:
            raise RuntimeError(f"oracle load_initial rc={rc}")

    def reset_charge(self):
        lib().or_sim_reset_charge(self.h)

    def deposit(self, s):
        lib().or_sim_deposit(self.h, s)

    def solve_poisson(self, dt=None, tol=-1.0):
        st = OrSolveStats()
        lib().or_sim_solve_poisson(self.h, self.dt if dt is None else dt, tol, C.byref(st))
        return st

    def push(self, s, dt=None):
        lib().or_sim_push(self.h, s, self.dt if dt is None else dt)

    def reduce(self, s, faithful=True):
        fs = OrFlowStats()
        lib().or_sim_reduce(self.h, s, int(faithful), C.byref(fs))
        return fs

    def ionize(self, dt=None):
        n = C.c_int(0)
        rc = lib().or_sim_ionize(self.h, self.dt if dt is None else dt, C.byref(n))
        return rc, n.value

    def hollow_cathode(self, dt=None):
        n = C.c_int(0)
        rc = lib().or_sim_hollow_cathode(self.h, self.dt if dt is None else dt, C.byref(n))
        return rc, n.value

    def reflux(self, dt=None):
        n = C.c_int(0)
        rc = lib().or_sim_reflux(self.h, self.dt if dt is None else dt, C.byref(n))
        return rc, n.value

    def cycle(self, cycle=0, faithful=True):
        st = OrSolveStats()
        fs = (OrFlowStats * max(self.ns, 1))()
        rc = lib().or_sim_cycle(self.h, cycle, int(faithful), C.byref(st), fs)
        if rc != 0:
            raise RuntimeError(f"oracle cycle rc={rc}")
        return st, list(fs)

    def pnum(self, s):
        return lib().or_sim_pnum(self.h, s)

    def particles(self, s, f32=False):
        n = self.pnum(s)
        if f32:
            arrs = [np.empty(n, np.float32) for _ in range(5)]
            fl = np.empty(n, np.int32)
            lib().or_sim_get_particles_f32(self.h, s, *[_p(a, C.c_float) for a in arrs], _p(fl, C.c_int))
        else:
            arrs = [np.empty(n, np.float64) for _ in range(5)]
            fl = np.empty(n, np.int32)
            lib().or_sim_get_particles(self.h, s, *[_p(a, C.c_double) for a in arrs], _p(fl, C.c_int))
        return dict(zip(("x", "y", "vx", "vy", "vz"), arrs), piflag=fl)

    def set_particles(self, s, x, y, vx, vy, vz, piflag=None, f32=False):
        n = len(x)
        if f32:
            arrs = [np.ascontiguousarray(a, np.float32) for a in (x, y, vx, vy, vz)]
            ct, fn = C.c_float, lib().or_sim_set_particles_f32
        else:
            arrs = [np.ascontiguousarray(a, np.float64) for a in (x, y, vx, vy, vz)]
            ct, fn = C.c_double, lib().or_sim_set_particles
        fl = np.zeros(n, np.int32) if piflag is None else np.ascontiguousarray(piflag, np.int32)
        fn(self.h, s, n, *[_p(a, ct) for a in arrs], _p(fl, C.c_int))

    def field(self, which):
        shp = self.shape(which)
        out = np.empty(shp, np.float64)
        lib().or_sim_get_field(self.h, FIELD_IDS[which], _p(out, C.c_double))
        return out

    def set_field(self, which, arr):
        a = np.ascontiguousarray(arr, np.float64).reshape(self.shape(which))
        lib().or_sim_set_field(self.h, FIELD_IDS[which], _p(a, C.c_double))

    def species_consts(self, s):
        v = [C.c_float() for _ in range(5)]
        lib().or_sim_species_consts(self.h, s, *[C.byref(x) for x in v])
        return dict(zip(("constE", "constB", "constX", "constY", "scale"), [x.value for x in v]))

    def poisson_size(self):
        return lib().or_sim_poisson_size(self.h)

    def poisson_residual(self, sol):
        a = np.ascontiguousarray(sol, np.float64)
        return lib().or_sim_poisson_residual(self.h, _p(a, C.c_double))

    def poisson_solution(self):
        out = np.empty(self.poisson_size(), np.float64)
        lib().or_sim_get_poisson_solution(self.h, _p(out, C.c_double))
        return out

    MOMENTS = ("n", "ux", "uy", "uz", "Pxx", "Pxy", "Pxz", "Pyy", "Pyz", "Pzz")

    def moments(self, sp, build=True):
        """Velocity moments of species sp (src/Moment.mm) as (ny+1, nx+1) arrays;
        build=True uses the GPU build's weights and FP64 sums."""
        shape = self.shape("rho")
        out = np.empty((10,) + shape, np.float32)
        lib().or_sim_moments(self.h, sp, 1 if build else 0, out.ctypes.data)
        return dict(zip(self.MOMENTS, out))


class Darwin:
    """The oracle's Darwin solve (src/EMField.mm:1138-1361) with its A_last state."""

    def __init__(self, ngx, ngy, ngb, perx, pery, dx, dy):
        self.a = (ngx, ngy, ngb, int(perx), int(pery), float(dx), float(dy))
        self.nx, self.ny = ngx + 2 * ngb, ngy + 2 * ngb
        self.shape = (ngy - int(pery) + 1, ngx - int(perx) + 1)
        self.lastAx = np.zeros(self.shape)
        self.lastAy = np.zeros(self.shape)

    def solve(self, jx, jy, dt):
        jx = np.ascontiguousarray(jx, np.float32)
        jy = np.ascontiguousarray(jy, np.float32)
        psi, ax, ay = (np.zeros(self.shape) for _ in range(3))
        nx, ny = self.nx, self.ny
        dex = np.zeros((ny + 1, nx + 2), np.float32)
        dey = np.zeros((ny + 2, nx + 1), np.float32)
        dbz = np.zeros((ny + 2, nx + 2), np.float32)
        lib().or_darwin(*self.a, dt, jx.ctypes.data, jy.ctypes.data, self.lastAx.ctypes.data,
                        self.lastAy.ctypes.data, psi.ctypes.data, ax.ctypes.data, ay.ctypes.data, dex.ctypes.data,
                        dey.ctypes.data, dbz.ctypes.data)
        return {"psi": psi, "Ax": ax, "Ay": ay, "delEx": dex, "delEy": dey, "delBz": dbz}


def det_deposit_rho(order, ngx, ngy, ngb, ix, iy, ox, oy):
    nx, ny = ngx + 2 * ngb, ngy + 2 * ngb
    acc = np.zeros((ny + 1) * (nx + 1), np.int64)
    ix, iy = np.ascontiguousarray(ix, np.int32), np.ascontiguousarray(iy, np.int32)
    ox, oy = np.ascontiguousarray(ox, np.float32), np.ascontiguousarray(oy, np.float32)
    lib().or_det_deposit_rho(order, ngx, ngy, ngb, len(ix), ix.ctypes.data, iy.ctypes.data, ox.ctypes.data,
                             oy.ctypes.data, acc.ctypes.data)
    return acc.reshape(ny + 1, nx + 1)


def det_deposit_j(order, ngx, ngy, ngb, ix, iy, ox, oy, vx, vy):
    nx, ny = ngx + 2 * ngb, ngy + 2 * ngb
    accx = np.zeros((ny + 1) * (nx + 2), np.int64)
    accy = np.zeros((ny + 2) * (nx + 1), np.int64)
    a = [np.ascontiguousarray(v, t) for v, t in ((ix, np.int32), (iy, np.int32), (ox, np.float32),
                                                 (oy, np.float32), (vx, np.float32), (vy, np.float32))]
    lib().or_det_deposit_j(order, ngx, ngy, ngb, len(a[0]), *[v.ctypes.data for v in a], accx.ctypes.data,
                           accy.ctypes.data)
    return accx.reshape(ny + 1, nx + 2), accy.reshape(ny + 2, nx + 1)


def shape_build(order, h):
    w = np.zeros(6, np.float32)
    lib().or_shape_build(order, C.c_float(h), _p(w, C.c_float))
    return w[: order + 1]


def shape_ref(order, h, f64=False):
    if f64:
        w = np.zeros(6, np.float64)
        lib().or_shape_ref_f64(order, float(h), _p(w, C.c_double))
    else:
        w = np.zeros(6, np.float32)
        lib().or_shape_ref_f32(order, C.c_float(h), _p(w, C.c_float))
    return w[: order + 1]


def pcg_stream(master_seed, first_slot, nslots, ndraws):
    out = np.zeros((nslots, ndraws), np.uint32)
    lib().or_pcg_stream(master_seed, first_slot, nslots, ndraws, _p(out, C.c_uint32))
    return out


def splitmix64_stream(seed, n):
    out = np.zeros(n, np.uint64)
    lib().or_splitmix64_stream(seed, n, _p(out, C.c_uint64))
    return out


def pcg32_raw(state, inc, n):
    out = np.zeros(n, np.uint32)
    lib().or_pcg32_raw(state, inc, n, _p(out, C.c_uint32))
    return out


def minstd_uniform(count):
    out = np.zeros(count, np.float64)
    lib().or_minstd_uniform(count, _p(out, C.c_double))
    return out


def num_threads():
    return lib().or_num_threads()


def fmt_sci(v):
    """src/XmlLogger.h:89-93: float-rounded, std::scientific, 6 digits."""
    return f"{float(np.float32(v)):.6e}"


def fmt_time(t):
    """std::ostream default formatting of a double (precision 6, %g)."""
    return f"{t:.6g}"
