"""ctypes bindings of libgample_b200.so (the C ABI in include/gample_gpu.h).

This is the binding a Python caller of the reference-facing C ABI uses; the
tests and bench.py drive the product through it. Loading fails loudly when the
compiled library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgample_b200.so")

GP_OK = 0
GP_ERR = {1: "argument", 2: "config", 3: "cuda", 4: "capacity", 5: "internal"}
FIELDS = {"rho": 0, "Ex": 1, "Ey": 2, "Bz": 3, "jx": 4, "jy": 5, "phi": 6, "sol": 7, "delEx": 8, "delEy": 9,
          "delBz": 10, "psi": 11, "Ax": 12, "Ay": 13}
PHASES = ("deposit", "solve", "push", "reduce", "sources", "sort")


class GpParticleState(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("vx", C.c_float), ("vy", C.c_float), ("vz", C.c_float),
                ("piflag", C.c_int32)]


PARTICLE_DTYPE = np.dtype([("x", np.float32), ("y", np.float32), ("vx", np.float32), ("vy", np.float32),
                           ("vz", np.float32), ("piflag", np.int32)])


class GpSolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("error", C.c_double), ("mean_cathode", C.c_double),
                ("electric_energy", C.c_double), ("electric_energy_increment", C.c_double),
                ("joule_heating", C.c_double), ("probe", C.c_double * 3), ("field_energy_cgs", C.c_double)]


class GpFlowStats(C.Structure):
    _fields_ = [("particle_number", C.c_uint32), ("pulled", C.c_uint32), ("pinum", C.c_int32 * 4),
                ("invalid", C.c_uint32), ("kinetic_energy", C.c_double),
                ("kinetic_energy_increment", C.c_double)]


class GampleError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"gample_b200 error {status} ({GP_ERR.get(status, '?')}): {msg}")
        self.status = status


_lib = None

EXPORTS = {
    # name: (restype, argtypes)
    "gp_init_parse_file": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "gp_init_parse_json": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "gp_init_dump": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "gp_init_free": (None, [C.c_void_p]),
    "gp_sim_create": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]),
    "gp_sim_free": (None, [C.c_void_p]),
    "gp_sim_initialize": (C.c_int, [C.c_void_p]),
    "gp_sim_run": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_sim_cycle_number": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "gp_sim_last_solve": (C.c_int, [C.c_void_p, C.POINTER(GpSolveStats)]),
    "gp_sim_last_flow": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(GpFlowStats)]),
    "gp_sim_synchronize": (C.c_int, [C.c_void_p]),
    "gp_sim_time_cycles": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float)]),
    "gp_sim_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_sim_phase_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "gp_field_dims": (C.c_int, [C.c_void_p] + [C.POINTER(C.c_int)] * 5),
    "gp_field_reset_charge": (C.c_int, [C.c_void_p]),
    "gp_field_solve_poisson": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(GpSolveStats)]),
    "gp_field_solve_darwin": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]),
    "gp_field_download": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    "gp_field_upload": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    "gp_field_set_solver": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "gp_particle_update": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int]),
    "gp_particle_reduce": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(GpFlowStats)]),
    "gp_particle_integrate_charge": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_particle_count": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_uint32)]),
    "gp_particle_push_stats": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_uint32)]),
    "gp_particle_sort": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "gp_particle_set_push_variant": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "gp_particle_download": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]),
    "gp_particle_upload": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_uint32]),
    "gp_particle_download_raw": (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 6 +
                                 [C.c_uint32, C.POINTER(C.c_uint32)]),
    "gp_collision_artificial_ionization": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_int)]),
    "gp_collision_hollow_cathode": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_int)]),
    "gp_collision_flux_reinjection": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_int)]),
    "gp_moments_integrate": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_moments_download": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    "gp_sim_output_field": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_sim_output_moments": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "gp_sim_save_progress": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_sim_load_progress": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_field_learned": (C.c_int, [C.c_void_p, C.c_int, C.c_float, C.c_uint64]),
    "gp_field_learned_stats": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gp_field_learned_bank": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_field_learned_train": (C.c_int, [C.c_void_p, C.c_int, C.c_float, C.c_uint64, C.c_void_p]),
    "gp_sim_reload": (C.c_int, [C.c_void_p, C.c_uint64]),
    "gp_ensemble_create": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "gp_ensemble_free": (None, [C.c_void_p]),
    "gp_ensemble_initialize": (C.c_int, [C.c_void_p]),
    "gp_ensemble_run": (C.c_int, [C.c_void_p, C.c_int]),
    "gp_ensemble_time_cycles": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float)]),
    "gp_ensemble_member": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "gp_nn_create": (C.c_int, [C.c_int, C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
    "gp_nn_free": (None, [C.c_void_p]),
    "gp_nn_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "gp_nn_loss_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_float)]),
    "gp_nn_train_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.POINTER(C.c_float)]),
    "gp_nn_layer_info": (C.c_int, [C.c_void_p, C.c_int] + [C.POINTER(C.c_int)] * 3),
    "gp_nn_param": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_size_t, C.c_int]),
    "gp_deposit_charge_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_uint32, C.c_float,
                                            C.c_void_p, C.c_void_p]),
    "gp_last_error": (C.c_char_p, []),
    "gp_version": (C.c_char_p, []),
    "gp_device_count": (C.c_int, []),
    "gp_kernel_launches": (C.c_ulonglong, []),
    "gp_release_cached_memory": (C.c_int, []),
}


def lib():
    """Load the compiled library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C gample_b200` "
                               "(the CUDA path has no fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in EXPORTS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != GP_OK:
        raise GampleError(status, lib().gp_last_error().decode(errors="replace"))


class Init:
    """Parsed condition file (-[Init parseInputFile:])."""

    def __init__(self, source):
        h = C.c_void_p()
        if isinstance(source, dict):
            check(lib().gp_init_parse_json(json.dumps(source).encode(), C.byref(h)))
        elif isinstance(source, str) and source.lstrip().startswith("{"):
            check(lib().gp_init_parse_json(source.encode(), C.byref(h)))
        else:
            check(lib().gp_init_parse_file(os.fspath(source).encode(), C.byref(h)))
        self.h = h

    def dump(self):
        n = C.c_size_t()
        check(lib().gp_init_dump(self.h, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        check(lib().gp_init_dump(self.h, buf, n.value, C.byref(n)))
        return json.loads(buf.value.decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().gp_init_free(self.h)
            self.h = None


class Sim:
    """One run: Particle objects, EMField, Collision and (optionally) logger."""

    def __init__(self, cond, log_name=None, reference_order=False):
        self.init = cond if isinstance(cond, Init) else Init(cond)
        h = C.c_void_p()
        check(lib().gp_sim_create(self.init.h, log_name.encode() if log_name else None,
                                  1 if reference_order else 0, C.byref(h)))
        self.h = h
        d = [C.c_int() for _ in range(5)]
        check(lib().gp_field_dims(self.h, *[C.byref(x) for x in d]))
        self.ngx, self.ngy, self.ngb, self.nkx, self.nky = [x.value for x in d]
        self.nx, self.ny = self.ngx + 2 * self.ngb, self.ngy + 2 * self.ngb

    def close(self):
        if getattr(self, "h", None):
            lib().gp_sim_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # -- main loop
    def initialize(self):
        check(lib().gp_sim_initialize(self.h))

    def run(self, n):
        check(lib().gp_sim_run(self.h, n))

    def time_cycles(self, n):
        ms = C.c_float()
        check(lib().gp_sim_time_cycles(self.h, n, C.byref(ms)))
        return ms.value

    def synchronize(self):
        check(lib().gp_sim_synchronize(self.h))

    def set_profiling(self, on=True):
        check(lib().gp_sim_set_profiling(self.h, int(on)))

    def phase_times(self):
        out = (C.c_double * 6)()
        check(lib().gp_sim_phase_times(self.h, out))
        return dict(zip(PHASES, list(out)))

    def cycle_number(self):
        c, t = C.c_int(), C.c_double()
        check(lib().gp_sim_cycle_number(self.h, C.byref(c), C.byref(t)))
        return c.value, t.value

    def last_solve(self):
        st = GpSolveStats()
        check(lib().gp_sim_last_solve(self.h, C.byref(st)))
        return st

    def last_flow(self, s):
        fs = GpFlowStats()
        check(lib().gp_sim_last_flow(self.h, s, C.byref(fs)))
        return fs

    # -- EMField
    def shape(self, which):
        nx, ny = self.nx, self.ny
        return {"rho": (ny + 1, nx + 1), "Ex": (ny + 1, nx + 2), "Ey": (ny + 2, nx + 1), "Bz": (ny + 2, nx + 2),
                "jx": (ny + 1, nx + 2), "jy": (ny + 2, nx + 1), "phi": (ny + 3, nx + 3),
                "sol": (self.nky + 1, self.nkx + 1), "delEx": (ny + 1, nx + 2), "delEy": (ny + 2, nx + 1),
                "delBz": (ny + 2, nx + 2), "psi": self.darwin_shape(), "Ax": self.darwin_shape(),
                "Ay": self.darwin_shape()}[which]

    def darwin_shape(self):
        """(nky_vec+1, nkx_vec+1): ngx (ngy) nodes plus one, minus one when periodic."""
        types = {b["position"]: b["type"] for b in self.init.dump().get("fieldBCs", [])}
        px = types.get("Xmin") == "periodic"
        py = types.get("Ymin") == "periodic"
        return (self.ngy - (1 if py else 0) + 1, self.ngx - (1 if px else 0) + 1)

    LEARNED_KEYS = ("loss", "iters_learned", "iters_plain", "ms_learned", "ms_plain", "ms_net", "rel0_learned",
                    "rel0_plain", "trained_steps")

    def reload(self, seed):
        """The initial load again from master seed `seed` (initialize() follows)."""
        check(lib().gp_sim_reload(self.h, seed))

    def learned_bank(self, capacity):
        check(lib().gp_field_learned_bank(self.h, capacity))

    def learned_train(self, steps, lr=1e-3, seed=0):
        out = (C.c_double * 3)()
        check(lib().gp_field_learned_train(self.h, steps, lr, seed, out))
        return {"loss_first": out[0], "loss_last": out[1], "samples": int(out[2])}

    def set_learned(self, mode, lr=1e-3, seed=0):
        check(lib().gp_field_learned(self.h, mode, lr, seed))

    def learned_stats(self):
        out = (C.c_double * 9)()
        check(lib().gp_field_learned_stats(self.h, out))
        return dict(zip(self.LEARNED_KEYS, list(out)))

    def solve_darwin(self, dt):
        it = (C.c_int * 3)()
        er = (C.c_double * 3)()
        check(lib().gp_field_solve_darwin(self.h, dt, it, er))
        return list(it), list(er)

    def field(self, which):
        dt = np.float64 if which in ("phi", "sol", "psi", "Ax", "Ay") else np.float32
        out = np.empty(self.shape(which), dt)
        check(lib().gp_field_download(self.h, FIELDS[which], out.ctypes.data, out.nbytes))
        return out

    def set_field(self, which, arr):
        dt = np.float64 if which in ("phi", "sol", "psi", "Ax", "Ay") else np.float32
        a = np.ascontiguousarray(arr, dt).reshape(self.shape(which))
        check(lib().gp_field_upload(self.h, FIELDS[which], a.ctypes.data, a.nbytes))

    def reset_charge(self):
        check(lib().gp_field_reset_charge(self.h))

    def solve_poisson(self, dt=0.0):
        st = GpSolveStats()
        check(lib().gp_field_solve_poisson(self.h, dt, C.byref(st)))
        return st

    def set_solver(self, tol, maxiter=1000):
        check(lib().gp_field_set_solver(self.h, tol, maxiter))

    # -- Particle
    def update(self, s, dt, fused_deposit=False):
        check(lib().gp_particle_update(self.h, s, dt, int(fused_deposit)))

    def reduce(self, s):
        fs = GpFlowStats()
        check(lib().gp_particle_reduce(self.h, s, C.byref(fs)))
        return fs

    def integrate_charge(self, s):
        check(lib().gp_particle_integrate_charge(self.h, s))

    def count(self, s):
        n = C.c_uint32()
        check(lib().gp_particle_count(self.h, s, C.byref(n)))
        return n.value

    def sort(self, s, path=0):
        """Sort species s by cell now (path 0 automatic, 1 block-local
        re-sort, 2 staged record scatter)."""
        check(lib().gp_particle_sort(self.h, s, path))

    def set_push_variant(self, s, particles, tables=True):
        """Fix the push's particles per chunk (2048 or 1024) and gather tables
        (order 3), or particles=0 for the autotuner."""
        check(lib().gp_particle_set_push_variant(self.h, s, particles, 1 if tables else 0))

    def push_stats(self, s):
        """(particles pushed without a window, chunks staged by bulk tensor
        copies, staging waits that timed out, chunks gathering through the
        per-cell tables, chunks depositing into lane-private windows,
        particles per chunk, gather tables allowed) of the last push."""
        out = (C.c_uint32 * 7)()
        check(lib().gp_particle_push_stats(self.h, s, out))
        return tuple(out)

    def particles(self, s):
        n = self.count(s)
        out = np.empty(n, PARTICLE_DTYPE)
        got = C.c_uint32()
        check(lib().gp_particle_download(self.h, s, out.ctypes.data, n, C.byref(got)))
        return out[: got.value]

    def set_particles(self, s, arr):
        a = np.ascontiguousarray(arr, PARTICLE_DTYPE)
        check(lib().gp_particle_upload(self.h, s, a.ctypes.data, len(a)))

    MOMENTS = ("n", "ux", "uy", "uz", "Pxx", "Pxy", "Pxz", "Pyy", "Pyz", "Pzz")

    def moments(self, s):
        """Velocity moments of species s as a dict of (ny+1, nx+1) arrays."""
        check(lib().gp_moments_integrate(self.h, s))
        out = {}
        for i, name in enumerate(self.MOMENTS):
            a = np.empty(self.shape("rho"), np.float32)
            check(lib().gp_moments_download(self.h, i, a.ctypes.data, a.nbytes))
            out[name] = a
        return out

    def particles_raw(self, s):
        n = self.count(s)
        cell = np.empty(n, np.int32)
        fl = [np.empty(n, np.float32) for _ in range(5)]
        got = C.c_uint32()
        check(lib().gp_particle_download_raw(self.h, s, cell.ctypes.data, *[a.ctypes.data for a in fl], n,
                                             C.byref(got)))
        return dict(cell=cell, ox=fl[0], oy=fl[1], vx=fl[2], vy=fl[3], vz=fl[4])

    # -- Collision
    def artificial_ionization(self, dt):
        n = C.c_int()
        check(lib().gp_collision_artificial_ionization(self.h, dt, C.byref(n)))
        return n.value

    def hollow_cathode(self, dt):
        n = C.c_int()
        check(lib().gp_collision_hollow_cathode(self.h, dt, C.byref(n)))
        return n.value

    def flux_reinjection(self, dt):
        n = C.c_int()
        check(lib().gp_collision_flux_reinjection(self.h, dt, C.byref(n)))
        return n.value


def device_count():
    return lib().gp_device_count()


def kernel_launches():
    return int(lib().gp_kernel_launches())


def release_cached_memory():
    """Return the device memory cached from closed simulations to the driver."""
    check(lib().gp_release_cached_memory())


class Net:
    """The learned warm-start network on the GPU (gp_nn_*)."""

    def __init__(self, h, w, seed=0):
        self.h, self.w = h, w
        p = C.c_void_p()
        check(lib().gp_nn_create(h, w, seed, C.byref(p)))
        self.p = p
        self.layers = []
        for i in range(12):
            a, b, c = C.c_int(), C.c_int(), C.c_int()
            check(lib().gp_nn_layer_info(self.p, i, C.byref(a), C.byref(b), C.byref(c)))
            self.layers.append((a.value, b.value, c.value))

    def close(self):
        if getattr(self, "p", None):
            lib().gp_nn_free(self.p)
            self.p = None

    def __del__(self):
        self.close()

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        out = np.empty((self.h, self.w), np.float32)
        check(lib().gp_nn_forward(self.p, x.ctypes.data, out.ctypes.data))
        return out

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        loss = C.c_float()
        check(lib().gp_nn_loss_grad(self.p, x.ctypes.data, t.ctypes.data, C.byref(loss)))
        return loss.value

    def train_step(self, x, t, lr):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        loss = C.c_float()
        check(lib().gp_nn_train_step(self.p, x.ctypes.data, t.ctypes.data, lr, C.byref(loss)))
        return loss.value

    def param(self, layer, which):
        cin, cout, kpad = self.layers[layer]
        n = cout * kpad if which in (0, 2) else cout
        a = np.empty(n, np.float32)
        check(lib().gp_nn_param(self.p, layer, which, a.ctypes.data, n, 0))
        return a.reshape(cout, kpad) if which in (0, 2) else a

    def set_param(self, layer, which, a):
        a = np.ascontiguousarray(a, np.float32).ravel()
        check(lib().gp_nn_param(self.p, layer, which, a.ctypes.data, a.size, 1))


class Ensemble:
    """Independent runs advanced together (gp_ensemble_*); member(i) gives a Sim view."""

    def __init__(self, conds, threads=8):
        self.inits = [c if isinstance(c, Init) else Init(c) for c in conds]
        arr = (C.c_void_p * len(self.inits))(*[i.h.value if isinstance(i.h, C.c_void_p) else i.h
                                               for i in self.inits])
        p = C.c_void_p()
        check(lib().gp_ensemble_create(arr, len(self.inits), threads, C.byref(p)))
        self.p = p
        self.members = []
        for k in range(len(self.inits)):
            h = C.c_void_p()
            check(lib().gp_ensemble_member(self.p, k, C.byref(h)))
            self.members.append(SimView(self.inits[k], h))

    def initialize(self):
        check(lib().gp_ensemble_initialize(self.p))

    def run(self, n):
        check(lib().gp_ensemble_run(self.p, n))

    def time_cycles(self, n):
        """run(n) timed on the device (ms, CUDA events on the member streams)."""
        ms = C.c_float()
        check(lib().gp_ensemble_time_cycles(self.p, n, C.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "p", None):
            for m in self.members:
                m.h = None
            lib().gp_ensemble_free(self.p)
            self.p = None

    def __del__(self):
        self.close()


class SimView(Sim):
    """A member of an Ensemble (not owned: freeing is the ensemble's)."""

    def __init__(self, init, handle):
        self.init = init
        self.h = handle
        d = [C.c_int() for _ in range(5)]
        check(lib().gp_field_dims(self.h, *[C.byref(x) for x in d]))
        self.ngx, self.ngy, self.ngb, self.nkx, self.nky = [x.value for x in d]
        self.nx, self.ny = self.ngx + 2 * self.ngb, self.ngy + 2 * self.ngb

    def close(self):
        self.h = None
