#!/usr/bin/env python
"""Particle-pushes/s of the 512x512 3rd-order electrostatic PIC step.

Workload (one "step" = one cycle of the reference's time loop: deposit,
Poisson solve to 1e-8 relative residual, gather + Boris push + absorbing
walls, compaction, density-restoring re-injection):
  512 x 512 grid, 3rd-order B-spline weighting, x Dirichlet (phi = 0) with
  absorbing particles, y periodic; electrons + Xe+ (m_i = 1836 * 131.29 m_e),
  256 particles/cell/species (67.1 M each, 134 M total), Maxwellian loads
  (Te = 10 eV, Ti = 0.1 eV), n = 5e10 cm^-3, dx = 0.5 Debye length,
  Bz = 0.02 T, dt * w_pe = 0.05, flux-Maxwellian re-injection at x = 0 of
  every absorbed particle. Seeded synthetic data (the reference's
  splitmix64/PCG32 loader, master seed 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0). --impl reference times the reference's CPU
algorithm (the C++ oracle restatement, OpenMP on all host cores) on a
bounded sample of the same workload.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

EC = 4.803204197e-10
ME = 9.10938188e-28
KB = 1.3806503e-16
EV_K = 11604.0
BYTES_PER_PUSH = 48  # read + write of cell, ox, oy, vx, vy, vz (6 x 4 B)
METRIC = "particle-pushes/s incl. field solve"


def workload(ppc=256, ngx=512, ngy=512, steps=1000, log_output=0):
    n = 5e10
    te_erg = 10.0 * 1.6021764262e-12
    lam_d = math.sqrt(te_erg / (4 * math.pi * n * EC ** 2))
    wpe = math.sqrt(4 * math.pi * n * EC ** 2 / ME)
    dx = 0.5 * lam_d
    dt = 0.05 / wpe
    npart = ppc * ngx * ngy
    src = [{"ParticleName": name, "GenerateType": "fluxMaxwellianAtXmin", "SrcSetMethod": "AbsorbedParticleNumber",
            "GenerateTemp": t} for name, t in (("electron", 10.0), ("ion_Xe1", 0.1))]
    return {
        "FlagForEquation": {"Particle": 2, "EMField": 1, "MCCollision": 0},
        "ParamForTimeIntegration": {"Start": 0, "End": steps, "TimeStep": dt, "LogOutput": log_output,
                                    "ParticleOutput": 0, "FieldOutput": 0, "ProgressOutput": 0,
                                    "ProjectName": "es512_o3", "RestartName": "es512_o3"},
        "ParamForComputing": {"MaximumParticleNumber": int(npart * 1.02) + 4096, "ThreadGroupSize": 256,
                              "MaxiterForPoisson": 100, "ToleranceForPoisson": 1e-8},
        "ParamForField": {"NumberOfGridX": ngx, "NumberOfGridY": ngy, "GridSizeOfX": dx, "GridSizeOfY": dx,
                          "InitializeTypeOfE": "Uniform", "AmplitudeOfE": [0.0, 0.0, 0.0],
                          "InitializeTypeOfB": "Uniform", "AmplitudeOfB": [0.0, 0.0, 200.0],
                          "WeightingOrder": 3, "BorisOrder": 2},
        "ParamForParticle": [
            {"ParticleName": "electron", "pNumSetMethod": "PtclNumPerCell", "pNumValue": ppc, "Charge": -EC,
             "Mass": ME, "WeightSetMethod": "InitialNumDens", "WeightValue": n,
             "GenerateType": "uniform-Gaussian", "InitialTemp": 10.0},
            {"ParticleName": "ion_Xe1", "pNumSetMethod": "PtclNumPerCell", "pNumValue": ppc, "Charge": EC,
             "Mass": 1836 * 131.29 * ME, "WeightSetMethod": "InitialNumDens", "WeightValue": n,
             "GenerateType": "uniform-Gaussian", "InitialTemp": 0.1}],
        "SourceForParticle": src,
        "BoundaryConditionForParticle": [
            {"RegionName": "Xmin", "BCType": "Delete"}, {"RegionName": "Xmax", "BCType": "Delete"},
            {"RegionName": "Ymin", "BCType": "periodic"}, {"RegionName": "Ymax", "BCType": "periodic"}],
        "BoundaryConditionForField": [
            {"RegionName": "Xmin", "BCType": "Dirichlet", "Value": 0.0},
            {"RegionName": "Xmax", "BCType": "Dirichlet", "Value": 0.0},
            {"RegionName": "Ymin", "BCType": "periodic"}, {"RegionName": "Ymax", "BCType": "periodic"}],
    }


def workload_periodic(ngx, order, ppc, dt_wpe, bz_gauss=0.0, darwin=False, drift_frac=0.0, steps=200):
    """Doubly periodic ES (or Darwin) PIC of electrons and Xe+ with the bench
    workload's plasma: Te = 10 eV, Ti = 0.1 eV, n = 5e10 cm^-3, dx = 0.5
    Debye length, uniform Bz, Poisson to 1e-8. drift_frac adds an electron
    drift along y of drift_frac * vte * sin(2 pi x / Lx) (the build-added
    SinusoidalDriftVel loader key)."""
    c = workload(ppc=ppc, ngx=ngx, ngy=ngx, steps=steps)
    n = 5e10
    wpe = math.sqrt(4 * math.pi * n * EC ** 2 / ME)
    c["ParamForTimeIntegration"]["TimeStep"] = dt_wpe / wpe
    c["SourceForParticle"] = []
    c["BoundaryConditionForParticle"] = [{"RegionName": r, "BCType": "periodic"} for r in ("Xmin", "Xmax", "Ymin", "Ymax")]
    c["BoundaryConditionForField"] = [{"RegionName": r, "BCType": "periodic"} for r in ("Xmin", "Xmax", "Ymin", "Ymax")]
    c["ParamForField"]["WeightingOrder"] = order
    c["ParamForField"]["AmplitudeOfB"] = [0.0, 0.0, bz_gauss]
    c["ParamForComputing"]["MaxiterForPoisson"] = 200
    if darwin:
        c["FlagForEquation"]["EMField"] = 2
        c["ParamForField"]["FlagForCurDens"] = 1
    if drift_frac:
        vte = math.sqrt(2 * KB * 10.0 * EV_K / ME)
        c["ParamForParticle"][0]["SinusoidalDriftVel"] = [0.0, drift_frac * vte, 0.0]
    return c


def config_legs(steps):
    """Device-timed cycles of the other reference configurations: config 1
    (128^2 doubly periodic, CIC, 64 ppc, w_ce / w_pe = 0.5, dt w_pe = 0.1)
    and config 3 (1024^2 doubly periodic Darwin, order 5, 100 ppc, electron
    drift 0.1 vte sin(2 pi x / L) along y, dt w_pe = 0.05, Bz 0)."""
    from gample_b200 import capi
    n = 5e10
    wpe = math.sqrt(4 * math.pi * n * EC ** 2 / ME)
    out = {}
    cases = {"config1_es128_o1_64ppc": (workload_periodic(128, 1, 64, 0.1, bz_gauss=0.5 * wpe * ME * 2.99792458e10 / EC),
                                        3, 4 * steps),
             "config3_darwin1024_o5_100ppc": (workload_periodic(1024, 5, 100, 0.05, darwin=True, drift_frac=0.1),
                                              2, steps)}
    for name, (cond, warm, k) in cases.items():
        sim = capi.Sim(cond)
        sim.initialize()
        sim.run(warm)
        n0 = sim.count(0) + sim.count(1)
        ms = sim.time_cycles(k)
        n1 = sim.count(0) + sim.count(1)
        st = sim.last_solve()
        out[name] = {"steps": k, "ms_per_step": ms / k, "particles": n1,
                     "pushes_per_s": 0.5 * (n0 + n1) * k / (ms / 1e3),
                     "poisson_iterations": st.iterations, "poisson_rel_residual": st.error}
        sim.close()
    return out


def config_block(ppc):
    return {"workload": f"es-pic 512x512, order 3, Dirichlet-x absorbing + periodic-y, {ppc} ppc/species "
                        f"({2 * ppc * 512 * 512 / 1e6:.1f} M particles), Bz 0.02 T, dt*wpe 0.05, "
                        "flux re-injection at x=0, Poisson rel. residual 1e-8",
            "grid": [512, 512], "weighting_order": 3, "ppc_per_species": ppc,
            "particles": 2 * ppc * 512 * 512, "poisson_tol": 1e-8,
            "l2": "inputs larger than L2 (particle state 3.2 GB per step)"}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_tensor_peak():
    """Sustained dense BF16 TFLOP/s of this pool's B200s (cuBLAS, seconds-long loop)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops_sustained"]), "measured"
    except Exception:
        return 1400.0, "fallback"


def load_traffic():
    """DRAM bytes per pushed particle of the push kernel, from the committed ncu
    summary (a 128-ppc capture of the same kernel; traffic scales with the
    particles processed)."""
    try:
        with open(os.path.join(ROOT, "profiles", "push_es512_o3.md")) as f:
            for line in f:
                if line.startswith("dram_bytes_per_particle:"):
                    return {"dram_bytes_per_particle": float(line.split(":", 1)[1])}
    except OSError:
        pass
    return None


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        t_end = time.time() + 3.0
        while len(self.lines) < 3 and time.time() < t_end and self.proc.poll() is None:
            time.sleep(0.05)  # short timed regions: keep at least a few samples
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, smax, reasons, power = [], None, set(), []
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}



def poisson_block(vcycles, unknowns, solve_ms, peak):
    """The solve against its memory roofline: about 96 algorithmic bytes per
    fine point per V(2,2) cycle (2 x 2 sweeps of 12 B, the 16-B FP64 residual
    and 8 B of transfer, times 4/3 for the coarser levels)."""
    per_cycle = 96.0 * unknowns
    ms_cycle = solve_ms / vcycles if vcycles else None
    achieved = per_cycle / (ms_cycle * 1e-3) / 1e9 if ms_cycle else None
    return {"vcycles_last_step": vcycles, "tolerance": 1e-8, "solve_ms_per_step": solve_ms,
            "ms_per_vcycle_incl_cg": ms_cycle, "algorithmic_bytes_per_vcycle": per_cycle,
            "achieved_gbs": achieved, "frac_of_hbm": achieved / peak if achieved else None,
            "note": "latency-bound: 10 dependent launches per CG iteration at 512^2 (one CUDA graph, "
                    "programmatic dependent launches), CG dot products fused into the finest post-smoother, "
                    "levels <= 1024 points in one CTA"}


NET_SPECS_RESIDUAL = [(1, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2), (64, 64, 3),
                      (64, 64, 3), (128, 64, 2), (96, 32, 1), (48, 16, 0), (16, 1, 0)]


def learned_leg(cond, seeds, samples, train_steps, eval_steps, lr=1e-3, warm=10):
    """Config-4 style learned warm start of the 512^2 Poisson solve. The
    network (residual formulation: the normalised residual of the previous
    solution in, a correction out, 4 levels of 3x3 convolutions, widths
    16/32/64/64, BF16 tcgen05 GEMMs) is trained offline on residual samples
    the simulator generates: the run is reloaded from master seeds 0..seeds-1
    and, after `warm` cycles, each of `samples` solves per seed is banked.
    Then, on a held-out seed, every solve runs twice to the same 1e-8
    residual: from the plain warm start (previous phi) and from previous phi
    plus the network's correction; V-cycles and times of both are reported."""
    from gample_b200 import capi
    sim = capi.Sim(cond)
    sim.set_learned(16, lr, 0)
    sim.learned_bank(seeds * samples)
    t0 = time.perf_counter()
    for seed in range(seeds):
        sim.reload(seed)
        sim.initialize()
        sim.set_learned(16, lr)
        sim.run(warm)
        sim.set_learned(16 | 8, lr)
        sim.run(samples)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    tr = sim.learned_train(train_steps, lr, 1)
    train_s = time.perf_counter() - t0
    sim.reload(seeds)  # held out
    sim.initialize()
    sim.set_learned(16, lr)
    sim.run(warm)
    sim.set_learned(16 | 1 | 4, lr)
    rows = []
    for _ in range(eval_steps):
        sim.run(1)
        rows.append(sim.learned_stats())
    h = (sim.nky + 1 + 7) // 8 * 8
    w = (sim.nkx + 1 + 7) // 8 * 8
    sim.close()
    mean = lambda k: sum(r[k] for r in rows) / len(rows)
    flops = sum(2.0 * (h >> lv) * (w >> lv) * 9 * ci * co for ci, co, lv in NET_SPECS_RESIDUAL)
    ms_net = mean("ms_net")
    return {"poisson_ms_plain": mean("ms_plain"), "poisson_ms_learned": mean("ms_learned"),
            "vcycles_plain": mean("iters_plain"), "vcycles_learned": mean("iters_learned"),
            "vcycle_gain": mean("iters_plain") / mean("iters_learned"),
            "start_residual_plain": mean("rel0_plain"), "start_residual_learned": mean("rel0_learned"),
            "speedup": mean("ms_plain") / mean("ms_learned"), "network_ms": ms_net,
            "network_tflops": flops / (ms_net * 1e-3) / 1e12 if ms_net > 0 else None,
            "network_tensor_frac": (flops / (ms_net * 1e-3) / 1e12) / load_tensor_peak()[0] if ms_net > 0 else None,
            "network_gflop_per_forward": flops / 1e9, "training_samples": tr["samples"],
            "training_seeds": seeds, "train_steps": train_steps, "train_s": train_s, "sample_generation_s": gen_s,
            "loss_first10": tr["loss_first"], "loss_last10": tr["loss_last"], "eval_steps": eval_steps,
            "eval_seed": seeds,
            "note": "residual formulation, trained offline on simulator samples (master seeds 0..seeds-1); the "
                    "multigrid reaches 1e-8 from either start; loss = mean square of the residual left"}


def ensemble_leg(members, steps, threads, seed=0):
    """Config-5 style batch: independent runs with grids from {64..512}^2,
    orders {1, 3, 5}, Bz in [0, 0.05] T and 16..256 particles per cell per
    species, advanced together (one stream per member, host thread pool) and,
    for comparison, one after the other; both timed on the device with CUDA
    events on the member streams."""
    import random
    from gample_b200 import capi
    rnd = random.Random(seed)
    conds = []
    for _ in range(members):
        n = rnd.choice([64, 128, 256, 512])
        c = workload(ppc=rnd.randint(16, 256), ngx=n, ngy=n, steps=steps)
        c["ParamForField"]["WeightingOrder"] = rnd.choice([1, 3, 5])
        c["ParamForField"]["AmplitudeOfB"] = [0.0, 0.0, rnd.uniform(0.0, 0.05) * 1e4]
        conds.append(c)
    ens = capi.Ensemble(conds, threads=threads)
    ens.initialize()
    ens.run(2)
    n0 = sum(m.count(0) + m.count(1) for m in ens.members)
    t0 = time.perf_counter()
    ms = ens.time_cycles(steps)
    el = time.perf_counter() - t0
    n1 = sum(m.count(0) + m.count(1) for m in ens.members)
    chunks = {}
    for m in ens.members:
        for sp in range(2):
            st = m.push_stats(sp)
            key = f"{st[5]}{'' if st[6] else ' no tables'}"
            chunks[key] = chunks.get(key, 0) + 1
    ens.close()
    del ens
    batched = 0.5 * (n0 + n1) * steps / (ms / 1e3)
    seq_ms, seq_n = 0.0, 0.0
    for c in conds:
        sim = capi.Sim(c)
        sim.initialize()
        sim.run(2)
        a = sim.count(0) + sim.count(1)
        seq_ms += sim.time_cycles(steps)
        seq_n += 0.5 * (a + sim.count(0) + sim.count(1)) * steps
        sim.close()
    sequential = seq_n / (seq_ms / 1e3)
    return {"members": members, "threads": threads, "steps": steps, "particles": n1,
            "ppc_range": [16, 256], "pushes_per_s": batched, "sequential_pushes_per_s": sequential,
            "speedup": batched / sequential, "ms": ms, "wall_s": el,
            "autotuned_push_variants": chunks,
            "timing": "CUDA events on the member streams: earliest member start to latest member end; "
                      "sequential: the sum of each member's device-timed cycles run alone"}


def steady_state_leg(sim, warm, steps):
    """The same run continued well past the initial cell sort: `warm` more
    cycles (absorption and re-injection settle, the electrons drift and the
    re-sort cadence sets in), then `steps` cycles timed with CUDA events on
    the library's stream, one call per cycle so that the cycles with a
    re-sort can be counted."""
    from gample_b200 import capi
    sim.run(warm)
    n0 = sim.count(0) + sim.count(1)
    l0 = capi.kernel_launches()
    ms, pulled, sorts = [], [], 0
    sim.set_profiling(True)
    prev = sim.phase_times()["sort"]
    for _ in range(steps):
        ms.append(sim.time_cycles(1))
        pulled.append(sim.last_flow(0).pulled + sim.last_flow(1).pulled)
        t = sim.phase_times()["sort"]
        sorts += t > prev
        prev = t
    sim.set_profiling(False)
    launches = capi.kernel_launches() - l0
    n1 = sim.count(0) + sim.count(1)
    total = sum(ms)
    return {"cycles_before_timing": warm, "steps": steps, "ms_per_step": total / steps,
            "pushes_per_s": 0.5 * (n0 + n1) * steps / (total / 1e3),
            "ms_per_step_min": min(ms), "ms_per_step_max": max(ms), "sorts": int(sorts),
            "absorbed_per_cycle": sum(pulled) / steps, "gpu_launches_per_step": launches / steps,
            "timing": "CUDA events per cycle on the library's stream (per-phase events on: ~1 % overhead)"}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def aggregate_ranks(ms, pushes, pg=None, device="cuda"):
    """Whole-job numbers of a replica run: the step time is the maximum over
    ranks (each rank's own CUDA-event time), the pushes the sum over ranks.
    Returns (ms_max, total pushes, pushes per second)."""
    ms_max, total = float(ms), float(pushes)
    if pg is not None:
        import torch
        t = torch.tensor([ms], device=device, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        c = torch.tensor([pushes], device=device, dtype=torch.float64)
        pg.all_reduce(c, op=pg.ReduceOp.SUM)
        ms_max, total = float(t.item()), float(c.item())
    return ms_max, total, total / (ms_max / 1e3)


def cpu_baseline_run(steps, warmup, ppc_sample, threads=None):
    """The oracle (C++ restatement of the reference's CPU arithmetic, OpenMP)
    on the same grid/physics with ppc_sample particles per cell per species."""
    from oracle import config as ocfg
    from oracle import lib as L
    cond = workload(ppc=ppc_sample)
    sim = L.OracleSim(ocfg.parse(cond), real64=False)
    sim.load_initial()
    sim.reset_charge()
    for s in range(2):
        sim.deposit(s)
    sim.solve_poisson(0.0)
    for c in range(warmup):
        sim.cycle(c + 1, faithful=False)
    n0 = sim.pnum(0) + sim.pnum(1)
    t0 = time.perf_counter()
    for c in range(steps):
        sim.cycle(warmup + c + 1, faithful=False)
    el = time.perf_counter() - t0
    n1 = sim.pnum(0) + sim.pnum(1)
    pushes = 0.5 * (n0 + n1) * steps
    return pushes / el, el, L.num_threads()


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    ppc = args.ref_ppc
    value, el, cores = cpu_baseline_run(args.steps, args.warmup, ppc)
    line = {"metric": METRIC, "value": value, "unit": "particle-pushes/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / max(args.steps, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded reference loader)",
            "config": config_block(ppc),
            "cpu_baseline": {"value": value, "unit": "particle-pushes/s", "cores": cores, "kind": "port",
                             "sample": f"full 512x512 grid and field solve, {ppc} ppc/species "
                                       f"({2 * ppc * 512 * 512 / 1e6:.1f} M particles) per step; the "
                                       "reference's Metal/AMGCL build does not exist on Linux, so its CPU "
                                       "algorithm is the oracle's C++ restatement"},
            "e2e": {"value": value, "unit": "particle-pushes/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_b200(args):
    world, rank, local = dist_setup()
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    from gample_b200 import capi

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    ppc = args.ppc
    cond = workload(ppc=ppc)
    if args.sort_interval:
        cond["ParamForComputing"]["SortInterval"] = args.sort_interval
    sim = capi.Sim(cond)
    sim.initialize()
    if args.warmup:
        sim.run(args.warmup)
    n0 = sim.count(0) + sim.count(1)
    clocks = ClockSampler(local)
    # per-phase CUDA events on the library's stream inside the timed region
    # (the push kernel's launch time for the roofline); not in profiler runs
    if not args.quick:
        sim.set_profiling(True)
    barrier()
    clocks.start()
    l0 = capi.kernel_launches()
    ms = sim.time_cycles(args.steps)
    launches = capi.kernel_launches() - l0
    barrier()
    clk = clocks.stop()
    ph = sim.phase_times() if not args.quick else None
    sim.set_profiling(False)
    n1 = sim.count(0) + sim.count(1)
    if args.quick:  # profiling runs: the timed cycles only
        if rank == 0:
            print(json.dumps({"quick": True, "ms_per_step": ms / args.steps, "particles": n1,
                              "pushes_per_s": 0.5 * (n0 + n1) * args.steps / (ms / 1e3),
                              "gpu_launches": launches}), flush=True)
        sim.close()
        return 0
    iters_last = sim.last_solve().iterations
    unknowns = (sim.nkx + 1) * (sim.nky + 1)
    pushes_rank = 0.5 * (n0 + n1) * args.steps
    ms_max, _, value = aggregate_ranks(ms, pushes_rank, pg)

    # Roofline of the dominant kernel (push + fused deposit), from the phase
    # events of the timed cycles: two launches (species) per cycle.
    prof_cycles = args.steps
    push_ms_per_launch = ph["push"] / (2 * prof_cycles)
    particles_per_launch = 0.25 * (n0 + n1)
    peak, peak_kind = load_peaks()
    achieved = BYTES_PER_PUSH * particles_per_launch / (push_ms_per_launch / 1e3) / 1e9
    tr = load_traffic()
    traffic = tr["dram_bytes_per_particle"] * particles_per_launch if tr else None
    variants = [sim.push_stats(sp)[5:7] for sp in range(2)]
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_kind": peak_kind, "kernel": "k_push (gather+Boris+BC+fused deposit)",
                "algorithmic_bytes_per_particle": BYTES_PER_PUSH,
                "phase_ms_per_step": {k: v / prof_cycles for k, v in ph.items()},
                "push_variant": [{"particles_per_chunk": v[0], "tables": bool(v[1])} for v in variants]}
    steady = steady_state_leg(sim, args.steady_warm, args.steady_steps) if args.steady_steps > 0 else None
    sim.close()
    del sim

    # End to end through the C ABI with host buffers: restart-style upload of
    # the initial particle state from pinned host memory, initial solve, K
    # logged cycles (CSV/XML written every cycle), download of the final
    # state to pinned host memory.
    e2e = None
    if rank == 0 or True:
        src = capi.Sim(cond)
        states = [src.particles(s) for s in range(2)]
        src.close()
        del src
        pinned = []
        for st in states:
            t = torch.empty(st.nbytes, dtype=torch.uint8, pin_memory=True)
            np.frombuffer(t.numpy(), dtype=np.uint8)[:] = st.view(np.uint8)
            pinned.append((t, len(st)))
        out_pinned = [torch.empty(int(st.nbytes * 1.02) + 4096 * 24, dtype=torch.uint8, pin_memory=True)
                      for st in states]
        with tempfile.TemporaryDirectory() as td:
            c2 = dict(cond)
            c2["ParamForTimeIntegration"] = dict(cond["ParamForTimeIntegration"], LogOutput=1)
            barrier()
            t0 = time.perf_counter()
            sim2 = capi.Sim(c2, log_name=os.path.join(td, "es512"))
            h2d = 0
            for s, (t, n) in enumerate(pinned):
                capi.check(capi.lib().gp_particle_upload(sim2.h, s, t.data_ptr(), n))
                h2d += n * 24
            sim2.initialize()
            sim2.run(args.steps)
            d2h = 0
            for s in range(2):
                n = sim2.count(s)
                got = capi.C.c_uint32()
                capi.check(capi.lib().gp_particle_download(sim2.h, s, out_pinned[s].data_ptr(),
                                                           out_pinned[s].numel() // 24, capi.C.byref(got)))
                d2h += got.value * 24
            n_e2e = 0.5 * (sum(len(s) for s in states) + sim2.count(0) + sim2.count(1))
            sim2.close()
            el = time.perf_counter() - t0
        # per-step diagnostics read back by the logger: solve stats (8 doubles)
        # and two species counters (2 x 48 B)
        diag = 64 + 96
        e2e = {"value": n_e2e * args.steps * world / el, "unit": "particle-pushes/s",
               "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps + diag),
               "wall_s": el, "includes": "sim create + restart upload + initial solve + K logged cycles + "
                                         "final download"}
    configs = config_legs(args.config_steps) if rank == 0 and args.config_steps > 0 else None
    ensemble = None
    if rank == 0 and args.ensemble > 0:
        ensemble = ensemble_leg(args.ensemble, args.ensemble_steps, args.ensemble_threads)
    learned = None
    if rank == 0 and args.learned_train > 0:
        learned = learned_leg(cond, args.learned_seeds, args.learned_samples, args.learned_train, args.learned_eval,
                              args.learned_lr)
    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        v, el, cores = cpu_baseline_run(args.cpu_steps, 1, args.cpu_ppc)
        cpu = {"value": v, "unit": "particle-pushes/s", "cores": cores, "kind": "port",
               "sample": f"oracle C++ restatement, full 512x512 grid + Poisson (FP64 CG to 1e-8), "
                         f"{args.cpu_ppc} ppc/species ({2 * args.cpu_ppc * 512 * 512 / 1e6:.1f} M particles), "
                         f"{args.cpu_steps} steps after 1 warm-up step, {el:.1f} s"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "particle-pushes/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded reference loader, splitmix64/PCG32)", "config": config_block(ppc),
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
                "gpu_launches": launches, "gpu_launches_per_step": launches / args.steps,
                "timing": "CUDA events around the K cycles on the library's stream, per-phase events inside "
                          "(roofline and poisson blocks); max over ranks",
                "poisson": poisson_block(iters_last, unknowns, roofline["phase_ms_per_step"]["solve"], peak),
                "steady_state": steady,
                "other_configs": configs,
                "learned_warm_start": learned,
                "ensemble": ensemble}
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def run_resort_probe(args):
    """The periodic re-sort's input, for profiling its kernels: the workload
    at --ppc run --resort-probe cycles without sorting (drifted particles,
    refilled holes, re-injected strays), then one block-local re-sort of the
    electrons, timed with CUDA events around the call's stream work."""
    from gample_b200 import capi
    cond = workload(ppc=args.ppc)
    cond["ParamForComputing"]["SortInterval"] = 1 << 30
    sim = capi.Sim(cond)
    sim.initialize()
    sim.run(args.resort_probe)
    slow = sim.push_stats(0)[0]
    sim.synchronize()
    t0 = time.perf_counter()
    sim.sort(0, 1)
    ms = 1e3 * (time.perf_counter() - t0)
    print(json.dumps({"resort_probe": args.resort_probe, "ppc": args.ppc, "electrons": sim.count(0),
                      "pushed_outside_window_before": slow, "sort_ms_host": ms}), flush=True)
    sim.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--ppc", type=int, default=256)
    ap.add_argument("--cpu-ppc", type=int, default=256)
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--ref-ppc", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--learned-train", type=int, default=2000, help="offline training steps of the warm-start network")
    ap.add_argument("--learned-seeds", type=int, default=20, help="master seeds whose runs give training samples")
    ap.add_argument("--learned-samples", type=int, default=25, help="residual samples banked per seed")
    ap.add_argument("--learned-lr", type=float, default=1e-3)
    ap.add_argument("--learned-eval", type=int, default=20)
    ap.add_argument("--config-steps", type=int, default=5,
                    help="timed cycles of the config-3 leg (config 1: 4x; 0: skip both)")
    ap.add_argument("--ensemble", type=int, default=64, help="members of the batched-ensemble leg (0: skip)")
    ap.add_argument("--ensemble-steps", type=int, default=10)
    ap.add_argument("--ensemble-threads", type=int, default=16)
    ap.add_argument("--steady-warm", type=int, default=200, help="cycles run before the steady-state leg")
    ap.add_argument("--steady-steps", type=int, default=50, help="cycles timed in the steady-state leg (0: skip)")
    ap.add_argument("--quick", action="store_true", help="timed cycles only (for profiler runs)")
    ap.add_argument("--sort-interval", type=int, default=0,
                    help="SortInterval of the main run (0: adaptive; profiler runs fix it so that the cadence does "
                         "not follow the profiler's timings)")
    ap.add_argument("--resort-probe", type=int, default=0,
                    help="profiler case: K cycles without sorting, then one re-sort of the electrons")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.resort_probe > 0:
        return run_resort_probe(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
