"""Benchmark: particle-steps/s of the PIC-MCC electron step (push + MCC +
deposit, with the FDTD field update inside every timed step) on the 2,000,000
electron workload (1,000,000 photoionizations by 8 keV photons in N2 at 1 Torr,
256 x 1024 cells of 5 um, dt = 1e-14 s, secondaries on, seed 1).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1); each rank runs an independent
replica of the workload (no data-path collective), timing is device-side
(CUDA events), max over ranks.  Rank 0 prints one JSON line.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gas-atenuator_b200"))

METRIC = "particle-steps/s (push+MCC+deposit), FP32 vs FP64 GPU at ≤0.5% yield error"
UNIT = "particle-steps/s"
WORKLOAD = dict(n_r=256, n_z=1024, delta=5e-6, dt=1e-14, torr=1.0, photo=1_000_000, e_keV=8.0,
                seed=1)
WORKLOAD_NAME = ("2,000,000 e- from 1,000,000 photoionizations at 8 keV (photoelectron 7.59 keV, "
                 "dipole about x; Auger 360 eV isotropic), N2 1 Torr 300 K, 256x1024 cells at 5 um, "
                 "dt 1e-14 s, Rayleigh sigma 50 um, secondaries on, seed 1")
L2_FLUSH_BYTES = 256 << 20
# algorithmic bytes: per alive particle-step, twice the state (read + written): FP32 split
# 24 B (int32 cell key, 2 x f32 offsets, 3 x f32 gamma*v), FP64 40 B (r, z, 3 x gamma*v); the
# id the random streams are keyed on is not counted.  Grid term per step: field gather
# (3 fields) + current (2 x int64).
BYTES_PER_PARTICLE = {"fp32_split": 48, "fp64": 80}
GRID_BYTES_PER_CELL = {"fp32_split": 3 * 4 + 2 * 8, "fp64": 3 * 8 + 2 * 8}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0}, "fallback"


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-i", str(self.device)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1])); mx.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------ ours (GPU)
SORT_PERIODS = (20, 30, 40, 60)     # candidates of the sort period for the autotuner
KNOBS = ("fdtd_tile_rows", "pass_chunk", "gather", "sort_period")


def workload_setup(precision, rank, knobs=None):
    from gasatt import abi
    from gasatt.workload import births, config
    w = WORKLOAD
    prec = abi.FP32_SPLIT if precision == "fp32_split" else abi.FP64
    cfg = config(w["n_r"], w["n_z"], w["delta"], w["dt"], w["torr"], precision=prec,
                 capacity=4_000_000, seed=replica_seed(rank), sort_period=20)
    for k, v in (knobs or {}).items():
        setattr(cfg, k, int(v))
    parts = births(w["photo"], w["e_keV"], w["n_z"] * w["delta"], seed=replica_seed(rank),
                   Rp=w["n_r"] * w["delta"])
    return cfg, parts


def make_sim(precision, device, rank, torch, knobs=None):
    from gasatt.sim import Sim
    cfg, parts = workload_setup(precision, rank, knobs)
    sim = Sim(cfg, device=device)
    sim.bind_stream()
    sim.load(*parts)
    return sim, parts


def tuned_knobs(precision, device, rank):
    """The launch-shape knobs (field patch rows, FP32 chunk size and gather
    source, sort period)
    the autotuner picks for this workload by coordinate descent; results do
    not depend on them (see gasatt.tune).  Returns ({knob: value}, {knob:
    {candidate: ms per step}})."""
    from gasatt.tune import knob_candidates, tune
    cfg, parts = workload_setup(precision, rank)
    knobs = knob_candidates(cfg)
    knobs["sort_period"] = SORT_PERIODS
    best, table = tune(cfg, parts, knobs=knobs, steps=200, device=device)
    return {k: int(getattr(best, k)) for k in knobs}, table


def counts(sim):
    from gasatt._lib import lib
    a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    lib.gasatt_sim_counts(sim.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    return a.value, b.value, c.value


def aligned_warmup(warmup, sort_period):
    """Warm-up steps stretched to a multiple of the sort period.  A run sorts
    at its steps 0, P, 2P, ... (counted from the load), so K timed steps that
    start on a multiple of P contain ceil(K / P) sorts: never fewer than their
    share of the periodic sort."""
    if sort_period <= 0:
        return warmup
    return -(-warmup // sort_period) * sort_period


def timed_run(sim, steps, warmup, torch, flush, dist_barrier, sort_period, phase_steps=300):
    """K steps, each preceded by an L2 flush (outside its event pair), through
    the production step graphs: the whole-step time, the periodic sort
    included when it falls in a step.  The host waits for each step before
    enqueuing the next flush; the flush (256 MiB) runs long enough for the
    next step's launch to be queued behind it.  Then `phase_steps` more
    flushed steps through the instrumented copies of the step graphs (event
    nodes right before and after each kernel) give the field update and the
    particle pass apart; those event nodes cost about 10 us per step, so they
    are kept out of the headline steps."""
    from gasatt._lib import lib
    stream = torch.cuda.current_stream()
    pre = aligned_warmup(warmup, sort_period)
    lib.gasatt_sim_enable_timing(sim.h, 0)
    sim.step(pre)
    torch.cuda.synchronize()
    d0 = sim.diag()
    l0 = sim.ctx.launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    step_ms = []
    dist_barrier()
    torch.cuda.synchronize()
    for _ in range(steps):
        flush()                                      # L2 cold before every timed step
        e0.record(stream)
        sim.step(1)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    dist_barrier()
    launches = sim.ctx.launches - l0
    d1 = sim.diag()
    # phases, in the instrumented step graphs
    fd = ctypes.c_float(); ps = ctypes.c_float(); mc = ctypes.c_float()
    pass_ms, fdtd_ms, mcc_ms = [], [], []
    lib.gasatt_sim_enable_timing(sim.h, 1)
    for _ in range(phase_steps):
        flush()
        sim.step(1)
        torch.cuda.synchronize()
        lib.gasatt_sim_last_timing(sim.h, ctypes.byref(fd), ctypes.byref(ps), ctypes.byref(mc))
        fdtd_ms.append(fd.value); pass_ms.append(ps.value); mcc_ms.append(mc.value)
    lib.gasatt_sim_enable_timing(sim.h, 0)
    dist_barrier()
    sorts = sum(1 for i in range(pre, pre + steps) if sort_period > 0 and i % sort_period == 0)
    return dict(step_ms=step_ms, pass_ms=pass_ms, fdtd_ms=fdtd_ms, mcc_ms=mcc_ms, d0=d0, d1=d1,
                launches=launches, sorts=sorts, warmup_steps=pre)


ME_C2_EV = 510998.95                                 # m_e c^2 [eV]


def energies_ev(p):
    """Kinetic energies [eV] of the live electrons of a Sim.read() dict."""
    a = p["r"] >= 0
    u2 = (p["ur"][a] ** 2 + p["ut"][a] ** 2 + p["uz"][a] ** 2) / 299792458.0 ** 2
    return ME_C2_EV * (u2 / (np.sqrt(1 + u2) + 1))


def accuracy_run(precision, device, rank, torch, steps, knobs):
    """The workload free-running for `steps` steps (its stated length): the
    event counts, the fields and the electrons' energies at the end."""
    sim, _ = make_sim(precision, device, rank, torch, knobs)
    sim.step(steps)
    torch.cuda.synchronize()
    out = dict(diag=sim.diag(), fields=sim.fields(), E=energies_ev(sim.read()))
    sim.close()
    return out


def compare_forms(a32, a64):
    """FP32 split form against the FP64 form after the same steps: yield
    error, field errors, the electron energy distribution (40 log bins from
    0.1 eV to 10 keV) and the mean energy, each with its Monte Carlo error."""
    d32, d64 = a32["diag"], a64["diag"]
    i32, i64 = d32["n_ionizations"], d64["n_ionizations"]
    pairs = list(zip(a32["fields"], a64["fields"]))
    ferr = max(float(np.linalg.norm((x - y).ravel()) / max(np.linalg.norm(y.ravel()), 1e-300))
               for x, y in pairs)
    fmax = max(float(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-300)) for x, y in pairs)
    E32, E64 = a32["E"], a64["E"]
    bins = np.logspace(-1, 4, 41)
    h32, _ = np.histogram(E32, bins)
    h64, _ = np.histogram(E64, bins)
    used = (h32 + h64) > 0
    chi2 = float(np.sum((h32[used] - h64[used]) ** 2 / (h32[used] + h64[used])))
    zbin = float(np.max(np.abs(h32 - h64) / np.sqrt(h64 + 1.0)))
    s32, s64 = np.sort(E32), np.sort(E64)
    grid = np.concatenate([s32, s64])
    ks = float(np.max(np.abs(np.searchsorted(s32, grid, side="right") / len(s32)
                             - np.searchsorted(s64, grid, side="right") / len(s64))))
    sig_mean = float(E64.std() / np.sqrt(len(E64)))
    dmean = float(E32.mean() - E64.mean())
    return {
        "yield_rel_err_fp32_vs_fp64": abs(i32 - i64) / max(i64, 1),
        "ionizations_fp32": int(i32), "ionizations_fp64": int(i64),
        "yield_diff_in_sigma": abs(i32 - i64) / max(math.sqrt(i64), 1.0),
        "field_rel_err_fp32_vs_fp64": ferr,
        "field_rel_err_definition": "max over Er, Ez, H of ||F32 - F64||_2 / ||F64||_2",
        "field_max_abs_rel_err_fp32_vs_fp64": fmax,
        "eedf_chi2": chi2, "eedf_dof": int(used.sum()),
        "eedf_max_bin_diff_in_sigma": zbin,
        "eedf_ks_distance": ks,
        "eedf_ks_critical_1pct": 1.63 * math.sqrt((len(E32) + len(E64)) / (len(E32) * len(E64))),
        "mean_energy_ev_fp32": float(E32.mean()), "mean_energy_ev_fp64": float(E64.mean()),
        "mean_energy_diff_in_sigma": abs(dmean) / sig_mean if sig_mean > 0 else 0.0,
        "electrons_fp32": int(len(E32)), "electrons_fp64": int(len(E64)),
        "kinetic_rel_fp32_vs_fp64": d32["kinetic_ev"] / d64["kinetic_ev"] - 1,
        "gates": {"yield_rel_err_max": 0.005, "field_rel_err_max": 1e-4,
                  "three_sigma": "eedf bins, mean energy and yield within 3 sigma"},
    }


def e2e_run(precision, device, rank, torch, steps_per_call=200, knobs=None):
    """Through the public C ABI with pinned HOST buffers: H2D of the electrons,
    steps_per_call steps, D2H of the result, all inside the timed region."""
    from gasatt._lib import lib
    sim, parts = make_sim(precision, device, rank, torch, knobs)
    r, z, ur, ut, uz, ids = parts
    n = len(r)
    cap = int(n * 1.1)
    c = 299792458.0
    g = np.sqrt(1 + (ur * ur + ut * ut + uz * uz) / (c * c))
    pos = torch.zeros(3 * cap, dtype=torch.float64).pin_memory()
    vel = torch.zeros(3 * cap, dtype=torch.float64).pin_memory()
    P, V = pos.numpy(), vel.numpy()

    def fill():
        P[:n] = r; P[cap:cap + n] = 0.0; P[2 * cap:2 * cap + n] = z
        V[:n] = ur / g; V[cap:cap + n] = ut / g; V[2 * cap:2 * cap + n] = uz / g

    def call(k):
        nio = ctypes.c_int64(n)
        rc = lib.gasatt_sim_run_host(sim.h, ctypes.c_void_p(pos.data_ptr()),
                                     ctypes.c_void_p(vel.data_ptr()), ctypes.byref(nio), cap, k)
        assert rc == 0, lib.gasatt_last_error(sim.ctx.handle)
        return nio.value

    fill()
    call(5)                                          # warm-up call
    fill()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    nout = call(steps_per_call)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    sim.close()
    return dict(ms=ms, n_in=n, n_out=nout, steps=steps_per_call,
                h2d=n * 6 * 8, d2h=nout * 6 * 8)


def cpu_baseline(target_s=12.0):
    """CPU oracle (plain C FP64 restatement, OpenMP on all host cores) on the
    same workload: full population, a bounded number of steps."""
    threads = os.cpu_count() or 1
    O, orc = oracle_workload(2_200_000)
    O.lib.orc_set_threads(threads)
    orc.prologue()
    t0 = time.perf_counter()
    orc.step()
    one = time.perf_counter() - t0
    steps = max(1, min(200, int(target_s / max(one, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(steps):
        orc.step()
    dt = time.perf_counter() - t0
    n_alive = int(orc.alive[:orc.n].sum())
    return {"value": n_alive * steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"full 2,000,000-electron population, {steps} steps after 1 warm-up step; "
                      f"{ORACLE_WHAT}; OpenMP {threads} threads"}


class Ranks:
    """The ranks of one run: independent replicas, one process per GPU.  Work
    adds up over ranks; time is the slowest rank's.  Reductions go through the
    process group on `device` ("cuda" with NCCL, "cpu" with gloo)."""

    def __init__(self, dist=None, world=1, rank=0, device="cpu"):
        self.dist, self.world, self.rank, self.device = dist, world, rank, device

    def _reduce(self, x, op):
        if self.world == 1:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x):
        return self._reduce(x, self.dist.ReduceOp.MAX if self.world > 1 else None)

    def sum(self, x):
        return self._reduce(x, self.dist.ReduceOp.SUM if self.world > 1 else None)

    def rate(self, units_local, ms_local):
        """Whole-job rate: all ranks' units over the slowest rank's time."""
        return self.sum(units_local) / (self.max(ms_local) / 1e3)


def replica_seed(rank):
    """Each rank simulates its own gas cell: the workload's seed offset by rank."""
    return WORKLOAD["seed"] + 1000 * rank


def run_ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    ranks = Ranks(dist, world, rank, "cuda")
    barrier, max_over_ranks, sum_over_ranks = ranks.barrier, ranks.max, ranks.sum

    flush_buf = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def flush():
        flush_buf.fill_(1)

    results = {}
    clocks = None
    tuned = {}
    accuracy_legs = {}
    for prec in ("fp32_split", "fp64"):
        knobs, table = tuned_knobs(prec, local, rank)
        # every rank uses the same launch shapes (and sorts in the same steps)
        knobs = {k: int(max_over_ranks(v)) for k, v in knobs.items()}
        tuned[prec] = (knobs, table)
        sp = knobs["sort_period"]
        sim, _ = make_sim(prec, local, rank, torch, knobs)
        if prec == "fp32_split":
            with ClockSampler(local) as cs:
                res = timed_run(sim, args.steps, args.warmup, torch, flush, barrier, sp)
            clocks = cs.summary()
        else:
            res = timed_run(sim, args.steps, args.warmup, torch, flush, barrier, sp)
        results[prec] = res
        sim.close()
        # the accuracy gates at the workload's stated length (2000 steps)
        accuracy_legs[prec] = accuracy_run(prec, local, rank, torch, args.accuracy_steps, knobs)
    e2e = e2e_run("fp32_split", local, rank, torch, steps_per_call=200,
                  knobs=tuned["fp32_split"][0])
    # the batched workload (48 uneven cells in one batch) in both forms
    c3 = {prec: c3_batched(prec, local, torch) for prec in ("fp32_split", "fp64")}

    pk, pk_src = peaks()
    hbm = float(pk.get("hbm_gbs", 6650.0))
    out = {}
    for prec, res in results.items():
        t_ms = sum(res["step_ms"])
        t_ms_max = max_over_ranks(t_ms)
        alive = 0.5 * (res["d0"]["n_alive"] + res["d1"]["n_alive"])
        tot = sum_over_ranks(alive * args.steps)
        pass_avg = sum(res["pass_ms"]) / len(res["pass_ms"])
        fdtd_avg = sum(res["fdtd_ms"]) / len(res["fdtd_ms"])
        mcc_avg = sum(res["mcc_ms"]) / len(res["mcc_ms"])
        ncell = WORKLOAD["n_r"] * WORKLOAD["n_z"]
        bytes_launch = alive * BYTES_PER_PARTICLE[prec] + ncell * GRID_BYTES_PER_CELL[prec]
        out[prec] = dict(value=tot / (t_ms_max / 1e3), ms_per_step=t_ms_max / args.steps,
                         pass_ms=pass_avg, fdtd_ms=fdtd_avg, mcc_ms=mcc_avg, alive=alive,
                         achieved_gbs=bytes_launch / (pass_avg / 1e3) / 1e9,
                         ionizations=res["d1"]["n_ionizations"] - res["d0"]["n_ionizations"],
                         ion_total=res["d1"]["n_ionizations"], launches=res["launches"],
                         bytes_launch=bytes_launch,
                         cell_updates_per_s=ncell / (fdtd_avg / 1e3))
    f32, f64 = out["fp32_split"], out["fp64"]
    accuracy = compare_forms(accuracy_legs["fp32_split"], accuracy_legs["fp64"])
    accuracy["steps"] = args.accuracy_steps
    e2e_ms = max_over_ranks(e2e["ms"])
    e2e_val = sum_over_ranks(e2e["n_in"] * e2e["steps"]) / (e2e_ms / 1e3)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()
        cpu["matlab_path"] = matlab_path_baseline()
    # DRAM bytes (read + write) of one k_pass32 launch from an ncu capture of
    # this workload, scaled from the captured launch's electron count to this
    # run's mean count (the traffic is per particle: state and id)
    traffic = None
    tp = os.path.join(ROOT, "profiles", "k_pass32_c2_traffic.json")
    if os.path.exists(tp):
        try:
            t = json.load(open(tp))
            traffic = t["bytes_per_launch"] * f32["alive"] / t["particles"]
        except Exception:
            traffic = None
    line = {
        "metric": METRIC, "value": f32["value"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": f32["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded photoionization births; N2 cross-sections from the reference CSVs)",
        "config": {"workload": WORKLOAD_NAME, "precision": "fp32_split (int32 cell key + f32 offsets "
                   "+ f32 gamma*v; f64 collision test, energy sharing, threshold subtraction)",
                   "global_electrons": int(sum_over_ranks(f32["alive"])),
                   "per_rank": "independent replica", "parallelism": f"replicas x{world}",
                   "l2": "flushed before every timed step (256 MiB write, outside the events)",
                   "sort_period": tuned["fp32_split"][0]["sort_period"],
                   "autotuned": {"knobs": tuned["fp32_split"][0],
                                 "ms_per_step": {k: {str(c): round(v, 5) for c, v in t.items()}
                                                 for k, t in tuned["fp32_split"][1].items()},
                                 "fp64_knobs": tuned["fp64"][0],
                                 "method": "coordinate descent, 200 steps per candidate on a "
                                           "fresh copy of the population"},
                   "fdtd_ratio": 1,
                   "timed": (f"{args.steps} whole steps (field update + particle pass; the periodic "
                             f"sort inside the step it falls in); warm-up stretched to "
                             f"{results['fp32_split']['warmup_steps']} steps so that the window "
                             f"holds ceil(K / sort period) = {results['fp32_split']['sorts']} sorts"),
                   "sorts_in_timed_steps": results["fp32_split"]["sorts"],
                   "phases": "pass_ms and fdtd_ms: 300 more flushed steps through instrumented "
                             "copies of the step graphs (event nodes right before and after each "
                             "kernel, which add about 10 us per step and are kept out of the "
                             "headline steps); roofline.achieved uses this pass_ms"},
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": e2e["h2d"] / e2e["steps"],
                "d2h_bytes_per_step": e2e["d2h"] / e2e["steps"],
                "call": f"gasatt_sim_run_host, {e2e['steps']} steps per call, pinned host x,y,z,vx,vy,vz in/out"},
        "gpu_launches": int(f32["launches"]),
        "roofline": {"bound": "hbm", "achieved": f32["achieved_gbs"], "peak": hbm, "unit": "GB/s",
                     "frac": f32["achieved_gbs"] / hbm, "traffic": traffic,
                     "kernel": "k_pass32 (fused push+MCC+deposit)",
                     "peak_source": f"{pk_src} hbm_gbs",
                     "bytes_per_launch": f32["bytes_launch"]},
        "fp64": {"value": f64["value"], "ms_per_step": f64["ms_per_step"], "pass_ms": f64["pass_ms"],
                 "sort_period": tuned["fp64"][0]["sort_period"], "sorts_in_timed_steps": results["fp64"]["sorts"],
                 "mcc_ms": f64["mcc_ms"], "fdtd_ms": f64["fdtd_ms"],
                 "achieved_gbs": f64["achieved_gbs"], "frac": f64["achieved_gbs"] / hbm},
        "fp32_over_fp64": f32["value"] / f64["value"],
        "batched": {"workload": "48 gas cells: p log-U(0.1, 10) Torr, grid from {64x256, 128x512, "
                                "256x1024, 512x2048} at 10 um, dt 2e-14 s, photon U(2, 20) keV, "
                                "photoionizations log-U(1e4, 1e6), seed 2; births drawn on the GPU; "
                                "one batch step = every cell one step",
                    "fp32_split": {k: c3["fp32_split"][k] for k in ("value", "ms_per_step", "electrons")},
                    "fp64": {k: c3["fp64"][k] for k in ("value", "ms_per_step", "electrons")},
                    "fp32_batched_over_fp64_batched": c3["fp32_split"]["value"] / c3["fp64"]["value"],
                    "steps": c3["fp32_split"]["steps"],
                    "l2": "not flushed (the 48 cells' state exceeds the L2)"},
        "accuracy": accuracy,
        "fdtd": {"cell_updates_per_s": f32["cell_updates_per_s"], "ms": f32["fdtd_ms"],
                 "note": "one cell-update = one cell advanced by a full particle step (H, E, H, E, H sub-updates)"},
        "pass_ms": f32["pass_ms"], "mcc_ms": f32["mcc_ms"],
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------ reference arm (CPU)
def oracle_workload(cap):
    """The workload's configuration, births and tables for the CPU oracle,
    built without the CUDA library (gasatt.workload / gasatt.tables load none)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    from gasatt import abi
    from gasatt.tables import N2Tables
    from gasatt.workload import births, config
    w = WORKLOAD
    cfg = config(w["n_r"], w["n_z"], w["delta"], w["dt"], w["torr"], precision=abi.FP64,
                 capacity=cap, seed=w["seed"], sort_period=0)
    parts = births(w["photo"], w["e_keV"], w["n_z"] * w["delta"], seed=w["seed"],
                   Rp=w["n_r"] * w["delta"])
    orc = O.Sim(cfg, N2Tables(), cap=cfg.capacity)
    orc.load(*parts)
    return O, orc


def matlab_path_baseline(target_s=8.0, max_steps=None):
    """The reference's MATLAB CPU path restated in C (electricmagneticfield3.m:
    111-319: half drifts with the wall and wedge/z rules, nearest-cell current,
    the field update in two halves, interp2 gather, explicit kick), OpenMP on
    every host core, on the full workload (electrons placed at azimuth 0 with
    v = u / gamma).  Its collisions come once per 1000 pushes
    (electron_transport_field2.m:157-160), outside a sample this short."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    from gasatt.workload import births
    w = WORKLOAD
    threads = os.cpu_count() or 1
    O.lib.orc_set_threads(threads)
    r, z, ur, ut, uz, _ = births(w["photo"], w["e_keV"], w["n_z"] * w["delta"], seed=w["seed"],
                                 Rp=w["n_r"] * w["delta"])
    g = np.sqrt(1 + (ur * ur + ut * ut + uz * uz) / 299792458.0 ** 2)
    m = O.MatlabCpuPath(w["n_r"], w["n_z"], w["delta"], w["dt"])
    m.load(r, np.zeros_like(r), z, ur / g, ut / g, uz / g)
    t0 = time.perf_counter()
    m.step()
    one = time.perf_counter() - t0
    steps = max(1, min(200, int(target_s / max(one, 1e-3))))
    if max_steps:
        steps = min(steps, max_steps)
    n0 = int(m.alive.sum())
    t0 = time.perf_counter()
    for _ in range(steps):
        m.step()
    dt = time.perf_counter() - t0
    n1 = int(m.alive.sum())
    return {"value": 0.5 * (n0 + n1) * steps / dt, "unit": UNIT, "cores": threads,
            "kind": "matlab-path port",
            "sample": f"full workload ({n0:,} electrons), {steps} steps after 1 warm-up step; "
                      f"the reference's MATLAB CPU push/deposit/field step "
                      f"(electricmagneticfield3.m:111-319) restated in C, OpenMP {threads} threads"}


ORACLE_WHAT = ("plain C FP64 restatement of the same corrected step (Boris push, null-collision "
               "MCC, fixed-point deposit, FDTD); the reference's own CPU path is MATLAB, "
               "which is not installed")


def run_reference(args):
    """The reference arm: the CPU oracle (the reference's algorithm restated in
    plain C, OpenMP on every host core) on the full 2,000,000-electron
    workload, K steps after W warm-up steps.  Rank 0 alone runs it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    O, orc = oracle_workload(4_000_000)
    O.lib.orc_set_threads(threads)
    orc.prologue()
    for _ in range(args.warmup):
        orc.step()
    alive0 = int(orc.alive[:orc.n].sum())
    t0 = time.perf_counter()
    for _ in range(args.steps):
        orc.step()
    dt = time.perf_counter() - t0
    alive1 = int(orc.alive[:orc.n].sum())
    value = 0.5 * (alive0 + alive1) * args.steps / dt
    mpath = matlab_path_baseline(max_steps=max(args.steps, 3))
    sample = (f"the full workload ({alive0:,} electrons at the first timed step, 256x1024 grid, FDTD "
              f"every step), {args.steps} steps after {args.warmup} warm-up steps; {ORACLE_WHAT}; "
              f"OpenMP {threads} threads")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded photoionization births; N2 cross-sections from the reference CSVs)",
            "config": {"workload": WORKLOAD_NAME, "precision": "fp64",
                       "global_electrons": alive0, "parallelism": "host threads x%d" % threads},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample, "matlab_path": mpath},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


C3_GRIDS = ((64, 256), (128, 512), (256, 1024), (512, 2048))


def c3_cells(n=48, seed=2):
    """The batched workload: n gas cells with pressure log-uniform in 0.1-10
    Torr, grid drawn from C3_GRIDS at 10 um, photon energy uniform in 2-20 keV,
    photoionizations log-uniform in 1e4-1e6 (seeded)."""
    rng = np.random.default_rng(seed)
    cells = []
    for i in range(n):
        nr, nz = C3_GRIDS[rng.integers(len(C3_GRIDS))]
        cells.append(dict(n_r=int(nr), n_z=int(nz), delta=10e-6, dt=2e-14,
                          torr=float(10 ** rng.uniform(-1, 1)), e_keV=float(rng.uniform(2, 20)),
                          photo=int(round(10 ** rng.uniform(4, 6))), seed=seed * 1000 + i))
    return cells


def c3_batched(precision, device, torch, steps=100, warmup=5, sort_period=30):
    """The 48 C3 gas cells (c3_cells) stepped as one batch in the given form:
    births drawn on the GPU with the workload's laws, `steps` whole steps
    timed with CUDA events after `warmup`.  Returns the rate (mean electrons
    x steps / time), ms per step and the electron count."""
    from gasatt import abi
    from gasatt.dropin import Context
    from gasatt.sim import Batch, Sim
    from gasatt.workload import config
    prec = abi.FP32_SPLIT if precision == "fp32_split" else abi.FP64
    ctx = Context(device)
    ctx.bind_stream()
    sims = []
    for c in c3_cells():
        cfg = config(c["n_r"], c["n_z"], c["delta"], c["dt"], c["torr"], precision=prec,
                     capacity=6 * c["photo"], seed=c["seed"], sort_period=sort_period)
        sim = Sim(cfg, ctx=ctx, device=device)
        sim.birth_photo(c["photo"], c["e_keV"], seed=c["seed"])
        sims.append(sim)
    batch = Batch(sims, sort_period=sort_period)
    stream = torch.cuda.current_stream(device)
    batch.step(warmup)
    torch.cuda.synchronize()
    a0 = sum(s.diag()["n_alive"] for s in sims)
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.step(steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    a1 = sum(s.diag()["n_alive"] for s in sims)
    batch.close()
    for s in sims:
        s.close()
    ctx.close()
    return {"value": 0.5 * (a0 + a1) * steps / (ms / 1e3), "ms_per_step": ms / steps,
            "electrons": int(a1), "steps": steps}


def run_c3(args):
    """Batched instances (one graph launch per step for all cells) against the
    same instances stepped one after another, in the form --precision; births
    drawn on the GPU as in the bench line's batched leg."""
    import torch
    from gasatt import abi
    from gasatt.dropin import Context
    from gasatt.sim import Batch, Sim
    from gasatt.workload import config
    torch.cuda.set_device(0)
    prec = abi.FP32_SPLIT if args.precision == "fp32_split" else abi.FP64
    ctx = Context(0)
    ctx.bind_stream()
    sims = []
    for c in c3_cells(args.c3_cells):
        cfg = config(c["n_r"], c["n_z"], c["delta"], c["dt"], c["torr"], precision=prec,
                     capacity=6 * c["photo"], seed=c["seed"], sort_period=30)
        sim = Sim(cfg, ctx=ctx)
        sim.birth_photo(c["photo"], c["e_keV"], seed=c["seed"])
        sims.append(sim)
    batch = Batch(sims, sort_period=30)
    stream = torch.cuda.current_stream()

    def alive():
        return sum(s.diag()["n_alive"] for s in sims)

    def timed(fn, k):
        torch.cuda.synchronize()
        a0 = alive()
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        return 0.5 * (a0 + alive()) * k / (ms / 1e3), ms / k

    batch.step(args.warmup)
    v_batch, ms_batch = timed(lambda: batch.step(1), args.steps)
    v_seq, ms_seq = timed(lambda: [s.step(1) for s in sims], args.steps)
    line = {"mode": "c3", "metric": METRIC, "unit": UNIT, "instances": len(sims),
            "steps": args.steps, "warmup": args.warmup, "electrons": alive(),
            "batched": {"value": v_batch, "ms_per_step": ms_batch},
            "one_after_another": {"value": v_seq, "ms_per_step": ms_seq},
            "batched_over_one_after_another": v_batch / v_seq,
            "config": {"workload": f"{len(sims)} cells: p log-U(0.1, 10) Torr, grid from "
                       "{64x256, 128x512, 256x1024, 512x2048} at 10 um, dt 2e-14 s, photon "
                       "U(2, 20) keV, photoionizations log-U(1e4, 1e6), seed 2",
                       "precision": args.precision, "sort_period": 30, "l2": "not flushed"}}
    print(json.dumps(line), flush=True)
    batch.close()
    for s in sims:
        s.close()


C5 = dict(n_r=256, n_z=1024, delta=10e-6, dt=2e-14, torr=5.0, photo=2_000_000, e_keV=8.0,
          seed=4, ion_subcycle=50)


def run_c5(args):
    """Electrons plus N2+ ions (one per ionization, Maxwellian at 300 K,
    pushed every 50 steps), 4,000,000 initial electrons at 5 Torr, both
    forms for the whole run: throughput, the growth of both species, exact
    charge conservation, the energy budget, and the FP32 form's drift from
    the FP64 form at the end."""
    import torch
    from gasatt import _lib
    from gasatt.sim import Sim, births, config
    torch.cuda.set_device(0)
    w = C5
    steps, chunk = args.c5_steps, 1000
    parts = births(w["photo"], w["e_keV"], w["n_z"] * w["delta"], seed=w["seed"],
                   Rp=w["n_r"] * w["delta"])
    n0 = len(parts[0])
    out = {}
    for prec, code in (("fp32_split", _lib.FP32_SPLIT), ("fp64", _lib.FP64)):
        cfg = config(w["n_r"], w["n_z"], w["delta"], w["dt"], w["torr"], precision=code,
                     capacity=args.c5_capacity, seed=w["seed"], sort_period=30,
                     ion_capacity=args.c5_capacity, ion_subcycle=w["ion_subcycle"])
        sim = Sim(cfg)
        sim.bind_stream()
        sim.load(*parts)
        stream = torch.cuda.current_stream()
        d_start = sim.diag()
        work, ms_total, trace = 0.0, 0.0, []
        done = 0
        while done < steps:
            k = min(chunk, steps - done)
            a0 = sim.diag()["n_alive"]
            e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            sim.step(k)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            d = sim.diag()
            work += 0.5 * (a0 + d["n_alive"]) * k
            ms_total += ms
            done += k
            trace.append(dict(step=done, electrons=d["n_alive"], ions=d["n_ions"],
                              ms_per_step=ms / k))
        d = sim.diag()
        # per-step cost of the ion sub-cycle: 100 steps with an event pair each
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(100)]
        torch.cuda.synchronize()
        for e0, e1 in evs:
            e0.record(stream); sim.step(1); e1.record(stream)
        torch.cuda.synchronize()
        per = [e0.elapsed_time(e1) for e0, e1 in evs]
        base = steps + 1                              # step index of the first of the 100
        push = [t for i, t in enumerate(per) if (base + i) % w["ion_subcycle"] == 0]
        plain = [t for i, t in enumerate(per) if (base + i) % w["ion_subcycle"] != 0]
        out[prec] = dict(value=work / (ms_total / 1e3), ms_total=ms_total, trace=trace,
                         start=d_start, end=d, fields=sim.fields(),
                         step_ms_plain=float(np.median(plain)),
                         step_ms_with_ion_push=float(np.median(push)) if push else None)
        sim.close()
    f32, f64 = out["fp32_split"], out["fp64"]

    def charge_ok(d):
        return d["n_ions"] - d["n_alive"] == -n0 + d["n_lost_wall"] - d["n_ion_lost_wall"]

    def energy(d):
        ev = 6.241509074e18 * d["field_energy_j"]
        return dict(electron_kinetic_ev=d["kinetic_ev"], ion_kinetic_ev=d["ion_kinetic_ev"],
                    field_energy_j=d["field_energy_j"], collision_loss_ev=d["collision_loss_ev"],
                    wall_loss_ev=d["wall_loss_ev"],
                    sum_ev=d["kinetic_ev"] + d["ion_kinetic_ev"] + ev + d["collision_loss_ev"]
                    + d["wall_loss_ev"])

    ferr = max(float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
               for a, b in zip(f32["fields"], f64["fields"]))
    e32, e64 = f32["end"], f64["end"]
    line = {"mode": "c5", "metric": METRIC, "unit": UNIT, "steps": steps,
            "value": f32["value"], "fp64_value": f64["value"],
            "fp32_over_fp64": f32["value"] / f64["value"],
            "ms_per_step": f32["ms_total"] / steps, "fp64_ms_per_step": f64["ms_total"] / steps,
            "step_ms_plain": f32["step_ms_plain"], "step_ms_with_ion_push": f32["step_ms_with_ion_push"],
            "electrons": {"initial": n0, "final_fp32": e32["n_alive"], "final_fp64": e64["n_alive"]},
            "ions": {"final_fp32": e32["n_ions"], "final_fp64": e64["n_ions"],
                     "lost_wall_fp32": e32["n_ion_lost_wall"], "overflow": bool((e32["status_flags"] | e64["status_flags"]) & 6)},
            "ionizations": {"fp32": e32["n_ionizations"], "fp64": e64["n_ionizations"],
                            "rel_diff": (e32["n_ionizations"] - e64["n_ionizations"]) / max(e64["n_ionizations"], 1)},
            "charge_conserved": {"fp32": charge_ok(e32), "fp64": charge_ok(e64),
                                 "net_charge_c_fp64": e64["net_charge_c"],
                                 "identity": "ions - electrons = -N0 + electrons lost - ions lost"},
            "energy_fp64": {"start": energy(f64["start"]), "end": energy(e64),
                            "sum_rel_change": energy(e64)["sum_ev"] / energy(f64["start"])["sum_ev"] - 1,
                            "note": "sum = electron + ion kinetic + field + given to the gas "
                                    "+ carried out by the electrons and ions absorbed at the wall; "
                                    "newborn ions add their thermal energy"},
            "drift_fp32_vs_fp64": {"field_rel_err_l2": ferr,
                                   "electron_kinetic_rel": e32["kinetic_ev"] / e64["kinetic_ev"] - 1,
                                   "ion_kinetic_rel": (e32["ion_kinetic_ev"] / e64["ion_kinetic_ev"] - 1)
                                   if e64["ion_kinetic_ev"] else None,
                                   "ions_rel": (e32["n_ions"] - e64["n_ions"]) / max(e64["n_ions"], 1)},
            "trace_fp32": f32["trace"][::max(1, len(f32["trace"]) // 10)],
            "config": {"workload": "4,000,000 e- from 2,000,000 photoionizations at 8 keV, N2 5 Torr "
                       "300 K, 256x1024 cells at 10 um, dt 2e-14 s, one N2+ ion (28 amu) per "
                       "ionization, Maxwellian 300 K, ion push every 50 steps, seed 4",
                       "capacity": args.c5_capacity, "sort_period": 30, "l2": "not flushed",
                       "timed": "whole steps incl. ion pushes, 1000-step chunks"}}
    print(json.dumps(line), flush=True)


C1 = dict(n_r=64, n_z=256, delta=10e-6, dt=2e-14, torr=1.0, photo=10_000, e_keV=8.0, seed=0)


def run_c1(args):
    """The reference's CPU-runnable case at full size: 20,000 electrons, 64 x
    256 cells at 10 um, 1 Torr, dt 2e-14 s, 500 steps.  The FP64 form against
    the CPU oracle of the same step (same random streams): agreement and
    both rates; the FP32 form's rate beside them."""
    import torch
    from gasatt import _lib
    from gasatt.sim import Sim, births, config
    from gasatt.tables import N2Tables
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    torch.cuda.set_device(0)
    w = C1
    steps = args.c1_steps
    parts = births(w["photo"], w["e_keV"], w["n_z"] * w["delta"], seed=w["seed"],
                   Rp=w["n_r"] * w["delta"])
    out = {}
    for prec, code in (("fp64", _lib.FP64), ("fp32_split", _lib.FP32_SPLIT)):
        cfg = config(w["n_r"], w["n_z"], w["delta"], w["dt"], w["torr"], precision=code,
                     capacity=200_000, seed=w["seed"], sort_period=30)
        sim = Sim(cfg)
        sim.bind_stream()
        sim.load(*parts)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        sim.step(steps)
        e1.record(); e1.synchronize()
        d = sim.diag()
        out[prec] = dict(ms=e0.elapsed_time(e1), diag=d, fields=sim.fields(), read=sim.read(),
                         cfg=cfg)
        sim.close()
    cfg = out["fp64"]["cfg"]
    O.lib.orc_set_threads(os.cpu_count() or 1)
    orc = O.Sim(cfg, N2Tables(), cap=cfg.capacity)
    orc.load(*parts)
    t0 = time.perf_counter()
    orc.prologue()
    for _ in range(steps):
        orc.step()
    cpu_s = time.perf_counter() - t0
    g = out["fp64"]
    ion, ela, exc, nul, lost, ovf = (int(x) for x in orc.counters)
    ferr = max(float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
               for a, b in zip(g["fields"], (orc.Er, orc.Ez, orc.H)))
    r, z, ur, ut, uz, ids, alive = orc.state_rz()
    a = alive.astype(bool)
    gr = g["read"]
    ga = gr["r"] >= 0
    same_ids = set(gr["id"][ga].tolist()) == set(ids[a].tolist())
    uerr = None
    if same_ids:
        o1, o2 = np.argsort(ids[a]), np.argsort(gr["id"][ga])
        umag = np.sqrt(ur[a] ** 2 + ut[a] ** 2 + uz[a] ** 2)[o1]
        du = np.sqrt((gr["ur"][ga][o2] - ur[a][o1]) ** 2 + (gr["ut"][ga][o2] - ut[a][o1]) ** 2
                     + (gr["uz"][ga][o2] - uz[a][o1]) ** 2)
        uerr = float((du / umag).max())
    n_mean = len(parts[0])
    line = {"mode": "c1", "metric": METRIC, "unit": UNIT, "steps": steps,
            "gpu_fp64": {"value": n_mean * steps / (g["ms"] / 1e3), "ms": g["ms"]},
            "gpu_fp32_split": {"value": n_mean * steps / (out["fp32_split"]["ms"] / 1e3),
                               "ms": out["fp32_split"]["ms"]},
            "cpu_oracle": {"value": n_mean * steps / cpu_s, "s": cpu_s,
                           "cores": os.cpu_count() or 1, "kind": "port"},
            "fp64_vs_oracle": {"counts_gpu": [g["diag"][k] for k in ("n_ionizations", "n_elastic",
                                                                   "n_excitation", "n_null",
                                                                   "n_lost_wall")],
                               "counts_oracle": [ion, ela, exc, nul, lost],
                               "same_population": same_ids,
                               "max_rel_u_err": uerr, "field_rel_err_l2": ferr},
            "fp32_vs_fp64_ionizations": [out["fp32_split"]["diag"]["n_ionizations"],
                                         g["diag"]["n_ionizations"]],
            "config": {"workload": "20,000 e- from 10,000 photoionizations at 8 keV, N2 1 Torr "
                       "300 K, 64x256 cells at 10 um, dt 2e-14 s, seed 0",
                       "rates": "initial electrons x steps / time (one call of all steps)"}}
    print(json.dumps(line), flush=True)


C4 = dict(n_r=1024, n_z=4096, delta=5e-6, dt=1e-14, torr=10.0, photo=8_000_000, e_keV=12.0,
          seed=3, capacity=64 << 20)


def run_c4(args):
    """The single large cascade: 16,000,000 electrons from 8,000,000
    photoionizations at 12 keV (drawn on the GPU), N2 at 10 Torr, 1024 x 4096
    cells at 5 um, capacity 64M, FP32 split form, sort period 30; the steps
    are timed in chunks with CUDA events (whole steps, sorts included)."""
    import torch
    from gasatt import _lib
    from gasatt.sim import Sim, config
    torch.cuda.set_device(0)
    w = C4
    steps, chunk = args.c4_steps, 500
    cfg = config(w["n_r"], w["n_z"], w["delta"], w["dt"], w["torr"], precision=_lib.FP32_SPLIT,
                 capacity=w["capacity"], seed=w["seed"], sort_period=30)
    sim = Sim(cfg)
    sim.bind_stream()
    sim.birth_photo(w["photo"], w["e_keV"], seed=w["seed"])
    stream = torch.cuda.current_stream()
    d0 = sim.diag()
    work, ms_total, trace, done = 0.0, 0.0, [], 0
    while done < steps:
        k = min(chunk, steps - done)
        a0 = sim.diag()["n_alive"]
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        sim.step(k)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        d = sim.diag()
        work += 0.5 * (a0 + d["n_alive"]) * k
        ms_total += ms
        done += k
        trace.append(dict(step=done, electrons=d["n_alive"], ms_per_step=ms / k))
    d = sim.diag()
    line = {"mode": "c4", "metric": METRIC, "unit": UNIT, "steps": steps,
            "value": work / (ms_total / 1e3), "ms_per_step": ms_total / steps,
            "electrons": {"initial": d0["n_alive"], "final": d["n_alive"]},
            "ionizations": d["n_ionizations"], "lost_wall": d["n_lost_wall"],
            "capacity_overflow": bool(d["status_flags"] & 2),
            "energy_ev": {"start": d0["kinetic_ev"],
                          "end_sum": d["kinetic_ev"] + d["collision_loss_ev"] + d["wall_loss_ev"]
                          + 6.241509074e18 * d["field_energy_j"]},
            "trace": trace[::max(1, len(trace) // 10)],
            "config": {"workload": "16,000,000 e- from 8,000,000 photoionizations at 12 keV (GPU "
                       "births), N2 10 Torr 300 K, 1024x4096 cells at 5 um, dt 1e-14 s, seed 3",
                       "precision": "fp32_split", "capacity": w["capacity"], "sort_period": 30,
                       "l2": "not flushed", "timed": "whole steps, 500-step chunks"}}
    print(json.dumps(line), flush=True)
    sim.close()


def c5_profile_sim(precision, torch):
    """The C5 cell with its ions already grown: the 4,000,000 birth electrons
    plus 4,000,000 ions at their positions (Maxwellian 300 K), so that the
    first ion push (step 50) handles a grown ion population."""
    from gasatt import _lib
    from gasatt.sim import Sim, births, config
    w = C5
    code = _lib.FP32_SPLIT if precision == "fp32_split" else _lib.FP64
    cfg = config(w["n_r"], w["n_z"], w["delta"], w["dt"], w["torr"], precision=code,
                 capacity=16_000_000, seed=w["seed"], sort_period=30, ion_capacity=16_000_000,
                 ion_subcycle=w["ion_subcycle"])
    parts = births(w["photo"], w["e_keV"], w["n_z"] * w["delta"], seed=w["seed"],
                   Rp=w["n_r"] * w["delta"])
    sim = Sim(cfg)
    sim.bind_stream()
    sim.load(*parts)
    n = len(parts[0])
    rng = np.random.default_rng(w["seed"])
    sig = np.sqrt(cfg.kb * cfg.gas_temperature / cfg.m_ion)
    sim.load_ions(parts[0], parts[1], *(rng.normal(0, sig, n) for _ in range(3)),
                  np.arange(n, dtype=np.uint64))
    return sim


def run_profile(args):
    """The step loop alone (warm-up then timed steps, no flush/e2e/baseline),
    for kernel profilers; --workload c5 adds the ion species."""
    import torch
    torch.cuda.set_device(0)
    if args.workload == "c5":
        sim = c5_profile_sim(args.precision, torch)
    else:
        sim, _ = make_sim(args.precision, 0, 0, torch)
    sim.step(args.warmup + args.steps)
    torch.cuda.synchronize()
    d = sim.diag()
    print(json.dumps({"mode": "profile", "precision": args.precision, "steps": args.steps,
                      "warmup": args.warmup, "alive": d["n_alive"],
                      "ionizations": d["n_ionizations"], "launches": sim.ctx.launches}))
    sim.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="bench", choices=["bench", "profile", "c1", "c3", "c4", "c5"],
                    help="profile: only the step loop of one precision (for ncu); "
                         "c3: 48 batched gas cells; c4: the 16M-electron cascade; "
                         "c5: electrons plus ions, long run")
    ap.add_argument("--accuracy-steps", type=int, default=2000,
                    help="length of the FP32-vs-FP64 accuracy runs (the workload's 2000 steps)")
    ap.add_argument("--c4-steps", type=int, default=5000)
    ap.add_argument("--c1-steps", type=int, default=500)
    ap.add_argument("--c5-steps", type=int, default=20_000)
    ap.add_argument("--workload", default="c2", choices=["c2", "c5"],
                    help="workload of --mode profile")
    ap.add_argument("--c5-capacity", type=int, default=80_000_000)
    ap.add_argument("--precision", default="fp32_split", choices=["fp32_split", "fp64"])
    ap.add_argument("--c3-cells", type=int, default=48,
                    help="--mode c3: the first N cells of the 48 (a smaller case for profiling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.mode == "profile":
        run_profile(args)
    elif args.mode == "c3":
        if not 1 <= args.c3_cells <= 48:
            ap.error("--c3-cells: 1 to 48")
        run_c3(args)
    elif args.mode == "c1":
        run_c1(args)
    elif args.mode == "c4":
        run_c4(args)
    elif args.mode == "c5":
        run_c5(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
