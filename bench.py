#!/usr/bin/env python
"""Benchmark of the B200 engine on the 1M-atom NVE step (one JSON line on rank 0).

Workload: N = 4*64^3 = 1 048 576 atoms, FCC at rho = 0.8442, T = 1.0,
rc = 2.5, dt = 0.005, seeded Maxwell-Boltzmann velocities (the library's own
engine::InitialCondition).  A step is one velocity-Verlet step of the whole
system (kick, drift, wrap, forces, kick) with its ThermodynamicMeasurement.

  value        FP64 drop-in path, atom-steps/s, state resident in HBM, CUDA
               events on the engine's stream, max over ranks
  mixed        same for the mixed-precision path (FP32 pair arithmetic)
  drift        |dE/E| of both paths over --drift-steps steps
  e2e          FP64 path through the C ABI from pinned host buffers: upload the
               SystemState, --steps steps with every per-step record read back
               to the host, download the SystemState
  roofline     the pair kernel (the dominant one) against the measured FP64 FMA peak
  cpu_baseline the CPU oracle (the reference's algorithm, its release flags) on
               the host cores, one 1M-atom system per thread

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""

import argparse
import ctypes
import json
import math
import os
import pathlib
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "lennard-jonesium_b200"))

METRIC = "atom-steps/s, 1M-atom LJ: FP32-pair vs FP64 on B200 at equal energy drift"
UNIT = "atom-steps/s"
WORK = dict(n_cells=64, T=1.0, rho=0.8442, rc=2.5, dt=0.005, seed=5489)
N_ATOMS = 4 * WORK["n_cells"] ** 3  # --cells changes it (profiling captures of a smaller case)
HBM_PEAK = None


def workload_config(extra=None):
    c = {"workload": f"FCC LJ fluid, N={N_ATOMS} (4*{WORK['n_cells']}^3), rho=0.8442, T=1.0, rc=2.5, "
                     "dt=0.005, seeded MB velocities, spline-truncated LJ, NVE velocity Verlet",
         "atoms": N_ATOMS, "cutoff": WORK["rc"], "time_delta": WORK["dt"],
         "l2": "per-step working set (state + neighbour list, > 400 MB) exceeds the 126 MB L2",
         "parallelism": "replicas only (one independent system per GPU)"}
    if extra:
        c.update(extra)
    return c


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "fallback": True}


def alg_flops_per_atom_step(N, L, rc, rho):
    """Algorithmic work of the reference's half-shell algorithm (candidate tests
    of the 27-cell stencil counted once per pair, kept pairs likewise):
    F = 9 C + 30 P, C = (27 rho a^3 - 1) / 2 candidate tests, P = (2 pi / 3) rho rc^3 pairs."""
    n_c = math.floor(L / rc)
    a = L / n_c
    C = (27 * rho * a ** 3 - 1) / 2
    P = (2 * math.pi / 3) * rho * rc ** 3
    return 9 * C + 30 * P, C, P


ALG_BYTES_PER_ATOM_STEP = 216.0  # each FP64 state vector read once and written once


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=__import__("torch").device("cuda", local))
    return ws, rank, local


def barrier(ws, device="cuda"):
    import torch
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    if device == "cuda":
        torch.cuda.synchronize()


def reduce_max(ws, x, device="cuda"):
    """The slowest rank's time: every rank runs its own system, the job takes as
    long as the last one."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(ws, atoms_per_rank, steps, sec_max):
    """Whole-job atom-steps/s of ws independent replicas timed as the slowest."""
    return ws * atoms_per_rank * steps / sec_max


def cpu_baseline(replicas, steps, warm=1):
    """The CPU oracle (reference algorithm, -O3 -ffast-math), one system per thread."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import ljref
    sec = ljref.bench(N_ATOMS, WORK["T"], WORK["rho"], WORK["seed"], WORK["rc"], WORK["dt"], warm, steps,
                      replicas, fast=True)
    return replicas * N_ATOMS * steps / sec, sec


def cpu_model():
    try:
        for l in open("/proc/cpuinfo"):
            if l.startswith("model name"):
                return l.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args, ws, rank):
    """--impl reference: the reference's algorithm on the host cores (the CPU oracle
    built with the reference's release flags; the reference itself needs Eigen and
    Boost, which this image lacks).  Rank 0 only."""
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import ljref
    cores = ljref.cpu_count()
    replicas = max(1, min(cores, 64))
    # every requested step up to 100 (each ~0.6 s of all host cores at 1M atoms
    # per system), so that the run stays within a few minutes
    steps = max(1, min(args.steps, 100))
    warm = max(1, min(args.warmup, 5))
    value, sec = cpu_baseline(replicas, steps, warm)
    sample = (f"{replicas} concurrent 1M-atom systems (one per thread, SimulationPool-style), "
              f"{warm} warm-up + {steps} timed steps each; CPU: {cpu_model()}")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "steps_requested": args.steps, "warmup": warm, "ms_per_step": 1e3 * sec / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config({"implementation": "CPU oracle restatement of the reference, "
                                                         "g++ -O3 -march=x86-64-v3 -ffast-math"}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": replicas, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


GRAPH_STEPS = 32     # steps per launch of the engine's long step graph
MIN_TIMED_STEPS = 320
PHASE_STEPS = 256    # steps of the per-phase timing pass behind the roofline's kernel time


def timed_step_count(requested):
    """Steps actually timed: the request rounded up to whole 32-step graph launches,
    and at least 320 steps, so that the timed region runs the same launches as a
    long run does (a shorter request would time the 8-step remainder graph and
    direct launches instead)."""
    k = max(int(requested), MIN_TIMED_STEPS)
    return -(-k // GRAPH_STEPS) * GRAPH_STEPS


def timed_steps(torch, g, K, ws):
    """K steps on the engine's stream bracketed by CUDA events (barrier + sync on both sides)."""
    stream = torch.cuda.ExternalStream(g.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(ws)
    e0.record(stream)
    g.step_async(K)
    e1.record(stream)
    g.synchronize()
    barrier(ws)
    return e0.elapsed_time(e1) / 1e3


def energy_drift(g, steps, equilibration=1000):
    """|dE/E| of the total energy over `steps` steps after `equilibration` steps
    (the FCC start melts in the first few hundred): the endpoint difference and
    a least-squares slope times the window length, both over |E| at its start."""
    import numpy as np
    g.step(equilibration, record=False)
    te = g.step(steps)[:, 3]
    E0 = abs(te[0])
    slope = np.polyfit(np.arange(steps, dtype=np.float64), te, 1)[0]
    return {"equilibration_steps": equilibration, "steps": steps,
            "endpoint_abs_rel": float(abs(te[-1] - te[0]) / E0),
            "fit_abs_rel": float(abs(slope) * steps / E0),
            "max_rel_excursion": float(abs(te - te[0]).max() / E0)}


def e2e_run(torch, g, x, v, K):
    """Public C-ABI path from pinned host buffers, copies inside the timed region."""
    from lennardjonesium import _native as nat
    N = g.N
    pin = [torch.zeros((N, 4), dtype=torch.float64, pin_memory=True) for _ in range(8)]
    pin[0][:, :3] = torch.from_numpy(x[:, :3])
    pin[1][:, :3] = torch.from_numpy(v[:, :3])
    rec = torch.zeros((K, 7), dtype=torch.float64, pin_memory=True)
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    L = nat.lib()
    stream = torch.cuda.ExternalStream(g.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    nat.check(L.lj_gpu_upload_state(g._ctx, P(pin[0]), P(pin[1]), P(pin[2]), P(pin[3]), 4, 0.0, 0.0, 0.0), g._ctx)
    nat.check(L.lj_gpu_step(g._ctx, K, P(rec)), g._ctx)
    t, pe, w = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    nat.check(L.lj_gpu_download_state(g._ctx, P(pin[4]), P(pin[5]), P(pin[6]), P(pin[7]), 4, ctypes.byref(t),
                                      ctypes.byref(pe), ctypes.byref(w)), g._ctx)
    e1.record(stream)
    e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    state_bytes = 4 * 32 * N
    return {"value": N * K / sec, "unit": UNIT, "h2d_bytes_per_step": state_bytes / K,
            "d2h_bytes_per_step": (state_bytes + 56 * K) / K,
            "steps": K,
            "path": f"lj_gpu_upload_state + lj_gpu_step(K = {K}, the timed step count; every record to the host) "
                    "+ lj_gpu_download_state, pinned host SystemState (4 x N doubles per vector); the state "
                    "upload and download are amortised over the K steps"}


def run_ours(args, ws, rank, local):
    import torch
    from lennardjonesium import GpuSystem, initial_condition, autotune
    from lennardjonesium import _native as nat

    torch.cuda.set_device(local)
    x, v, L = initial_condition(N_ATOMS, WORK["T"], WORK["rho"], WORK["seed"] + rank)
    peaks = measured_peaks()
    f64 = ctypes.c_double()
    f32 = ctypes.c_double()
    nat.check(nat.lib().lj_gpu_fma_peaks(local, ctypes.byref(f64), ctypes.byref(f32)))
    F_alg, C, P = alg_flops_per_atom_step(N_ATOMS, L, WORK["rc"], WORK["rho"])

    K = timed_step_count(args.steps)
    results = {}
    tuning = {}
    for prec in ("fp64", "mixed"):
        extra = {"mixed_per_pair": True} if prec == "mixed" and args.mixed_per_pair else {}
        if args.autotune:
            kw, tuned_ms = autotune(N_ATOMS, L, x, v, steps=256, cutoff=WORK["rc"], dt=WORK["dt"], precision=prec,
                                    device=local, **extra)
            tuning[prec] = dict(kw, tuned_ms_per_step=tuned_ms)
        else:
            kw = dict({"skin": args.skin, "force_block": args.block}, **extra)
        g = GpuSystem(N_ATOMS, L, cutoff=WORK["rc"], dt=WORK["dt"], precision=prec, device=local, **kw)
        g.upload(x, v=v)
        g.step_async(args.warmup)
        g.synchronize()
        launches0 = g.stats()["kernel_launches"]
        with ClockSampler(local) as clk:
            sec = timed_steps(torch, g, K, ws)
        launches = g.stats()["kernel_launches"] - launches0
        sec = reduce_max(ws, sec)
        ph = g.step_timed(PHASE_STEPS)
        st = g.stats()
        results[prec] = dict(sec=sec, phases=ph, clocks=clk.summary(), launches=launches, stats=st, g=g)

    # energy drift at equal length for both paths (fresh systems from the same state)
    drift = {}
    if args.drift_steps > 0:
        for prec in ("fp64", "mixed"):
            g = results[prec]["g"]
            g.upload(x, v=v)
            drift[prec] = energy_drift(g, args.drift_steps)

    e2e = e2e_run(torch, results["fp64"]["g"], x, v, K)

    r64 = results["fp64"]
    value = job_throughput(ws, N_ATOMS, K, r64["sec"])
    ph = r64["phases"]
    t_force = ph["force_ms"] / ph["steps"] / 1e3
    flops = F_alg * N_ATOMS
    achieved = flops / t_force / 1e12
    traffic = None
    tfile = ROOT / "profiles" / "force_fp64_traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get("bytes_per_launch_full_size")
    roofline = {"bound": "fp64", "achieved": achieved, "peak": f64.value, "unit": "TFLOP/s",
                "frac": achieved / f64.value, "traffic": traffic,
                "kernel": "force_fp64_kernel (pair force + second kick + partial sums)",
                "peak_source": "measured: project DFMA microbenchmark on this GPU (lj_gpu_fma_peaks)",
                "alg_flops_per_atom_step": F_alg, "candidates_per_atom": C, "pairs_per_atom": P,
                "kernel_ms": t_force * 1e3,
                "kernel_time_source": f"CUDA events around the pair kernel in a per-phase pass of {PHASE_STEPS} steps",
                "hbm_frac_of_measured": (ALG_BYTES_PER_ATOM_STEP * N_ATOMS / (r64["sec"] / K)) / 1e9
                / peaks.get("hbm_gbs", 6650.0)}
    rm = results["mixed"]
    phm = rm["phases"]
    t_force_m = phm["force_ms"] / phm["steps"] / 1e3
    mixed = {"value": job_throughput(ws, N_ATOMS, K, rm["sec"]), "unit": UNIT, "ms_per_step": 1e3 * rm["sec"] / K,
             "speedup_vs_fp64": r64["sec"] / rm["sec"],
             "roofline": {"bound": "fp32", "achieved": flops / t_force_m / 1e12, "peak": f32.value,
                          "unit": "TFLOP/s", "frac": flops / t_force_m / 1e12 / f32.value,
                          "kernel_ms": t_force_m * 1e3},
             "phases_ms_per_step": {k: phm[k] / phm["steps"] for k in ("kick_drift_ms", "rebuild_ms", "force_ms",
                                                                        "finalize_ms")}}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "steps_requested": args.steps,
            "warmup": args.warmup,
            "ms_per_step": 1e3 * r64["sec"] / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config({"precision": "fp64 (drop-in); mixed reported under 'mixed'",
                                       "mixed_accumulation": "every pair in FP64" if args.mixed_per_pair
                                       else "FP32 sums of 8 pairs into FP64"}),
            "clocks": r64["clocks"], "e2e": e2e, "gpu_launches": r64["launches"], "roofline": roofline,
            "mixed": mixed, "drift": drift,
            "phases_ms_per_step": {k: ph[k] / ph["steps"] for k in ("kick_drift_ms", "rebuild_ms", "force_ms",
                                                                     "finalize_ms")},
            "list_builds_per_step": ph["rebuilds"] / ph["steps"],
            "tuning": tuning or {"fixed": True, "skin": 0.3 if args.skin is None else args.skin,
                                 "force_block": args.block or 128},
            "fma_peaks_tflops": {"fp64": f64.value, "fp32": f32.value}}
    if ws == 1 and rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import ljref
        cores = max(1, min(ljref.cpu_count(), 64))
        cval, csec = cpu_baseline(cores, 2, 1)
        line["cpu_baseline"] = {"value": cval, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": f"{cores} concurrent 1M-atom systems, one per thread, 1 warm-up + 2 "
                                          f"timed steps each (CPU oracle, reference release flags); CPU: {cpu_model()}"}
    for r in results.values():
        r["g"].close()
    if rank == 0:
        print(json.dumps(line), flush=True)


SWEEP = dict(systems=64, T=(0.5, 2.0, 8), rho=(0.05, 1.0, 8), n=(5, 20), rc=2.5, dt=0.005, eq=2000, prod=5000,
             chunk=200, seed=2024, tol=0.05)


def sweep_systems():
    """The sweep workload: an 8 x 8 grid of rho in [0.05, 1.0] and T in [0.5, 2.0]
    (the reference's linspace, T outer), N = 4 n^3 with n ~ U{5..20} from a fixed seed."""
    import numpy as np
    from lennardjonesium import initial_condition
    from lennardjonesium.tools import linspace
    rng = np.random.default_rng(SWEEP["seed"])
    ns = rng.integers(SWEEP["n"][0], SWEEP["n"][1] + 1, size=SWEEP["systems"])
    out = []
    for k, (T, rho) in enumerate((t, d) for t in linspace(*SWEEP["T"]) for d in linspace(*SWEEP["rho"])):
        N = 4 * int(ns[k]) ** 3
        x, v, L = initial_condition(N, T, rho, SWEEP["seed"] + k)
        out.append(dict(N=N, T=T, rho=rho, x=x, v=v, L=L))
    return out


def sweep_files_arm():
    """The same 8 x 8 (T, rho) grid through the drop-in API: lennardjonesium.run_sweep
    with the reference's control protocol (equilibration with temperature
    rescales, then 10 observations 500 steps apart) writing every run's four
    files, N = 4000 per run (the sweep configuration has one particle count).
    Wall clock of the whole call."""
    import tempfile
    import lennardjonesium as lj
    sc = lj.SweepConfiguration()
    sc.system.temperature_start, sc.system.temperature_stop, sc.system.temperature_steps = 0.5, 2.0, 8
    sc.system.density_start, sc.system.density_stop, sc.system.density_steps = 0.05, 1.0, 8
    sc.system.particle_count = 4000
    sc.equilibration.adjustment_interval, sc.equilibration.steady_state_time = 200, 2000
    sc.equilibration.timeout = 10000
    sc.observation.observation_interval, sc.observation.observation_count = 500, 10
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        res = lj.run_sweep(pathlib.Path(d) / "sweep.ini", echo_status=False, random_seed=2024,
                           sweep_config_object=sc, batched=True)
        sec = time.perf_counter() - t0
    runs = res.completed + res.equilibration_aborted + res.observation_aborted
    steps = sum(r.event_data.total_time_steps for r in runs)
    return {"value": 4000 * steps / sec, "unit": "atom-steps/s", "seconds": sec, "runs": len(runs),
            "completed": len(res.completed), "total_steps": steps,
            "config": "T 0.5..2.0 x rho 0.05..1.0 (8 x 8), N=4000, eq: rescale check every 200 steps, steady "
                      "2000, timeout 10000; obs: 10 x 500 steps; four files per run"}


def batch_window_stats(lib, b, systems, recs, reps=50):
    """ThermodynamicAnalyzer over each system's last len(recs) records: all systems
    in one device call (lj_batch_window_stats, from the batch's record ring)
    against the host restatement over the same records, which the host must
    first hold (recs: the last chunk's records, steps x systems x 7)."""
    import numpy as np
    from lennardjonesium import _native as nat
    from lennardjonesium import window_stats_host
    W, nsys = recs.shape[0], recs.shape[1]
    dens = np.array([sy["N"] / sy["L"] ** 3 for sy in systems])
    obs = (nat.Observation * nsys)()
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    nat.check(lib.lj_batch_window_stats(b, W, P(dens), obs))
    t0 = time.perf_counter()
    for _ in range(reps):
        nat.check(lib.lj_batch_window_stats(b, W, P(dens), obs))
    t_dev = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        host = [window_stats_host(recs[:, s, :], systems[s]["N"], dens[s]) for s in range(nsys)]
    t_host = (time.perf_counter() - t0) / reps
    rel = max(abs(getattr(obs[s], f) - host[s][f]) / max(abs(host[s][f]), 1e-300)
              for s in range(nsys) for f, _ in obs[s]._fields_ if f != "density")
    return {"systems": nsys, "records": W, "device_call_us": 1e6 * t_dev, "host_restatement_us": 1e6 * t_host,
            "max_rel_diff": rel,
            "note": "wall clock per call; the device call includes its synchronisation and the copy of the results"}


def run_sweep_bench(args):
    """Batched engine vs the same 64 systems run one after another on the GPU: identical
    protocol in both arms (chunks of 200 steps; during the first 2000 steps a system
    whose mean T over the chunk is off by >= 5% is rescaled to its target)."""
    import numpy as np
    import torch
    from lennardjonesium import GpuSystem
    from lennardjonesium import _native as nat
    systems = sweep_systems()
    nsys = len(systems)
    total_steps = SWEEP["eq"] + SWEEP["prod"]
    chunk = SWEEP["chunk"]
    lib = nat.lib()
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)

    table = (nat.BatchSystem * nsys)()
    for s, sy in enumerate(systems):
        table[s].particle_count = sy["N"]
        for k in range(3):
            table[s].box[k] = sy["L"]
        table[s].time_delta = SWEEP["dt"]
        table[s].skin = -1.0
    # batch autotuner (skin x pair-kernel block size) on the sweep's own state; both
    # arms then run with the chosen parameters, so their records stay comparable bit for bit
    tune = nat.BatchTuning()
    xs = np.concatenate([sy["x"] for sy in systems])
    vs = np.concatenate([sy["v"] for sy in systems])
    nat.check(lib.lj_batch_autotune(table, nsys, SWEEP["rc"], 0, P(xs), P(vs), 4, 200, ctypes.byref(tune)))
    for s in range(nsys):
        table[s].skin = tune.skin

    # batched: one chunk-graph launch per 200-step chunk
    b = ctypes.c_void_p()
    nat.check(lib.lj_batch_create(table, nsys, SWEEP["rc"], 0, ctypes.byref(b)))
    nat.check(lib.lj_batch_set_force_block(b, tune.force_block))
    nat.check(lib.lj_batch_set_list_tile(b, tune.list_cells_per_block))
    for s, sy in enumerate(systems):
        nat.check(lib.lj_batch_upload_system(b, s, P(sy["x"]), P(sy["v"]), 4))
    recs = np.zeros((chunk, nsys, 7))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for step in range(0, total_steps, chunk):
        nat.check(lib.lj_batch_step(b, chunk, P(recs)))
        if step + chunk <= SWEEP["eq"]:
            for s, sy in enumerate(systems):
                if abs(recs[:, s, 5].mean() / sy["T"] - 1) >= SWEEP["tol"]:
                    nat.check(lib.lj_batch_set_temperature(b, s, sy["T"], None))
    torch.cuda.synchronize()
    t_batched = time.perf_counter() - t0
    final_batched = recs[-1].copy()
    wstats = batch_window_stats(lib, b, systems, recs)
    lib.lj_batch_destroy(b)

    # sequential, one context at a time
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    final_seq = np.zeros((nsys, 7))
    for s, sy in enumerate(systems):
        with GpuSystem(sy["N"], sy["L"], cutoff=SWEEP["rc"], dt=SWEEP["dt"], skin=tune.skin,
                       force_block=tune.force_block) as g:
            g.upload(sy["x"], v=sy["v"])
            for step in range(0, total_steps, chunk):
                r = g.step(chunk)
                if step + chunk <= SWEEP["eq"] and abs(r[:, 5].mean() / sy["T"] - 1) >= SWEEP["tol"]:
                    g.set_temperature(sy["T"])
            final_seq[s] = r[-1]
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    atoms = sum(sy["N"] for sy in systems)
    files = sweep_files_arm()
    line = {"metric": "batched 64-system (T, rho) sweep vs sequential GPU runs", "unit": "atom-steps/s",
            "value": atoms * total_steps / t_batched, "sequential": atoms * total_steps / t_seq,
            "speedup": t_seq / t_batched, "seconds_batched": t_batched, "seconds_sequential": t_seq,
            "systems": nsys, "atoms": atoms, "steps": total_steps,
            "identical_final_records": bool(np.array_equal(final_batched, final_seq)),
            "tuning": {"skin": tune.skin, "force_block": tune.force_block,
                       "list_cells_per_block": tune.list_cells_per_block,
                       "tuned_ms_per_step": tune.ms_per_step, "source": "lj_batch_autotune, 200 steps per candidate"},
            "run_sweep_files": files,
            "window_stats": wstats,
            "config": {"workload": "8x8 grid rho in [0.05,1.0] x T in [0.5,2.0], N=4n^3, n~U{5..20} (seed 2024), "
                                   "rc=2.5, dt=0.005, 2000 equilibration + 5000 production steps, FP64",
                       "timing": "wall clock around synchronised device work (host decisions included)"}}
    print(json.dumps(line), flush=True)


LONG = dict(n_cells=100, T=0.9, rho=0.8, rc=2.5, dt=0.004, seed=2718, rdf_every=100, rdf_bins=200, rdf_rmax=4.0)


def run_long_bench(args):
    """4M-atom (4 * 100^3 FCC) run at rho = 0.8, T = 0.9, dt = 0.004: the mixed path
    with an RDF histogram (200 bins to 4 sigma) every 100 steps, and the same run on
    the FP64 path for the drift comparison.  Device time of both runs (steps and RDF
    sampling) by CUDA events on each engine's stream."""
    import numpy as np
    import torch
    from lennardjonesium import GpuSystem, initial_condition
    N = 4 * LONG["n_cells"] ** 3
    x, v, L = initial_condition(N, LONG["T"], LONG["rho"], LONG["seed"])
    steps = max(LONG["rdf_every"], args.long_steps - args.long_steps % LONG["rdf_every"])
    out = {}
    for prec in ("mixed", "fp64"):
        with GpuSystem(N, L, cutoff=LONG["rc"], dt=LONG["dt"], precision=prec) as g:
            g.upload(x, v=v)
            g.step(8)  # graph capture and first neighbour list outside the timed region
            g.upload(x, v=v)
            te = []
            g.rdf_reset()
            g.rdf_accumulate(LONG["rdf_bins"], LONG["rdf_rmax"])  # sizes the RDF scratch outside the timed region
            g.rdf_reset()
            stream = torch.cuda.ExternalStream(g.stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(steps // LONG["rdf_every"]):
                te.append(g.step(LONG["rdf_every"])[:, 3])
                g.rdf_accumulate(LONG["rdf_bins"], LONG["rdf_rmax"])  # device-side sum, no sync
            e1.record(stream)
            e1.synchronize()
            sec = e0.elapsed_time(e1) / 1e3
            hist, samples = g.rdf_read()
            assert samples == steps // LONG["rdf_every"]
            hist = hist.astype(np.float64)
            te = np.concatenate(te)
            w = 200
            out[prec] = {"ms_per_step": 1e3 * sec / steps, "atom_steps_per_s": N * steps / sec,
                         "abs_rel_drift": float(abs(te[-w:].mean() - te[:w].mean()) / abs(te[:w].mean())),
                         "max_rel_excursion": float(abs(te - te[0]).max() / abs(te[0])),
                         "list_builds": g.stats()["list_builds"], "hist": hist}
    # normalised g(r) of both runs and their largest difference
    edges = np.linspace(0.0, LONG["rdf_rmax"], LONG["rdf_bins"] + 1)
    shell = 4.0 / 3.0 * np.pi * (edges[1:] ** 3 - edges[:-1] ** 3)
    samples = steps // LONG["rdf_every"]
    # ordered pairs: g(r) = hist / (samples N rho shell volume)
    gr = {p: out[p].pop("hist") / (samples * N * (N / L ** 3) * shell) for p in out}
    peak = int(np.argmax(gr["mixed"]))
    line = {"metric": "4M-atom mixed-precision NVE with RDF sampling (atom-steps/s, incl. sampling)",
            "unit": "atom-steps/s", "value": out["mixed"]["atom_steps_per_s"], "steps": steps, "atoms": N,
            "mixed": out["mixed"], "fp64": out["fp64"],
            "speedup_vs_fp64": out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"],
            "rdf": {"samples": samples, "bins": LONG["rdf_bins"], "rmax": LONG["rdf_rmax"],
                    "first_peak_r": float(0.5 * (edges[peak] + edges[peak + 1])),
                    "first_peak_g": float(gr["mixed"][peak]),
                    "max_abs_diff_vs_fp64": float(np.abs(gr["mixed"] - gr["fp64"]).max())},
            "config": {"workload": f"FCC LJ fluid N={N} (4*100^3), rho=0.8, T=0.9, rc=2.5, dt=0.004, seeded MB "
                                   "velocities; RDF 200 bins to 4 sigma every 100 steps", "data": "synthetic"}}
    print(json.dumps(line), flush=True)


OUTPUTS = dict(n_cells=40, T=1.0, rho=0.8442, seed=5489, steps=2000, every=250, window=1000, reps=200)


def run_output_bench(args):
    """The outputs beside the path on one 256 000-atom system (4 * 40^3 FCC, rho
    0.8442, T 1.0, FP64): the trajectory stream (a frame every 250 of 2000 steps in
    the snapshot format, written by the background thread while the GPU steps on)
    against the same 2000 steps without it, by CUDA events on the engine's stream;
    and the ThermodynamicAnalyzer window statistics over the last 1000 records on
    the device against the host restatement over the same records."""
    import tempfile
    import torch
    from lennardjonesium import GpuSystem, initial_condition, window_stats_host
    N = 4 * OUTPUTS["n_cells"] ** 3
    x, v, L = initial_condition(N, OUTPUTS["T"], OUTPUTS["rho"], OUTPUTS["seed"])
    steps, W, reps = OUTPUTS["steps"], OUTPUTS["window"], OUTPUTS["reps"]
    with GpuSystem(N, L) as g:
        g.upload(x, v=v)
        g.step(64, record=False)  # graph capture and the first list outside the timed regions
        stream = torch.cuda.ExternalStream(g.stream)

        def device_seconds(fn):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            fn()
            e1.record(stream)
            g.synchronize()
            return e0.elapsed_time(e1) / 1e3

        plain = device_seconds(lambda: g.step_async(steps))
        with tempfile.TemporaryDirectory() as d:
            path = pathlib.Path(d) / "trajectory.csv"
            g.trajectory_open(path, OUTPUTS["every"])
            t0 = time.perf_counter()
            with_frames = device_seconds(lambda: g.step_async(steps))
            frames = g.trajectory_close()
            wall = time.perf_counter() - t0
            nbytes = path.stat().st_size
        recs = g.step(W)
        rho = N / L ** 3
        dev = g.window_stats(W, rho)
        host = window_stats_host(recs, N, rho)
        t0 = time.perf_counter()
        for _ in range(reps):
            g.window_stats(W, rho)
        t_dev = (time.perf_counter() - t0) / reps
        t0 = time.perf_counter()
        for _ in range(reps):
            window_stats_host(recs, N, rho)
        t_host = (time.perf_counter() - t0) / reps
    rel = max(abs(dev[k] - host[k]) / max(abs(host[k]), 1e-300) for k in dev)
    line = {"metric": "trajectory stream and window statistics beside the 256 000-atom step",
            "unit": "ms per step", "value": 1e3 * with_frames / steps, "steps": steps, "atoms": N,
            "trajectory": {"every": OUTPUTS["every"], "frames": frames, "bytes": nbytes,
                           "ms_per_step_without": 1e3 * plain / steps, "ms_per_step_with": 1e3 * with_frames / steps,
                           "device_time_overhead": with_frames / plain - 1.0,
                           "wall_s_until_written": wall, "rows_per_s": frames * N / wall},
            "window_stats": {"records": W, "device_call_us": 1e6 * t_dev, "host_restatement_us": 1e6 * t_host,
                             "max_rel_diff": rel},
            "config": {"workload": f"FCC LJ fluid N={N} (4*40^3), rho=0.8442, T=1.0, rc=2.5, dt=0.005, FP64; "
                                   "a frame every 250 of 2000 steps; analyzer over the last 1000 records",
                       "data": "synthetic"}}
    print(json.dumps(line), flush=True)


ADJ = dict(N=4000, rho=0.8, T=1.2, steps=200, k=20, dt=0.005, seed=4000, h=1e-6)


def run_adjoint_bench(args):
    """Differentiable NVE at N = 4000 (4 * 10^3 FCC), rho = 0.8, T = 1.2, 200 steps,
    checkpoints every 20: time of one forward pass and of one backward (adjoint)
    pass on the device, and the gradient against central finite differences
    (h = 1e-6) for epsilon, sigma and a random unit direction of the positions."""
    import numpy as np
    import torch
    from lennardjonesium import AdjointNVE, initial_condition
    x, v, L = initial_condition(ADJ["N"], ADJ["T"], ADJ["rho"], ADJ["seed"])
    x, v = x[:, :3].copy(), v[:, :3].copy()
    with AdjointNVE(ADJ["N"], L, ADJ["steps"], checkpoint_every=ADJ["k"], time_delta=ADJ["dt"]) as e:
        e.forward(x, v)
        e.backward(1.0, 1.0)  # warm-up
        torch.cuda.synchronize()
        reps = max(3, min(args.steps, 20))
        t0 = time.perf_counter()
        for _ in range(reps):
            e.forward(x, v)
        t1 = time.perf_counter()
        for _ in range(reps):
            g = e.backward(1.0, 1.0)
        t2 = time.perf_counter()
        pe, p, _ = e.forward(x, v)
        g = e.backward(1.0, 1.0)
        rng = np.random.default_rng(1)
        d = rng.standard_normal(x.shape)
        d /= np.linalg.norm(d)
        h = ADJ["h"]

        def loss(xs, eps, sig):
            e.set_potential(eps, sig)
            a, b, _ = e.forward(xs, v)
            return a + b

        checks = {"epsilon": ((loss(x, 1 + h, 1) - loss(x, 1 - h, 1)) / (2 * h), g["epsilon"]),
                  "sigma": ((loss(x, 1, 1 + h) - loss(x, 1, 1 - h)) / (2 * h), g["sigma"]),
                  "x0_direction": ((loss(x + h * d, 1, 1) - loss(x - h * d, 1, 1)) / (2 * h), float((g["x0"] * d).sum()))}
    fwd, bwd = (t1 - t0) / reps, (t2 - t1) / reps
    line = {"metric": "differentiable NVE gradient (forward + adjoint) per second", "unit": "gradients/s",
            "value": 1.0 / (fwd + bwd), "forward_ms": 1e3 * fwd, "backward_ms": 1e3 * bwd,
            "forward_atom_steps_per_s": ADJ["N"] * ADJ["steps"] / fwd,
            "loss": {"pe_avg": pe, "p_avg": p},
            "fd_check": {k: {"central_difference": fd, "adjoint": ad, "rel_err": abs(ad - fd) / abs(fd)}
                         for k, (fd, ad) in checks.items()},
            "config": {"workload": "N=4000 (4*10^3 FCC), rho=0.8, T=1.2, rc=2.5 sigma, dt=0.005, 200 steps, FP64, "
                                   "checkpoint every 20; loss = time-averaged PE + virial pressure",
                       "timing": "wall clock around synchronised calls (host-driven per-step launches)",
                       "data": "synthetic"}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--drift-steps", type=int, default=10000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="skip the autotuner (skin and pair-kernel block size per precision)")
    ap.add_argument("--skin", type=float, default=None, help="with --no-autotune: Verlet skin (default 0.3)")
    ap.add_argument("--block", type=int, default=0, help="with --no-autotune: pair-kernel block size (default 128)")
    ap.add_argument("--mixed-per-pair", action="store_true",
                    help="mixed path: add every pair force in FP64 (default: FP32 sums of 8 pairs)")
    ap.add_argument("--workload", choices=("single", "sweep", "long", "adjoint", "outputs"), default="single",
                    help="single: the 1M-atom benchmark line; sweep: batched vs sequential 64-system sweep; "
                         "long: 4M-atom mixed-precision run with RDF sampling against FP64; "
                         "adjoint: differentiable NVE gradient at N = 4000; outputs: trajectory stream "
                         "and window statistics beside the 256 000-atom step")
    ap.add_argument("--long-steps", type=int, default=20000, help="steps of the long workload")
    ap.add_argument("--cells", type=int, default=64,
                    help="FCC cells per box edge (N = 4 cells^3); 64 is the benchmark workload")
    args = ap.parse_args()
    global N_ATOMS
    WORK["n_cells"] = args.cells
    N_ATOMS = 4 * args.cells ** 3
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "sweep":
        run_sweep_bench(args)
        return
    if args.workload == "long":
        run_long_bench(args)
        return
    if args.workload == "adjoint":
        run_adjoint_bench(args)
        return
    if args.workload == "outputs":
        run_output_bench(args)
        return
    if args.impl == "reference":
        # CPU only: rank 0 runs the reference arm, the other ranks exit at once
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    ws, rank, local = dist_setup(args)
    try:
        run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
