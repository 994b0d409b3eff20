#!/usr/bin/env python
"""Benchmark: batched L-FTS Langevin steps/s on B200.

Workload (one "step" = one Langevin step of every replica, each replica doing
its Leimkuhler-Matthews update and its Anderson-mixing saddle-point search to
error 1e-4): AB diblock f=0.5, chiN=17, nbar=100, continuous chain N=90
(ds=1/90), grid 64^3, box 7.3 R0, dt=0.8, 64 replicas per GPU, FP64.  Replica r
has seed 1000+r (PCG64) for its initial Normal(0,1) fields and its noise.
Synthetic data; nothing is read from disk.

  value     replica-steps/s with this step's noise already in HBM
  e2e       the same through the public BatchedLFTS.step API: noise drawn on
            the host (PCG64, as the reference driver draws it), copied in, the
            per-replica statistics copied out, every step
  roofline  the fused continuous contour step (lfts_step_continuous) at the
            workload's batch shape, timed with CUDA events on its stream
  cpu_baseline / --impl reference
            the reference's own CPU platform (oracle/_ref, OpenMP over
            propagators) through the same driver on this host

usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Langevin steps/s @ saddle err 1e-4 (batched L-FTS, plain FP64)"
METRIC_FP32 = "Langevin steps/s @ saddle err 1e-4 (batched L-FTS, FP32 propagators, FP64 reductions)"
UNIT = "replica-steps/s"


# The batched L-FTS workloads: diblock64 is the headline (64^3, 64 replicas);
# diblock96 is the system of the learned-start study run with the plain solver.
WORKLOADS = {
    "diblock64": {"nx": 64, "lx": 7.3, "f": 0.5, "chin": 17.0, "nbar": 100, "replicas": 64, "seed": 1000},
    "diblock96": {"nx": 96, "lx": 8.0, "f": 0.4, "chin": 18.0, "nbar": 200, "replicas": 16, "seed": 2000},
}


def workload_config(R, nx, name="diblock64"):
    """The benchmark workload as both arms report it."""
    w = WORKLOADS[name]
    return {"workload": f"batched L-FTS: {R} replicas/GPU of AB diblock f={w['f']} chiN={w['chin']:g} nbar={w['nbar']} "
                        f"N=90, {nx}^3 box {w['lx']}, dt=0.8, saddle tol 1e-4, AM max_hist 20",
            "replicas_per_gpu": R, "grid": [nx] * 3, "N": 90,
            "l2": f"inputs ({R} replicas x 4 propagators x 46 slices x {8 * nx ** 3 / 2 ** 20:.0f} MB) far exceed the 126 MB L2"}


def params(nx=64, lx=7.3, f=0.5, chin=17.0, nbar=100):
    return {
        "nx": [nx] * 3, "lx": [lx] * 3, "chain_model": "continuous", "ds": 1 / 90,
        "segment_lengths": {"A": 1.0, "B": 1.0}, "chi_n": {"A,B": chin},
        "distinct_polymers": [{"volume_fraction": 1.0, "blocks": [{"type": "A", "length": f}, {"type": "B", "length": 1 - f}]}],
        "langevin": {"dt": 0.8, "nbar": nbar}, "saddle": {"max_iter": 100, "tolerance": 1e-4},
        "am": {"max_hist": 20, "start_error": 5e-1, "mix_min": 0.01, "mix_init": 0.01},
    }


def workload_params(name, nx=None):
    w = WORKLOADS[name]
    return params(nx or w["nx"], w["lx"], w["f"], w["chin"], w["nbar"])


def initial_fields(seed, M):
    rng = np.random.Generator(np.random.PCG64(seed))
    return {"A": rng.normal(0.0, 1.0, M), "B": rng.normal(0.0, 1.0, M)}


class Clocks:
    """nvidia-smi clock/throttle samples during a timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            out, _ = self.proc.communicate(timeout=10)
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def load_reference():
    """The reference CPU build (oracle/_ref), loaded under a private name."""
    import glob
    import importlib.machinery
    import importlib.util
    hits = glob.glob(os.path.join(ROOT, "oracle", "_ref", "langevinfts*.so"))
    if not hits:
        return None
    loader = importlib.machinery.ExtensionFileLoader("langevinfts", hits[0])
    spec = importlib.util.spec_from_file_location("langevinfts", hits[0], loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def reference_sample(n_iter, threads, timeout=900, workload="diblock64"):
    """Time n_iter saddle-point iterations of one replica on the reference CPU
    platform through the same driver; returns (seconds per iteration, threads).
    Runs in a child process: the reference keeps two grids of reals and two of
    complex spectra per contour step on the stack (CpuSolverPseudo.cpp:127-128,
    8.3 MB at 64^3) and needs an unlimited stack and OMP_STACKSIZE, as its
    README and driver set them."""
    import resource
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_STACKSIZE="1G")

    def unlimited_stack():
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--ref-sample", str(n_iter), "--threads", str(threads),
                        "--workload", workload],
                       env=env, preexec_fn=unlimited_stack, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        sys.stderr.write(r.stdout[-2000:] + r.stderr[-2000:])
        return None
    return tuple(json.loads(r.stdout.strip().splitlines()[-1]))


def _reference_sample_child(n_iter, threads, workload="diblock64"):
    ref = load_reference()
    if ref is None:
        return None
    from langevinfts_b200.lfts import LFTS
    p = workload_params(workload)
    seed = WORKLOADS[workload]["seed"]
    sim = LFTS(p, random_seed=seed, module=ref, platform="cpu-mkl")
    M = sim.M
    w = initial_fields(seed, M)
    S = len(sim.monomer_types)
    w_aux = sim.mpt.to_aux_fields(np.array([w[t] for t in sim.monomer_types]))
    sim.am.reset_count()
    ts = []
    err = 1e20
    for _ in range(n_iter + 1):
        t0 = time.perf_counter()
        phi = sim.compute_concentrations(w_aux)
        h = sim.mpt.compute_func_deriv(w_aux, phi, sim.mpt.aux_fields_imag_idx)
        old, err = err, float(np.max(np.std(h, axis=1)))
        for c, i in enumerate(sim.mpt.aux_fields_imag_idx):
            h[c] *= sim.dt_scaling[i]
        w_aux[sim.mpt.aux_fields_imag_idx] = np.reshape(
            sim.am.calculate_new_fields(w_aux[sim.mpt.aux_fields_imag_idx], -h, old, err), [len(sim.mpt.aux_fields_imag_idx), M])
        ts.append(time.perf_counter() - t0)
    print(json.dumps([float(np.mean(ts[1:])), threads]))
    return 0


def _reference_steps_child(k_max, budget_s, workload="diblock64"):
    """The reference CPU platform through the driver: the initial saddle-point
    search of one replica (untimed, its warm-up), then Langevin steps until
    k_max are done or the next one would pass budget_s of timed work (at
    least one).  Prints [seconds per step, saddle iterations per step, steps,
    initial iterations, failed steps, threads]."""
    ref = load_reference()
    if ref is None:
        return 1
    from langevinfts_b200.lfts import LFTS
    p = workload_params(workload)
    seed = WORKLOADS[workload]["seed"]
    sim = LFTS(p, random_seed=seed, module=ref, platform="cpu-mkl")
    it0, _ = sim.start(initial_fields(seed, sim.M))
    ts, its, fails = [], [], 0
    while len(ts) < max(k_max, 1):
        if ts and sum(ts) + ts[-1] > budget_s:
            break
        t0 = time.perf_counter()
        it, _, _, failed = sim.step()
        ts.append(time.perf_counter() - t0)
        its.append(it)
        fails += int(failed)
    print(json.dumps([float(np.mean(ts)), float(np.mean(its)), len(ts), int(it0), fails,
                      int(os.environ.get("OMP_NUM_THREADS", "1"))]))
    return 0


REFERENCE_STEP_BUDGET_S = 150.0


def run_reference(args):
    """--impl reference: the reference's CPU implementation on this host, one
    replica at a time, real Langevin steps (each with its own saddle-point
    search) after the initial search; its own iteration counts."""
    import resource
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    if load_reference() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference CPU build) is missing"}))
        return 0
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_STACKSIZE="1G")
    t_run = time.perf_counter()
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--ref-steps", str(args.steps), "--ref-budget",
                        str(REFERENCE_STEP_BUDGET_S), "--workload", args.workload], env=env, capture_output=True, text=True,
                       timeout=3000, preexec_fn=lambda: resource.setrlimit(
                           resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY)))
    t_run = time.perf_counter() - t_run
    if r.returncode != 0:
        sys.stderr.write(r.stdout[-2000:] + r.stderr[-2000:])
        print(json.dumps({"impl": "reference", "unavailable": "the reference CPU platform failed on this host (see stderr)"}))
        return 0
    t_step, ips, n, it0, fails, thr = json.loads(r.stdout.strip().splitlines()[-1])
    v = 1.0 / t_step
    sample = (f"initial saddle-point search of 1 replica ({it0} iterations, untimed), then {n} timed Langevin step(s) "
              f"of that replica ({ips:.1f} saddle iterations per step, its own count; {fails} failed), {args.nx}^3, N=90; "
              f"reference CPU platform (project FFT in place of MKL), {thr} OpenMP threads; steps stop after "
              f"{REFERENCE_STEP_BUDGET_S:.0f} s of timed work")
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": n,
           "steps_requested": args.steps, "warmup": 0, "ms_per_step": 1000.0 * t_step, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": dict(workload_config(args.replicas, args.nx, args.workload), parallelism="reference CPU platform, OpenMP threads",
                          reference_sample="one replica; replica-steps/s = 1 / (seconds per Langevin step)",
                          mean_saddle_iterations=ips, initial_saddle_iterations=it0, failed_steps=fails,
                          run_seconds=t_run),
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": thr, "kind": "reference", "sample": sample},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def step_traffic_per_job(s_bytes):
    """DRAM bytes (read + write) per (replica, key, contour step) of one
    continuous step, from the ncu summary committed under profiles/ (the line
    'dram_bytes_per_job_step f64 <bytes>', captured one kernel at a time at 32
    jobs), or None when it is absent."""
    tag = {8: "f64", 4: "f32"}[s_bytes]
    try:
        with open(os.path.join(ROOT, "profiles", "step_continuous_64cubed.txt")) as fh:
            for line in fh:
                f = line.split()
                if len(f) == 3 and f[0] == "dram_bytes_per_job_step" and f[1] == tag:
                    return float(f[2])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------- single-system statistics
# compute_statistics of one system through the langevinfts API: configs 1 (32^3
# diblock) and 3 (48^3 discrete branched mixture), seeded normal fields.
STAT_CONFIGS = {
    "diblock32_continuous": {
        "nx": [32, 32, 32], "lx": [4.0, 4.0, 4.0], "model": "continuous", "ds": 0.01, "bonds": {"A": 1.0, "B": 1.0},
        "polymers": [(1.0, [["A", 0.5, 0, 1], ["B", 0.5, 1, 2]])], "seed": 1, "sigma": 1.0},
    "branched48_discrete": {
        "nx": [48, 48, 48], "lx": [5.0, 5.0, 5.0], "model": "discrete", "ds": 1 / 60,
        "bonds": {"A": 1.0, "B": 1.0, "C": 1.0},
        "polymers": [(0.5, [["A", 20 / 60, 0, 1], ["B", 20 / 60, 0, 2], ["C", 20 / 60, 0, 3]]),
                     (0.3, [["B", 5 / 60, i, i + 1] for i in range(8)] + [["A", 6 / 60, i, 8 + i] for i in range(1, 9)]),
                     (0.2, [["A", 30 / 60, 0, 1]])], "seed": 3, "sigma": 2.0},
}


def time_statistics(module, platform, cfg, reps, warm):
    """Median wall time (s) of compute_statistics and the partition functions."""
    f = module.PlatformSelector.create_factory(platform, False)
    cb = f.create_computation_box(cfg["nx"], cfg["lx"])
    mol = f.create_molecules_information(cfg["model"], cfg["ds"], cfg["bonds"])
    for vf, blocks in cfg["polymers"]:
        mol.add_polymer(vf, blocks)
    pa = f.create_propagator_analyzer(mol, True)
    solver = f.create_pseudospectral_solver(cb, mol, pa)
    rng = np.random.Generator(np.random.PCG64(cfg["seed"]))
    M = cb.get_n_grid()
    w = {t: rng.normal(0, cfg["sigma"], M) for t in sorted(cfg["bonds"])}
    for _ in range(warm):
        solver.compute_statistics(w)
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        solver.compute_statistics(w)
        ts.append(time.perf_counter() - t0)
    Q = [solver.get_total_partition(p) for p in range(len(cfg["polymers"]))]
    return float(np.median(ts)), Q


def _reference_statistics_child(name, threads):
    ref = load_reference()
    if ref is None:
        return 1
    t, Q = time_statistics(ref, "cpu-mkl", STAT_CONFIGS[name], reps=3, warm=1)
    print(json.dumps([t, Q, threads]))
    return 0


def run_statistics(args):
    """One JSON line per config: GPU and reference-CPU compute_statistics times."""
    import resource
    from langevinfts_b200 import langevinfts as L
    ncpu = os.cpu_count() or 1
    for name, cfg in STAT_CONFIGS.items():
        t_gpu, Q_gpu = time_statistics(L, "cuda", cfg, reps=20, warm=3)
        ref = {}
        for threads in sorted({1, min(ncpu, 8)}):
            env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_STACKSIZE="1G")
            r = subprocess.run([sys.executable, os.path.abspath(__file__), "--ref-statistics", name, "--threads", str(threads)],
                               env=env, capture_output=True, text=True, timeout=1800,
                               preexec_fn=lambda: resource.setrlimit(resource.RLIMIT_STACK,
                                                                     (resource.RLIM_INFINITY, resource.RLIM_INFINITY)))
            if r.returncode == 0:
                t_ref, Q_ref, _ = json.loads(r.stdout.strip().splitlines()[-1])
                ref[f"{threads}_threads_ms"] = 1e3 * t_ref
                ref["Q_rel_diff"] = float(np.max(np.abs(np.array(Q_gpu) / np.array(Q_ref) - 1)))
        print(json.dumps({"statistics": name, "grid": cfg["nx"], "gpu_ms": 1e3 * t_gpu, "reference_cpu": ref,
                          "timing": "median of 20 (GPU) / 3 (CPU) compute_statistics calls, wall clock"}))
    return 0


# ---------------------------------------------------------------- SCFT (config 2)
def scft_params(platform_tol=1e-8, max_iter=2000):
    """64^3 SCFT of a conformationally asymmetric AB diblock: f = 0.36, chiN = 20,
    epsilon = b_A / b_B = 1.2, box 3.6 per side relaxing with stress, Anderson
    mixing with 20 histories, tolerance 1e-8.  N = 100 contour steps: with
    f = 0.36 the A block of an N = 90 chain would have 32.4 segments, which the
    reference (and this module) rejects."""
    eps, f = 1.2, 0.36
    den = eps * eps * f + (1 - f)
    return {"nx": [64, 64, 64], "lx": [3.6, 3.6, 3.6], "chain_model": "continuous", "ds": 1 / 100,
            "segment_lengths": {"A": (eps * eps / den) ** 0.5, "B": (1.0 / den) ** 0.5}, "chi_n": {"A,B": 20.0},
            "distinct_polymers": [{"volume_fraction": 1.0, "blocks": [{"type": "A", "length": f},
                                                                       {"type": "B", "length": 1 - f}]}],
            "box_is_altering": True, "scale_stress": 1.0,
            "optimizer": {"name": "am", "max_hist": 20, "start_error": 1e-2, "mix_min": 0.1, "mix_init": 0.1},
            "max_iter": max_iter, "tolerance": platform_tol}


def scft_initial(nx, chin=20.0):
    M = int(np.prod(nx))
    x = np.arange(nx[0]) * 2 * np.pi / nx[0]
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    g = (np.sin(X) * np.cos(Y) + np.sin(Y) * np.cos(Z) + np.sin(Z) * np.cos(X)).reshape(-1)
    rng = np.random.Generator(np.random.PCG64(2))
    return {"A": chin * g + 0.1 * rng.normal(0, 1, M), "B": -chin * g + 0.1 * rng.normal(0, 1, M)}


def host_scft_sample(module, platform, n_iter):
    """n_iter iterations of the scft.py loop driven from numpy through the public
    API of a module (fields to and from the host every iteration); median
    seconds per iteration after the first."""
    from langevinfts_b200.scft import build_system
    p = scft_params()
    _, _, mpt, f, cb, molecules, analyzer = build_system(p, module, platform)
    solver = f.create_pseudospectral_solver(cb, molecules, analyzer)
    M = cb.get_n_grid()
    dv = cb.get_volume() / M
    am = f.create_anderson_mixing(2 * M + 3, 20, 1e-2, 0.1, 0.1)
    init = scft_initial(p["nx"])
    w = np.array([init["A"], init["B"]])
    w -= w.mean(axis=1, keepdims=True)
    err, ts = 1e20, []
    for _ in range(n_iter):
        t0 = time.perf_counter()
        solver.compute_statistics({"A": w[0], "B": w[1]})
        phi = np.array([solver.get_total_concentration(t) for t in ("A", "B")])
        wd = mpt.matrix_chi @ phi - mpt.matrix_p @ w
        wd -= wd.mean(axis=1, keepdims=True)
        old, err = err, np.sqrt(dv * np.sum(wd ** 2) / (1.0 + dv * np.sum(w ** 2)))
        solver.compute_stress()
        st = np.array(solver.get_stress())
        err += np.sqrt(np.sum(st ** 2))
        new = am.calculate_new_fields(np.concatenate([w.reshape(-1), cb.get_lx()]),
                                      np.concatenate([wd.reshape(-1), -st]), old, err)
        lx0 = np.array(cb.get_lx())
        cb.set_lx(list((1 + np.clip((new[-3:] - lx0) / lx0, -0.1, 0.1)) * lx0))
        solver.update_laplacian_operator()
        w = new[:2 * M].reshape(2, M).copy()
        w -= w.mean(axis=1, keepdims=True)
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts[1:] if len(ts) > 1 else ts))


def _reference_scft_child(n_iter, threads):
    ref = load_reference()
    if ref is None:
        return 1
    print(json.dumps([host_scft_sample(ref, "cpu-mkl", n_iter), threads]))
    return 0


def run_learned(args):
    """Ablation of the learned saddle-point start on the workload's system:
    equilibrate, collect (w_-, w_+prev) -> w_+ pairs from the plain solver,
    train the U-Net, then run the same Langevin steps (same state, same host
    noise) with and without the learned start and compare saddle iterations."""
    import torch
    from langevinfts_b200 import langevinfts as L
    from langevinfts_b200.lfts import BatchedLFTS
    from langevinfts_b200.learned import generate_pairs, train
    from langevinfts_b200.ensemble import replica_seeds
    torch.cuda.init()
    R = args.replicas
    p = workload_params(args.workload, args.nx)
    seeds = replica_seeds(0, R, base=WORKLOADS[args.workload]["seed"])
    sim = BatchedLFTS(p, seeds, module=L, platform="cuda" if args.precision == "fp64" else "cuda-fp32")
    sim.engine.autotune()
    sim.start([initial_fields(s, sim.M) for s in seeds])
    for _ in range(args.warmup):
        sim.step()
    t0 = time.time()
    X, Y, it_gen = generate_pairs(sim, args.learned_steps)
    t_gen = time.time() - t0
    t0 = time.time()
    start, hist = train(X, Y, seconds=args.learned_train, tcgen05=False)  # torch autograd over cuDNN, torch AdamW
    t_train = time.time() - t0
    t0 = time.time()
    start_tc, hist_tc = train(X, Y, seconds=args.learned_train)  # every convolution on tcgen05, AdamW kernel
    t_train_tc = time.time() - t0
    from langevinfts_b200.learned import ablation
    res = ablation(sim, [None, start, start_tc], args.steps)
    plain, learned, learned_tc = [(r["mean_iterations"], R * args.steps / r["seconds"], r["failed"]) for r in res]
    print(json.dumps({"metric": "mean saddle-point iterations per Langevin step (learned start ablation)",
                      "workload": args.workload, "grid": [args.nx] * 3, "replicas": R, "precision": args.precision,
                      "plain": {"mean_iterations": plain[0], "replica_steps_per_s": plain[1], "failed": plain[2]},
                      "learned": {"mean_iterations": learned[0], "replica_steps_per_s": learned[1], "failed": learned[2]},
                      "learned_tcgen05": {"mean_iterations": learned_tc[0], "replica_steps_per_s": learned_tc[1],
                                          "failed": learned_tc[2], "train_seconds": t_train_tc, "epochs": len(hist_tc),
                                          "loss_first_last": [hist_tc[0][1], hist_tc[-1][1]],
                                          "network": "trained and run on lfts_conv3d_bf16 / lfts_conv3d_wgrad_bf16 (tcgen05)"},
                      "steps": args.steps, "training_pairs": int(len(X)), "data_steps": args.learned_steps,
                      "data_seconds": t_gen, "train_seconds": t_train, "epochs": len(hist),
                      "loss_first_last": [hist[0][1], hist[-1][1]],
                      "model": "3-level periodic 3D U-Net, 24 base channels, 3^3 kernels; 'learned': trained by torch autograd over "
                               "cuDNN (BF16 autocast) and torch AdamW; both run their inference on lfts_conv3d_bf16",
                      "timing": "wall clock around the steps, host noise"}))
    return 0


def structure_function_step(sim, w_aux, phi):
    """This step's contribution to S_AB(k) of every replica, the term
    examples/fts/lfts.py:756-767 accumulates (mu_A(k) conj(phi_B(k)), transforms
    of the host fields by numpy.fft.rfftn), scaled by V sqrt(nbar) as its
    recording does (:780-782).  Real part, [R, nx, ny, nz/2+1]."""
    nx = list(sim.cb.get_nx())
    M, S = sim.M, sim.S
    a, b = 0, 1  # the pair (A, B) in monomer_types order
    out = []
    for r in range(sim.R):
        phib = np.fft.rfftn(phi[r, b].reshape(nx)) / M
        mua = np.zeros_like(phib)
        for k in range(S - 1):
            mua += np.fft.rfftn(w_aux[r, k].reshape(nx)) * sim.mpt.matrix_a_inv[k, a] / sim.mpt.eigenvalues[k] / M
        out.append((mua * np.conj(phib)).real)
    return np.array(out) * sim.cb.get_volume() * np.sqrt(sim.params["langevin"]["nbar"])


def radial_bins(sim, nbins):
    """|k| of the half spectrum and its bin index (nbins bins up to the largest |k|/2)."""
    nx, lx = list(sim.cb.get_nx()), list(sim.cb.get_lx())
    ks = [2 * np.pi * np.fft.fftfreq(n, d=l / n) for n, l in zip(nx[:-1], lx[:-1])]
    ks.append(2 * np.pi * np.fft.rfftfreq(nx[-1], d=lx[-1] / nx[-1]))
    K = np.sqrt(sum(np.meshgrid(*[k ** 2 for k in ks], indexing="ij")))
    edges = np.linspace(0.0, K.max() / 2, nbins + 1)
    idx = np.digitize(K, edges) - 1
    return K, edges, idx


def run_ensemble(args):
    """Ensemble statistics of the three forms against the plain FP64 run
    (examples/fts/lfts.py:733-767 records the same quantities).  After
    args.warmup plain FP64 steps from the seeded start, each form runs the same
    args.steps Langevin steps from that state with the same PCG64 noise:
      fp64          plain batched FP64
      fp32          FP32 propagators, compensated FP64 reductions
      fp32_learned  FP32 with the learned saddle-point start (trained in this
                    run on pairs from plain FP32 steps that continue the state)
    Per replica the time averages of H, dH/dchiN and the radially averaged
    S_AB(k) (every --sf-period steps) are formed; each form is compared with
    fp64 in units of the standard error over replicas: paired (the mean of the
    per-replica differences / its standard error) and unpaired (difference of
    the ensemble means / the combined standard error).  One JSON line."""
    import torch
    from langevinfts_b200 import langevinfts as L
    from langevinfts_b200.ensemble import replica_seeds
    from langevinfts_b200.learned import generate_pairs, train
    from langevinfts_b200.lfts import BatchedLFTS
    torch.cuda.init()
    R, K = args.replicas, args.steps
    p = workload_params(args.workload, args.nx)
    seeds = replica_seeds(0, R, base=WORKLOADS[args.workload]["seed"])
    t_all = time.time()
    sims = {"cuda": BatchedLFTS(p, seeds, module=L, platform="cuda"),
            "cuda-fp32": BatchedLFTS(p, seeds, module=L, platform="cuda-fp32")}
    for s_ in sims.values():
        s_.engine.autotune()
    sim = sims["cuda"]
    sim.start([initial_fields(s, sim.M) for s in seeds])
    for _ in range(args.warmup):
        sim.step()
    w0, xi0 = sim.fields(), sim.engine.get_noise_prev()
    rng0 = [g.bit_generator.state for g in sim.rngs]

    def restore(s_):
        s_.engine.set_fields(w0)
        s_.engine.find_saddle_point()
        s_.engine.set_noise_prev(xi0)
        for g, st in zip(s_.rngs, rng0):
            g.bit_generator.state = st
    # the learned start: pairs from plain FP32 steps continuing the equilibrated state
    f32 = sims["cuda-fp32"]
    restore(f32)
    t0 = time.time()
    X, Y, _ = generate_pairs(f32, learned_pair_steps(f32.R))
    start, hist = train(X, Y, seconds=args.learned_train)
    t_train = time.time() - t0
    _, edges, idx = radial_bins(sim, args.sf_bins)
    forms = [("fp64", "cuda", None), ("fp32", "cuda-fp32", None), ("fp32_learned", "cuda-fp32", start)]
    rec = {}
    for name, plat, st in forms:
        s_ = sims[plat]
        restore(s_)
        # per replica sums over the steps that met the tolerance: a failed step
        # restores the fields and records nothing, as lfts.py:712-737 does
        Hs, dHs, nok = np.zeros(R), np.zeros(R), np.zeros(R)
        sf, nsf = np.zeros([R, args.sf_bins]), np.zeros(R)
        H_steps, iters, fails = [], [], 0
        t0 = time.time()
        for k in range(K):
            out = s_.step(start=st)
            ok = 1.0 - np.array(out["failed"], dtype=float)
            h = np.nan_to_num(np.array(out["hamiltonian"]))
            Hs += ok * h
            dHs += ok * np.nan_to_num(np.array([d["A,B"] for d in s_.h_deriv_chin(out)]))
            nok += ok
            H_steps.append(np.where(ok > 0, h, np.nan))
            iters.append(out["iterations"])
            fails += int(sum(out["failed"]))
            if (k + 1) % args.sf_period == 0:
                sk = structure_function_step(s_, s_.fields(), s_.engine.get_concentrations(s_.S))
                for b in range(args.sf_bins):
                    m = idx == b
                    if m.any():
                        sf[:, b] += ok * sk[:, m].mean(axis=1)
                nsf += ok
        rec[name] = {"H": Hs / np.maximum(nok, 1), "dH": dHs / np.maximum(nok, 1), "sf": sf / np.maximum(nsf, 1)[:, None],
                     "H_steps": np.array(H_steps), "iters": np.array(iters), "fails": fails, "seconds": time.time() - t0}
        sys.stderr.write(f"[ensemble] {name}: {K} steps in {rec[name]['seconds']:.0f} s, mean iterations "
                         f"{np.mean(iters):.2f}, <H> {rec[name]['H'].mean():.6f}, failed {fails}\n")

    def compare(a, b):
        """a, b: per-replica time averages [R] (or [R, nb]); z-scores."""
        d = a - b
        se_p = d.std(axis=0, ddof=1) / np.sqrt(R)
        se_u = np.sqrt(a.var(axis=0, ddof=1) / R + b.var(axis=0, ddof=1) / R)
        z_p = np.where(se_p > 0, d.mean(axis=0) / np.where(se_p > 0, se_p, 1), 0.0)
        z_u = (a.mean(axis=0) - b.mean(axis=0)) / np.where(se_u > 0, se_u, 1)
        return d.mean(axis=0), z_p, z_u, se_u
    base = rec["fp64"]
    res = {}
    nb_low = max(1, args.sf_bins // 2)
    for name in ("fp32", "fp32_learned"):
        r = rec[name]
        dh, zp, zu, se = compare(r["H"], base["H"])
        dd, zdp, zdu, sed = compare(r["dH"], base["dH"])
        ds, zsp, zsu, ses = compare(r["sf"], base["sf"])
        res[name] = {
            "H": {"mean": float(r["H"].mean()), "diff": float(dh), "z_paired": float(zp), "z_unpaired": float(zu),
                  "se_unpaired": float(se),
                  "max_abs_diff_per_step": float(np.nanmax(np.abs(r["H_steps"] - base["H_steps"])))},
            "dH_dchiN": {"mean": float(r["dH"].mean()), "diff": float(dd), "z_paired": float(zdp), "z_unpaired": float(zdu)},
            "S_AB_k": {"max_abs_z_paired": float(np.max(np.abs(zsp[:nb_low]))),
                       "max_abs_z_unpaired": float(np.max(np.abs(zsu[:nb_low]))),
                       "max_rel_diff": float(np.max(np.abs(ds[:nb_low]) / np.maximum(np.abs(base["sf"].mean(0)[:nb_low]), 1e-300))),
                       "bins_compared": nb_low},
            "mean_saddle_iterations": float(r["iters"].mean()), "failed_steps": r["fails"],
            "seconds": r["seconds"], "replica_steps_per_s_wall": R * K / r["seconds"]}
    out = {"ensemble": "forms vs plain FP64, same state and noise", "workload": workload_config(R, args.nx, args.workload),
           "replicas": R, "steps": K, "equilibration_steps": args.warmup, "sf_period": args.sf_period,
           "sf_bins": args.sf_bins, "sf_k_edges": [float(e) for e in edges[:nb_low + 1]],
           "criterion": "z_unpaired: (form mean - fp64 mean) / combined standard error over replicas, |z| <= 2 is "
                        "agreement within 2 sigma; z_paired: mean per-replica difference / its standard error (same "
                        "noise, so it resolves the deterministic offset of the form, reported with its size in diff)",
           "fp64": {"H_mean": float(base["H"].mean()), "H_se_replicas": float(base["H"].std(ddof=1) / np.sqrt(R)),
                    "dH_dchiN_mean": float(base["dH"].mean()), "mean_saddle_iterations": float(base["iters"].mean()),
                    "failed_steps": base["fails"], "seconds": base["seconds"],
                    "S_AB_k_low": [float(v) for v in base["sf"].mean(0)[:nb_low]]},
           "forms": res, "learned_training": {"pairs": int(len(X)), "seconds": t_train, "epochs": len(hist),
                                               "loss_first_last": [hist[0][1], hist[-1][1]]},
           "total_seconds": time.time() - t_all}
    print(json.dumps(out))
    return 0


def run_conv(args):
    """The U-Net convolutions on the tensor cores (lfts_conv3d_bf16) against
    torch's conv3d (cuDNN, BF16, channels-last) for every layer shape of the
    24-channel U-Net at the workload grid, batch 8 (the learned start's batch):
    CUDA-event time per launch, FLOP/s on the real channels, fraction of the
    measured BF16 peak."""
    import torch
    import torch.nn.functional as F
    from langevinfts_b200.learned import conv3d_tcgen05, pack_conv
    torch.cuda.init()
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(pk)) if os.path.exists(pk) else {}
    peak = float(peaks.get("bf16_tflops", 1590.0))
    N, B, b = args.nx, 8, 24
    # (name, cin real, cin padded, cout, kernel, level)
    layers = [("e1a", 2, 16, b, 3, 0), ("e1b", b, 32, b, 3, 0), ("e2a", b, 32, 2 * b, 3, 1), ("e2b", 2 * b, 48, 2 * b, 3, 1),
              ("e3a", 2 * b, 48, 4 * b, 3, 2), ("e3b", 4 * b, 96, 4 * b, 3, 2), ("d2a", 6 * b, 144, 2 * b, 3, 1),
              ("d2b", 2 * b, 48, 2 * b, 3, 1), ("d1a", 3 * b, 80, b, 3, 0), ("d1b", b, 32, b, 3, 0), ("out", b, 32, 1, 1, 0)]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    rows, tot_us, tot_us_ref, tot_flop = [], 0.0, 0.0, 0.0
    if args.conv_layer:
        layers = [l for l in layers if l[0] == args.conv_layer]
        if not layers:
            raise SystemExit(f"--conv-layer: no layer {args.conv_layer}")
    for name, ci, cip, co, k, lev in layers:
        n = N >> lev
        conv = torch.nn.Conv3d(ci, co, k).cuda()
        layer = pack_conv(conv, list(range(ci)), cip)
        x = torch.randn(B, n, n, n, cip, device="cuda").to(torch.bfloat16)
        xr = x[..., :ci].permute(0, 4, 1, 2, 3).contiguous(memory_format=torch.channels_last_3d)
        convb = conv.to(torch.bfloat16).to(memory_format=torch.channels_last_3d)
        flop = 2.0 * B * n ** 3 * ci * co * k ** 3

        def ours():
            conv3d_tcgen05(x, layer, True)

        def ref():
            F.relu(convb(F.pad(xr, (k // 2,) * 6, mode="circular") if k > 1 else xr))

        res = []
        for fn in (ours, ref):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            ev[0].record()
            for _ in range(args.steps):
                fn()
            ev[1].record()
            ev[1].synchronize()
            res.append(ev[0].elapsed_time(ev[1]) * 1e3 / args.steps)
        # forward + backward (input and weight gradients) of the layer
        from langevinfts_b200.learned import _ConvFn
        xg = x.detach().clone().requires_grad_(True)
        xrg = xr.detach().clone().requires_grad_(True)
        gy = torch.randn(B, n, n, n, layer[2], device="cuda").to(torch.bfloat16)
        gyr = gy[..., :co].permute(0, 4, 1, 2, 3).contiguous(memory_format=torch.channels_last_3d)
        convb.weight.requires_grad_(True)

        def ours_b():
            _ConvFn.apply(xg, conv.weight, conv.bias, list(range(ci)), cip, True).backward(gy)

        def ref_b():
            F.relu(convb(F.pad(xrg, (k // 2,) * 6, mode="circular") if k > 1 else xrg)).backward(gyr)

        for fn in (ours_b, ref_b):
            for _ in range(2):
                fn()
            torch.cuda.synchronize()
            ev[0].record()
            for _ in range(args.steps):
                fn()
            ev[1].record()
            ev[1].synchronize()
            res.append(ev[0].elapsed_time(ev[1]) * 1e3 / args.steps)
        tot_us, tot_us_ref, tot_flop = tot_us + res[0], tot_us_ref + res[1], tot_flop + flop
        rows.append({"layer": name, "grid": n, "cin": ci, "cout": co, "k": k, "tcgen05_us": res[0], "cudnn_us": res[1],
                     "tcgen05_tflops": flop / res[0] / 1e6, "cudnn_tflops": flop / res[1] / 1e6,
                     "fwd_bwd_tcgen05_us": res[2], "fwd_bwd_cudnn_us": res[3]})
    print(json.dumps({"metric": "U-Net convolution time per forward (batch 8)", "grid": [N] * 3, "layers": rows,
                      "total_tcgen05_us": tot_us, "total_cudnn_us": tot_us_ref,
                      "total_fwd_bwd_tcgen05_us": sum(r["fwd_bwd_tcgen05_us"] for r in rows),
                      "total_fwd_bwd_cudnn_us": sum(r["fwd_bwd_cudnn_us"] for r in rows),
                      "tcgen05_tflops": tot_flop / tot_us / 1e6, "peak_bf16_tflops": peak,
                      "frac_of_peak": tot_flop / tot_us / 1e6 / peak,
                      "note": "FLOPs on the real channels; cuDNN timing includes its circular pad"}))
    return 0


def run_scft(args):
    """SCFT of config 2 with the device loop in FP64 and FP32, and the time per
    iteration of the host-driven loop; one JSON line."""
    from langevinfts_b200.scft import SCFT
    out = {"scft": "64^3 AB diblock f=0.36 chiN=20 eps=1.2 N=100, box relaxation, AM 20, tolerance 1e-8"}
    res = {}
    for platform in ("cuda", "cuda-fp32"):
        # FP32 propagators level off near 1e-6 in the field error: stop at 1e-5
        sim = SCFT(scft_params(1e-8 if platform == "cuda" else 1e-5), platform=platform)
        t0 = time.perf_counter()
        st = sim.run(scft_initial([64, 64, 64]))
        t = time.perf_counter() - t0
        res[platform] = st
        out[platform] = {"iterations": st["iterations"], "error_level": st["error_level"], "energy": st["energy"],
                         "lx": list(sim.cb.get_lx()), "seconds": t, "ms_per_iteration": 1e3 * t / st["iterations"]}
    a, b = res["cuda"], res["cuda-fp32"]
    out["fp32_vs_fp64"] = {"energy_abs_diff": abs(a["energy"] - b["energy"]),
                           "lx_max_rel_diff": float(np.max(np.abs(np.array(out["cuda-fp32"]["lx"]) /
                                                                  np.array(out["cuda"]["lx"]) - 1)))}
    from langevinfts_b200 import langevinfts as L
    out["host_driven_ms_per_iteration"] = 1e3 * host_scft_sample(L, "cuda", 20)
    import resource
    threads = min(os.cpu_count() or 1, 8)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_STACKSIZE="1G")
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--ref-scft", "3", "--threads", str(threads)], env=env,
                       capture_output=True, text=True, timeout=1800,
                       preexec_fn=lambda: resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY)))
    if r.returncode == 0:
        out["reference_cpu_ms_per_iteration"] = {f"{threads}_threads": 1e3 * json.loads(r.stdout.strip().splitlines()[-1])[0],
                                                 "sample": "3 iterations of the same host loop on the reference CPU platform"}
    print(json.dumps(out))
    return 0


# timed steps of each variant (capped so the default run stays within minutes)
VARIANT_STEPS_MAX = 8
# plain Langevin steps whose fields train the learned start (about LEARNED_PAIRS
# pairs: 16 steps at 64 replicas, 64 at 16), and its time budget (s)
LEARNED_PAIRS = 1024
LEARNED_TRAIN_S = 120.0


def learned_pair_steps(replicas):
    return int(min(64, max(16, -(-LEARNED_PAIRS // replicas))))


def time_batched(sim, K, start=None):
    """value and e2e of K Langevin steps of a started BatchedLFTS: value with
    each step's noise already in HBM (CUDA events on the engine stream), e2e
    through the public step() with the noise drawn on the host every step and
    the statistics copied out.  Returns (value, e2e, iterations, failed, launches, d2h bytes per step)."""
    import torch
    from concurrent.futures import ThreadPoolExecutor
    R = sim.R
    stream = torch.cuda.ExternalStream(sim.engine.stream_ptr())
    noises = [torch.from_numpy(sim.draw_noise()).cuda() for _ in range(K)]
    torch.cuda.synchronize()
    iters, fails = [], 0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    k0 = sim.engine.kernel_launches()
    ev[0].record(stream)
    for k in range(K):
        st = sim.step_device(noises[k].data_ptr(), start=start)
        iters += st["iterations"]
        fails += sum(st["failed"])
    ev[1].record(stream)
    ev[1].synchronize()
    launches = sim.engine.kernel_launches() - k0
    t = ev[0].elapsed_time(ev[1]) / 1000.0
    del noises
    pool_noise = sim.draw_noise()
    torch.cuda.synchronize()
    ex = ThreadPoolExecutor(max_workers=1)
    nxt = ex.submit(sim.draw_noise)
    d2h = 0
    e0 = time.perf_counter()
    ev[2].record(stream)
    for k in range(K):
        st = sim.step(pool_noise, start=start)
        d2h += 8 * (len(st["error"]) * 4 + len(st["partitions"]) + len(st["aux_mean"]) + len(st["aux_msq"]))
        pool_noise = nxt.result()
        nxt = ex.submit(sim.draw_noise)
    ev[3].record(stream)
    ev[3].synchronize()
    t_e2e = max(time.perf_counter() - e0, ev[2].elapsed_time(ev[3]) / 1000.0)
    ex.shutdown(wait=False)
    return R * K / t, R * K / t_e2e, iters, int(fails), int(launches), int(d2h / max(K, 1))


def run_variants(args, value_fp64):
    """The forms beside the plain batched FP64 headline, same workload:
      fp32              FP32 propagators and FFTs, FP64 reductions (cuda-fp32)
      fp32_learned      the same with the learned saddle-point start: a U-Net
                        trained in this run (tensor-core kernels, AdamW kernel)
                        on about LEARNED_PAIRS pairs from plain FP32 steps
      fp64_one_replica  the unbatched plain FP64 form: one replica per engine
    Each carries value, e2e, mean saddle iterations, failed steps and its
    ratio to the plain FP64 value."""
    from langevinfts_b200 import langevinfts as L
    from langevinfts_b200.ensemble import replica_seeds
    from langevinfts_b200.learned import generate_pairs, train
    from langevinfts_b200.lfts import BatchedLFTS
    K = min(args.steps, VARIANT_STEPS_MAX)
    p = workload_params(args.workload, args.nx)
    seeds = replica_seeds(0, args.replicas, base=WORKLOADS[args.workload]["seed"])
    out = {}

    def entry(v, e, iters, fails, launches, d2h, sim, extra=None):
        d = {"value": v, "e2e": {"value": e, "unit": UNIT, "h2d_bytes_per_step": sim.R * sim.mpt.R * sim.M * 8,
                                 "d2h_bytes_per_step": d2h},
             "unit": UNIT, "steps": K, "mean_saddle_iterations": float(np.mean(iters)), "failed_steps": fails,
             "gpu_launches": launches, "vs_plain_fp64_value": v / value_fp64}
        if extra:
            d.update(extra)
        return d
    sim = BatchedLFTS(p, seeds, module=L, platform="cuda-fp32")
    tune = sim.engine.autotune()
    sim.start([initial_fields(s, sim.M) for s in seeds])
    for _ in range(args.warmup):
        sim.step()
    r = time_batched(sim, K)
    out["fp32"] = entry(*r, sim, {"dtype": "f32", "step_autotune": tune,
                                  "platform": "cuda-fp32: FP32 propagators and FFTs, compensated FP64 reductions"})
    sys.stderr.write(f"[bench] fp32 {r[0]:.3f} {UNIT} ({np.mean(r[2]):.2f} iterations)\n")
    t0 = time.time()
    pair_steps = learned_pair_steps(sim.R)
    X, Y, _ = generate_pairs(sim, pair_steps)
    t_pairs = time.time() - t0
    start, hist = train(X, Y, seconds=LEARNED_TRAIN_S)
    r = time_batched(sim, K, start=start)
    out["fp32_learned"] = entry(*r, sim, {
        "dtype": "f32", "training_pairs": int(len(X)), "pair_steps": pair_steps, "pair_seconds": t_pairs,
        "train_seconds": LEARNED_TRAIN_S, "epochs": len(hist), "loss_first_last": [hist[0][1], hist[-1][1]],
        "network": "3-level periodic 3D U-Net, 24 base channels; convolutions forward and backward on lfts_conv3d_bf16 / "
                   "lfts_conv3d_wgrad_bf16 (tcgen05), AdamW on lfts_adamw_f32, inference on lfts_conv3d_bf16"})
    sys.stderr.write(f"[bench] fp32_learned {r[0]:.3f} {UNIT} ({np.mean(r[2]):.2f} iterations)\n")
    del sim
    one = BatchedLFTS(p, seeds[:1], module=L, platform="cuda")
    one.start([initial_fields(seeds[0], one.M)])
    for _ in range(args.warmup):
        one.step()
    K1 = max(K, 10)
    r = time_batched(one, K1)
    out["fp64_one_replica"] = entry(*r, one, {"dtype": "f64", "steps": K1, "replicas": 1,
                                              "note": "the plain FP64 form without batching: one replica per engine"})
    for v in out.values():
        v["vs_fp64_one_replica_value"] = v["value"] / out["fp64_one_replica"]["value"]
    sys.stderr.write(f"[bench] fp64 one replica {r[0]:.3f} {UNIT}\n")
    return out


def roofline_step_kernel(nx, njobs, reps=20, prec=8, impl=None):
    """Time lfts_step_continuous at the batch shape of the workload (njobs =
    replicas x propagators per schedule slot) with CUDA events on its stream.
    Every job has its own field factors, as the two keys of a slot of each
    replica do; inputs, outputs, factors and spectra (njobs x 10 MB at 64^3)
    exceed the 126 MB L2."""
    import torch
    from langevinfts_b200.capi import Context, StepJob, check
    ctx = Context([nx] * 3, precision=prec)
    if impl:
        check(ctx.lib.lfts_set_step_impl(ctx.h, impl.encode()))
    name = C.create_string_buffer(64)
    check(ctx.lib.lfts_step_impl(ctx.h, name, 64))
    M, Mc = ctx.M, ctx.Mc
    sb = prec  # bytes per real
    lx = (C.c_double * 3)(7.3, 7.3, 7.3)
    bond, bondh = ctx.malloc(Mc * sb), ctx.malloc(Mc * sb)
    check(ctx.lib.lfts_bond_tables(ctx.h, 1.0, 1 / 90, lx, bond, bondh))
    w = ctx.upload(np.random.default_rng(0).normal(0, 1, njobs * M))
    fac = ctx.malloc(njobs * M * sb)
    check(ctx.lib.lfts_field_factors_batch(ctx.h, w, -1 / 360, fac, njobs))
    q = ctx.malloc(njobs * 2 * M * sb)
    check(ctx.lib.lfts_memset_async(ctx.h, q, 0, njobs * 2 * M * sb))
    ones = np.ones(M, dtype=np.float64 if prec == 8 else np.float32)
    for j in range(njobs):
        ctx.h2d(q + j * 2 * M * sb, ones)
    spec = ctx.malloc(njobs * 2 * Mc * 2 * sb)
    jobs = (StepJob * njobs)(*[StepJob(q + j * 2 * M * sb, 0, q + (j * 2 + 1) * M * sb, 0, fac + j * M * sb, bond, bondh,
                                       spec + j * 2 * Mc * 2 * sb, None, 0, 0) for j in range(njobs)])
    jp = ctx.upload(np.frombuffer(jobs, dtype=np.uint8))
    stream = torch.cuda.ExternalStream(ctx.lib.lfts_ctx_stream(ctx.h))
    for _ in range(3):
        check(ctx.lib.lfts_step_continuous(ctx.h, jp, njobs, 0))
    ctx.sync()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    for _ in range(reps):
        check(ctx.lib.lfts_step_continuous(ctx.h, jp, njobs, 0))
    ev[1].record(stream)
    ev[1].synchronize()
    ms = ev[0].elapsed_time(ev[1]) / reps
    ctx.close()
    roofline_step_kernel.impl = name.value.decode()
    return ms, M, Mc


def time_realspace_step(nx, njobs, reps=20, bc=("absorbing", "absorbing", "reflecting", "reflecting", "periodic", "periodic")):
    """CUDA-event time of one lfts_step_realspace call at njobs jobs of an nx^3
    FP64 box with the given walls; returns (ms, M)."""
    import torch
    from langevinfts_b200.capi import Context, StepJob, check
    ctx = Context([nx] * 3, precision=8)
    M = ctx.M
    codes = {"periodic": 0, "reflecting": 1, "absorbing": 2}
    tab = np.zeros(ctx.lib.lfts_realspace_table_size(ctx.h))
    check(ctx.lib.lfts_realspace_tables(ctx.h, 1.0, 1 / 90, 3, (C.c_double * 3)(*[7.3 / nx] * 3),
                                        (C.c_int * 6)(*[codes[b] for b in bc]), tab.ctypes.data))
    tdev = ctx.upload(tab)
    fac = ctx.malloc(njobs * M * 8)
    check(ctx.lib.lfts_field_factors_batch(ctx.h, ctx.upload(np.random.default_rng(0).normal(0, 1, njobs * M)), -1 / 360, fac,
                                           njobs))
    q = ctx.malloc(njobs * 2 * M * 8)
    for j in range(njobs):
        ctx.h2d(q + j * 2 * M * 8, np.ones(M))
    spec = ctx.malloc(njobs * 2 * M * 8)
    jobs = (StepJob * njobs)(*[StepJob(q + j * 2 * M * 8, 0, q + (j * 2 + 1) * M * 8, 0, fac + j * M * 8, tdev, None,
                                       spec + j * 2 * M * 8, None, 0, 0) for j in range(njobs)])
    jp = ctx.upload(np.frombuffer(jobs, dtype=np.uint8))
    stream = torch.cuda.ExternalStream(ctx.lib.lfts_ctx_stream(ctx.h))
    for _ in range(3):
        check(ctx.lib.lfts_step_realspace(ctx.h, jp, njobs, 0, 3))
    ctx.sync()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    for _ in range(reps):
        check(ctx.lib.lfts_step_realspace(ctx.h, jp, njobs, 0, 3))
    ev[1].record(stream)
    ev[1].synchronize()
    ms = ev[0].elapsed_time(ev[1]) / reps
    ctx.close()
    return ms, M


def run_ours(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    os.environ.setdefault("CUDA_DEVICE_ORDER", "PCI_BUS_ID")
    from langevinfts_b200 import langevinfts as L
    from langevinfts_b200.lfts import BatchedLFTS

    R = args.replicas
    p = workload_params(args.workload, args.nx)
    from langevinfts_b200.ensemble import max_over_ranks, replica_seeds
    seeds = replica_seeds(rank, R, base=WORKLOADS[args.workload]["seed"])
    f = L.PlatformSelector.create_factory("cuda", False)
    sim = BatchedLFTS(p, seeds, module=L, platform="cuda" if args.precision == "fp64" else "cuda-fp32")
    M = sim.M
    tune = sim.engine.autotune()  # step implementation timed at this batch (before the first captured graph)
    sim.engine.set_step_graph(args.step_graph == "on")
    st0 = sim.start([initial_fields(s, M) for s in seeds])
    for _ in range(args.warmup):
        sim.step()
    stream = torch.cuda.ExternalStream(sim.engine.stream_ptr())
    nreal = sim.mpt.R

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- value: noise for the K steps already on the device
    noises = [torch.from_numpy(sim.draw_noise()).cuda() for _ in range(args.steps)]
    barrier()
    iters, fails = [], 0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    k0 = sim.engine.kernel_launches()
    with Clocks(local) as clk:
        ev[0].record(stream)
        for k in range(args.steps):
            s = sim.engine.step_device(noises[k].data_ptr())
            iters += s["iterations"]
            fails += sum(s["failed"])
        ev[1].record(stream)
        ev[1].synchronize()
    barrier()
    launches = sim.engine.kernel_launches() - k0
    t = ev[0].elapsed_time(ev[1]) / 1000.0
    # ---- e2e: public API with host noise in and statistics out every step
    pool_noise = sim.draw_noise()
    barrier()
    e0 = time.perf_counter()
    ev2 = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev2[0].record(stream)
    from concurrent.futures import ThreadPoolExecutor
    ex = ThreadPoolExecutor(max_workers=1)
    nxt = ex.submit(sim.draw_noise)
    d2h = 0
    for k in range(args.steps):
        s = sim.step(pool_noise)
        d2h += 8 * (len(s["error"]) * 4 + len(s["partitions"]) + len(s["aux_mean"]) + len(s["aux_msq"]))
        pool_noise = nxt.result()
        nxt = ex.submit(sim.draw_noise)
    ev2[1].record(stream)
    ev2[1].synchronize()
    t_e2e = max(time.perf_counter() - e0, ev2[0].elapsed_time(ev2[1]) / 1000.0)
    ex.shutdown(wait=False)
    t, t_e2e = max_over_ranks([t, t_e2e])
    value = world * R * args.steps / t
    e2e = world * R * args.steps / t_e2e
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    sys.stderr.write(f"[bench] value {value:.3f} {UNIT}, e2e {e2e:.3f}, mean saddle iterations {np.mean(iters):.2f}, "
                     f"failed {fails}, launches {launches}\n")
    # ---- roofline of the fused continuous step at the workload batch shape
    njobs = 2 * R  # two propagators per schedule slot (A and B side) per replica
    s_bytes = 8 if args.precision == "fp64" else 4
    ms, Mg, Mcg = roofline_step_kernel(args.nx, njobs, prec=s_bytes)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    unit_bytes = s_bytes * (12 * Mg + 24 * Mcg)  # pass-model bytes per (replica, key, contour step)
    achieved = njobs * unit_bytes / (ms * 1e-3) / 1e9
    traffic = step_traffic_per_job(s_bytes) if args.nx == 64 else None
    if traffic is not None:
        traffic *= njobs
    # ---- CPU baseline: the reference CPU platform on a bounded sample
    cpu = None
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        r = reference_sample(1, threads, workload=args.workload)
        sys.stderr.write(f"[bench] reference CPU sample: {r}\n")
        if r is not None:
            mean_iters = float(np.mean(iters))
            cpu = {"value": 1.0 / (r[0] * mean_iters), "unit": UNIT, "cores": r[1], "kind": "reference",
                   "sample": f"2 saddle-point iterations of 1 replica ({args.nx}^3, N=90) on the reference CPU platform "
                             f"(first discarded), {r[0]:.2f} s/iteration x {mean_iters:.1f} iterations per step measured above"}
    out = {
        "metric": METRIC if args.precision == "fp64" else METRIC_FP32, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * t / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32", "data": "synthetic",
        "config": {**workload_config(R, args.nx, args.workload), "parallelism": f"replicas x{world}", "step_autotune": tune,
                   "step_graph": ("one CUDA graph per Langevin step (saddle loop as a device-controlled WHILE node)"
                                  if sim.engine.step_graph() else "saddle loop driven from the host"),
                   "mean_saddle_iterations": float(np.mean(iters)) if iters else None, "failed_steps": fails,
                   "initial_saddle_iterations": max(st0["iterations"])},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": R * nreal * M * 8,
                "d2h_bytes_per_step": int(d2h / max(args.steps, 1))},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "lfts_step_continuous (5 fused FFT-pass kernels)",
                     "launch_ms": ms, "jobs_per_launch": njobs,
                     "bytes_model": f"{s_bytes}*(12M+24Mc) per job (pass model), peak = measured hbm_gbs",
                     "traffic_source": "ncu dram bytes per job-step captured one kernel at a time at 32 jobs "
                                       "(profiles/step_continuous_64cubed.txt) x jobs per launch; at 128 jobs L2 "
                                       "keeps less, so this is a lower bound"},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_variants and args.precision == "fp64":
        out["variants"] = run_variants(args, value)
    print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="diblock64", choices=sorted(WORKLOADS),
                    help="diblock64: 64^3, 64 replicas (the headline); diblock96: 96^3, 16 replicas")
    ap.add_argument("--replicas", type=int, default=None)
    ap.add_argument("--nx", type=int, default=None)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                    help="fp64 (the headline) or fp32 propagators with FP64 reductions (platform cuda-fp32)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--step-graph", default="on", choices=["on", "off"],
                    help="off: drive the saddle loop from the host (one graph per iteration) instead of one graph per step")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the fp32 / fp32_learned / one-replica FP64 forms after the headline")
    ap.add_argument("--ref-sample", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--ref-steps", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--ref-budget", type=float, default=REFERENCE_STEP_BUDGET_S, help=argparse.SUPPRESS)
    ap.add_argument("--ref-statistics", default="", help=argparse.SUPPRESS)
    ap.add_argument("--ref-scft", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--scft", action="store_true", help="SCFT of the 64^3 asymmetric diblock (device loop, FP64 and FP32)")
    ap.add_argument("--conv", action="store_true", help="time the tensor-core U-Net convolutions against cuDNN")
    ap.add_argument("--conv-layer", default=None, help="with --conv: time only this layer (e1a ... d1b, out; for profiling)")
    ap.add_argument("--ensemble", action="store_true",
                    help="ensemble <H>, dH/dchiN and S(k) of the FP32 and learned forms against plain FP64 (same noise)")
    ap.add_argument("--sf-period", type=int, default=5, help=argparse.SUPPRESS)
    ap.add_argument("--sf-bins", type=int, default=24, help=argparse.SUPPRESS)
    ap.add_argument("--learned", action="store_true",
                    help="ablation of the learned saddle-point start (U-Net) on the workload's system")
    ap.add_argument("--learned-steps", type=int, default=20, help="plain Langevin steps that make the training pairs")
    ap.add_argument("--learned-train", type=float, default=60.0, help="training time budget (s)")
    ap.add_argument("--statistics", action="store_true",
                    help="time compute_statistics of single systems (configs 1 and 3) on the GPU and the reference CPU")
    ap.add_argument("--threads", type=int, default=1, help=argparse.SUPPRESS)
    ap.add_argument("--step-impl", default=None,
                    help="with --kernel-only: the step implementation to time (default: the context's own choice)")
    ap.add_argument("--realspace", action="store_true",
                    help="with --kernel-only: time the real-space Crank-Nicolson step (lfts_step_realspace) instead")
    ap.add_argument("--kernel-only", action="store_true",
                    help="only time the fused continuous step at 2*replicas jobs (for profiling)")
    args = ap.parse_args()
    if args.replicas is None:
        args.replicas = WORKLOADS[args.workload]["replicas"]
    if args.nx is None:
        args.nx = WORKLOADS[args.workload]["nx"]
    if args.ref_sample:
        return _reference_sample_child(args.ref_sample, args.threads, args.workload)
    if args.ref_steps:
        return _reference_steps_child(args.ref_steps, args.ref_budget, args.workload)
    if args.ref_statistics:
        return _reference_statistics_child(args.ref_statistics, args.threads)
    if args.ref_scft:
        return _reference_scft_child(args.ref_scft, args.threads)
    if args.statistics:
        return run_statistics(args)
    if args.scft:
        return run_scft(args)
    if args.learned:
        return run_learned(args)
    if args.conv:
        return run_conv(args)
    if args.ensemble:
        return run_ensemble(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.kernel_only and args.realspace:
        import torch
        torch.cuda.init()
        ms, M = time_realspace_step(args.nx, 2 * args.replicas, reps=args.steps)
        # compulsory bytes per job: q in, q out, the factors (8 B each) and the
        # two intermediate sweeps written and read once (4 x 8 B)
        unit = 8 * 7 * M
        print(json.dumps({"kernel": "lfts_step_realspace", "jobs": 2 * args.replicas, "nx": args.nx, "launch_ms": ms,
                          "bytes_per_job": unit, "GBps": 2 * args.replicas * unit / (ms * 1e-3) / 1e9}))
        return 0
    if args.kernel_only:
        import torch
        torch.cuda.init()
        sb = 8 if args.precision == "fp64" else 4
        ms, M, Mc = roofline_step_kernel(args.nx, 2 * args.replicas, reps=args.steps, prec=sb, impl=args.step_impl)
        unit = sb * (12 * M + 24 * Mc)
        print(json.dumps({"kernel": "lfts_step_continuous", "impl": roofline_step_kernel.impl, "precision": args.precision,
                          "jobs": 2 * args.replicas, "nx": args.nx, "launch_ms": ms,
                          "pass_model_GBps": 2 * args.replicas * unit / (ms * 1e-3) / 1e9}))
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
