"""Generate tests/golden/lfts64_reference.npz: the benchmark L-FTS system
(64^3 AB diblock, f=0.5, chiN=17, nbar=100, N=90, box 7.3, dt=0.8, saddle
tolerance 1e-4, Anderson mixing with 20 histories) run on the reference's own
CPU platform (oracle/_ref, built by oracle/Makefile) for two replicas, seeds
1000 and 1001: the initial saddle-point search from seeded Normal(0, 1) fields,
then one Langevin step with the replica's PCG64 noise.

Stored per replica: saddle iterations and errors of both searches, the
Hamiltonian after the step, and the auxiliary fields after each search as
(a) their values at 2048 fixed grid indices, (b) four projections onto seeded
Normal(0, 1) vectors (PCG64(777), regenerated by the test), (c) sum, sum of
squares and max |w|.  The full fields (2 x 2 MB per snapshot) are not stored.

Usage (CPU, here; about 5 minutes per replica):
    python tests/golden/make_lfts64_golden.py
The reference CPU step keeps 8 MB of variable-length arrays on the stack per
call at 64^3, so this script re-executes itself with an unlimited stack.
"""
import json
import os
import resource
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SEEDS = [1000, 1001]
N_SAMPLE = 2048
N_PROJ = 4


def lfts64_params():
    return {
        "nx": [64, 64, 64], "lx": [7.3, 7.3, 7.3], "chain_model": "continuous", "ds": 1 / 90,
        "segment_lengths": {"A": 1.0, "B": 1.0}, "chi_n": {"A,B": 17.0},
        "distinct_polymers": [{"volume_fraction": 1.0, "blocks": [{"type": "A", "length": 0.5}, {"type": "B", "length": 0.5}]}],
        "langevin": {"dt": 0.8, "nbar": 100}, "saddle": {"max_iter": 100, "tolerance": 1e-4},
        "am": {"max_hist": 20, "start_error": 5e-1, "mix_min": 0.01, "mix_init": 0.01},
    }


def initial_fields(seed, M):
    rng = np.random.Generator(np.random.PCG64(seed))
    return {"A": rng.normal(0.0, 1.0, M), "B": rng.normal(0.0, 1.0, M)}


def sample_indices(n_total):
    return np.sort(np.random.Generator(np.random.PCG64(4242)).choice(n_total, N_SAMPLE, replace=False))


def projection_vectors(n_total):
    return np.random.Generator(np.random.PCG64(777)).normal(0.0, 1.0, [N_PROJ, n_total])


def summarize(w, idx, proj):
    x = w.reshape(-1)
    return {"sample": x[idx].tolist(), "proj": (proj @ x).tolist(), "sum": float(x.sum()),
            "sumsq": float(x @ x), "maxabs": float(np.max(np.abs(x)))}


def child(seed):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from tests import refmod
    from langevinfts_b200.lfts import LFTS
    ref = refmod.load()
    p = lfts64_params()
    sim = LFTS(p, random_seed=seed, module=ref, platform="cpu-mkl")
    n_total = len(sim.monomer_types) * sim.M
    idx, proj = sample_indices(n_total), projection_vectors(n_total)
    it0, err0 = sim.start(initial_fields(seed, sim.M))
    out = {"seed": seed, "start": {"iterations": int(it0), "error": float(err0), "hamiltonian": float(sim.hamiltonian),
                                   "w_aux": summarize(sim.w_aux, idx, proj)}}
    it1, err1, h1, failed = sim.step()
    out["step1"] = {"iterations": int(it1), "error": float(err1), "hamiltonian": float(h1), "failed": bool(failed),
                    "w_aux": summarize(sim.w_aux, idx, proj)}
    print("RESULT " + json.dumps(out))


def main():
    if len(sys.argv) > 2 and sys.argv[1] == "--child":
        return child(int(sys.argv[2]))
    env = dict(os.environ, OMP_STACKSIZE="1G", OMP_NUM_THREADS=str(max(1, (os.cpu_count() or 2) // len(SEEDS))))

    def unlimited():
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    procs = [subprocess.Popen([sys.executable, os.path.abspath(__file__), "--child", str(s)], env=env, preexec_fn=unlimited,
                              stdout=subprocess.PIPE, text=True) for s in SEEDS]
    res = []
    for pr in procs:
        out, _ = pr.communicate()
        if pr.returncode != 0:
            raise SystemExit(f"reference run failed ({pr.returncode})")
        res.append(json.loads([l for l in out.splitlines() if l.startswith("RESULT ")][-1][7:]))
    M = 64 ** 3
    arrays = {"seeds": np.array(SEEDS), "sample_idx": sample_indices(2 * M)}
    for tag in ("start", "step1"):
        arrays[f"{tag}_iterations"] = np.array([r[tag]["iterations"] for r in res])
        arrays[f"{tag}_error"] = np.array([r[tag]["error"] for r in res])
        arrays[f"{tag}_hamiltonian"] = np.array([r[tag]["hamiltonian"] for r in res])
        for k in ("sample", "proj"):
            arrays[f"{tag}_w_{k}"] = np.array([r[tag]["w_aux"][k] for r in res])
        for k in ("sum", "sumsq", "maxabs"):
            arrays[f"{tag}_w_{k}"] = np.array([r[tag]["w_aux"][k] for r in res])
    arrays["step1_failed"] = np.array([r["step1"]["failed"] for r in res])
    np.savez_compressed(os.path.join(HERE, "lfts64_reference.npz"), **arrays)
    print(json.dumps({k: v.tolist() for k, v in arrays.items() if v.size <= 4}))


if __name__ == "__main__":
    main()
