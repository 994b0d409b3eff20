"""The benchmark L-FTS system end to end against the reference build.

64^3 AB diblock (f=0.5, chiN=17, nbar=100, N=90, box 7.3, dt=0.8, saddle
tolerance 1e-4, Anderson mixing with 20 histories), two replicas with seeds
1000 and 1001 on BatchedLFTS: the register-resident 64^3 step kernels, the
device saddle control, the device Anderson solve and the per-replica active
masks together.  tests/golden/lfts64_reference.npz holds the same runs on the
reference's own CPU platform (made by tests/golden/make_lfts64_golden.py):
the initial saddle-point search from seeded Normal(0, 1) fields, then one
Langevin step with the replica's PCG64 noise.  Saddle iterations must be
equal; the Hamiltonian and the fields agree to 1e-8 relative (FP64).
"""
import os

import numpy as np
import pytest

from tests.golden.make_lfts64_golden import initial_fields, lfts64_params, projection_vectors

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lfts64_reference.npz")


def check_fields(w, g, tag, r, proj):
    x = w.reshape(-1)
    ref_max = g[f"{tag}_w_maxabs"][r]
    assert np.max(np.abs(x[g["sample_idx"]] - g[f"{tag}_w_sample"][r])) <= 1e-8 * ref_max, (tag, r)
    p = proj @ x
    scale = np.sqrt(x @ x) * np.sqrt(x.size)  # |v| ~ sqrt(n) for a Normal(0, 1) vector
    assert np.max(np.abs(p - g[f"{tag}_w_proj"][r])) <= 1e-8 * scale, (tag, r)
    assert abs(x @ x / g[f"{tag}_w_sumsq"][r] - 1) < 1e-8, (tag, r)
    assert abs(np.max(np.abs(x)) / ref_max - 1) < 1e-8, (tag, r)


def test_benchmark_system_64cubed_follows_reference_build():
    from langevinfts_b200 import langevinfts as L
    from langevinfts_b200.lfts import BatchedLFTS
    g = np.load(GOLD)
    seeds = [int(s) for s in g["seeds"]]
    sim = BatchedLFTS(lfts64_params(), seeds, module=L)
    assert sim.engine.step_implementation() == "register-64"
    proj = projection_vectors(sim.S * sim.M)
    st = sim.start([initial_fields(s, sim.M) for s in seeds])
    assert list(st["iterations"]) == list(g["start_iterations"])
    np.testing.assert_allclose(st["hamiltonian"], g["start_hamiltonian"], rtol=1e-8)
    w = sim.fields()
    for r in range(len(seeds)):
        check_fields(w[r], g, "start", r, proj)
    st = sim.step()
    assert list(st["iterations"]) == list(g["step1_iterations"])
    assert not any(st["failed"])
    np.testing.assert_allclose(st["hamiltonian"], g["step1_hamiltonian"], rtol=1e-8)
    np.testing.assert_allclose(st["error"], g["step1_error"], rtol=1e-6)
    w = sim.fields()
    for r in range(len(seeds)):
        check_fields(w[r], g, "step1", r, proj)
