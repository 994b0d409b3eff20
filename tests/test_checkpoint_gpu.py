"""Checkpoint and resume of batched L-FTS replicas in the reference driver's
file format (examples/fts/lfts.py:569-629): a run continued from the files of
step 2 follows the uninterrupted run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REFERENCE_KEYS = {"initial_params", "dim", "nx", "lx", "monomer_types", "chi_n", "chain_model", "ds", "dt", "nbar",
                  "eigenvalues", "aux_fields_real", "aux_fields_imag", "matrix_a", "matrix_a_inverse", "langevin_step",
                  "random_generator", "random_state_state", "random_state_inc", "normal_noise_prev",
                  "w_A", "w_B", "phi_A", "phi_B"}


def params():
    return {
        "nx": [16, 16, 16], "lx": [4.0, 4.0, 4.0], "chain_model": "continuous", "ds": 1 / 20,
        "segment_lengths": {"A": 1.0, "B": 1.0}, "chi_n": {"A,B": 17.0},
        "distinct_polymers": [{"volume_fraction": 1.0, "blocks": [{"type": "A", "length": 0.5}, {"type": "B", "length": 0.5}]}],
        "langevin": {"dt": 0.8, "nbar": 100}, "saddle": {"max_iter": 100, "tolerance": 1e-4},
        "am": {"max_hist": 20, "start_error": 5e-1, "mix_min": 0.01, "mix_init": 0.01},
    }


def test_batched_checkpoint_resume(tmp_path):
    from scipy.io import loadmat
    from langevinfts_b200.lfts import BatchedLFTS
    a = BatchedLFTS(params(), random_seeds=[21, 22])
    rng = np.random.Generator(np.random.PCG64(3))
    a.start([{"A": rng.normal(0, 1, a.M), "B": rng.normal(0, 1, a.M)} for _ in range(a.R)])
    a.step()
    a.step()
    paths = [str(tmp_path / f"fields_r{r}.mat") for r in range(a.R)]
    a.save_simulation_data(paths)
    cont = [a.step() for _ in range(3)]
    w_a = a.fields()

    d = loadmat(paths[1], squeeze_me=True)
    assert REFERENCE_KEYS <= set(d)
    assert int(d["langevin_step"]) == 2 and str(d["random_generator"]) == "PCG64"

    b = BatchedLFTS(params(), random_seeds=[0, 0])  # streams come from the files
    b.continue_run(paths)
    assert b.langevin_step == 2
    resumed = [b.step() for _ in range(3)]
    w_b = b.fields()
    for s_a, s_b in zip(cont, resumed):
        assert list(s_a["iterations"]) == list(s_b["iterations"])
        np.testing.assert_allclose(s_b["hamiltonian"], s_a["hamiltonian"], rtol=1e-9)
    assert np.max(np.abs(w_b - w_a)) <= 1e-9 * np.max(np.abs(w_a))
    assert b.langevin_step == a.langevin_step == 5
