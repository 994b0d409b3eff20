"""Structure function and dH/dchiN of the batched L-FTS engine against the
reference driver's host arithmetic (examples/fts/lfts.py:265-274, 753-767),
evaluated with numpy.fft.rfftn on the fields the engine holds."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def params(nx):
    return {
        "nx": nx, "lx": [0.25 * n for n in nx], "chain_model": "continuous", "ds": 1 / 20,
        "segment_lengths": {"A": 1.0, "B": 1.0}, "chi_n": {"A,B": 15.0},
        "distinct_polymers": [{"volume_fraction": 1.0, "blocks": [{"type": "A", "length": 0.4}, {"type": "B", "length": 0.6}]}],
        "langevin": {"dt": 0.8, "nbar": 100}, "saddle": {"max_iter": 100, "tolerance": 1e-4},
        "am": {"max_hist": 20, "start_error": 5e-1, "mix_min": 0.01, "mix_init": 0.01},
    }


def host_sf(sim, phi, w_aux):
    """One step's <u(k) phi(-k)> of every replica, as lfts.py:757-767 computes it."""
    nx, M, S = list(sim.cb.get_nx()), sim.M, sim.S
    out = {}
    for r in range(sim.R):
        phi_f = [np.fft.rfftn(np.reshape(phi[r, i], nx)) / M for i in range(S)]
        mu_f = []
        for i in range(S):
            mu = np.zeros_like(phi_f[0])
            for k in range(S - 1):
                mu += np.fft.rfftn(np.reshape(w_aux[r, k], nx)) * sim.mpt.matrix_a_inv[k, i] / sim.mpt.eigenvalues[k] / M
            mu_f.append(mu)
        for a, b in sim.sf_pairs():
            key = sim.monomer_types[a] + "," + sim.monomer_types[b]
            out.setdefault(key, []).append(mu_f[a] * np.conj(phi_f[b]))
    return {k: np.array(v) for k, v in out.items()}


@pytest.mark.parametrize("nx", [[16, 12, 10], [24, 24, 24]])
def test_structure_function_and_h_deriv(nx):
    from langevinfts_b200.lfts import BatchedLFTS
    sim = BatchedLFTS(params(nx), random_seeds=[11, 12, 13])
    rng = np.random.Generator(np.random.PCG64(5))
    sim.start([{"A": rng.normal(0, 1, sim.M), "B": rng.normal(0, 1, sim.M)} for _ in range(sim.R)])
    expect = None
    for _ in range(2):
        stats = sim.step()
        w_aux, phi = sim.fields(), sim.engine.get_concentrations(sim.S)
        sim.accumulate_structure_function()
        one = host_sf(sim, phi, w_aux)
        expect = one if expect is None else {k: expect[k] + one[k] for k in one}
        # dH/dchiN from the returned moments against numpy means of the fields
        for r, dH in enumerate(sim.h_deriv_chin(stats)):
            for key in sim.chi_n:
                ref = sim.mpt.h_const_deriv_chin[key]
                for i in range(sim.S - 1):
                    ref += sim.mpt.h_coef_mu2_deriv_chin[key][i] * np.mean(w_aux[r, i] ** 2)
                    ref += sim.mpt.h_coef_mu1_deriv_chin[key][i] * np.mean(w_aux[r, i])
                assert abs(dH[key] - ref) <= 1e-10 * max(1.0, abs(ref))
    got = sim.structure_function(reset=True)
    assert sorted(got) == sorted(expect) == ["A,A", "A,B", "B,B"]
    for key in expect:
        assert got[key].shape == expect[key].shape
        scale = np.max(np.abs(expect[key]))
        assert np.max(np.abs(got[key] - expect[key])) <= 1e-10 * scale, key
    cleared = sim.structure_function(reset=False)
    assert all(np.max(np.abs(v)) == 0.0 for v in cleared.values())


def test_fft_forward_matches_numpy_rfftn():
    """lfts_fft_forward through the C ABI on a batch of fields."""
    import ctypes as C
    from langevinfts_b200.capi import Context, StepJob, check
    for nx in ([16, 12, 10], [64, 64, 64], [5, 4, 3]):
        ctx = Context(nx, precision=8)
        M, Mc = ctx.M, ctx.Mc
        rng = np.random.default_rng(1)
        fields = [rng.normal(0, 1, M) for _ in range(3)]
        specs = [ctx.malloc(Mc * 16) for _ in fields]
        jobs = (StepJob * 3)(*[StepJob(ctx.upload(f), 0, None, 0, None, None, None, sp, None, 0, 0)
                               for f, sp in zip(fields, specs)])
        jp = ctx.upload(np.frombuffer(jobs, dtype=np.uint8))
        check(ctx.lib.lfts_fft_forward(ctx.h, jp, 3))
        for f, sp in zip(fields, specs):
            got = ctx.d2h(sp, (Mc,), np.complex128)
            ref = np.fft.rfftn(np.reshape(f, nx)).reshape(-1)
            assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
        ctx.close()
    ctx32 = Context([8, 8, 8], precision=4)
    assert ctx32.lib.lfts_fft_forward(ctx32.h, C.c_void_p(1), 1) < 0
    ctx32.close()
