"""L-FTS trajectories on the GPU against the reference's CPU platform.

The same driver (langevinfts_b200.lfts.LFTS, the arithmetic of the reference's
examples/fts/lfts.py) runs once on the reference build (oracle/_ref) and once
on this package; BatchedLFTS runs several replicas at once.  With identical
PCG64 noise the first Langevin steps agree: saddle iterations exactly,
Hamiltonian and fields to 1e-8 relative (FP64; the saddle loop amplifies
round-off differences of the two FFTs only mildly over a few steps).
"""
import numpy as np
import pytest

from tests import refmod

pytestmark = pytest.mark.gpu


def small_params(max_iter=100):
    return {
        "nx": [16, 16, 16], "lx": [4.0, 4.0, 4.0], "chain_model": "continuous", "ds": 1 / 20,
        "segment_lengths": {"A": 1.0, "B": 1.0}, "chi_n": {"A,B": 17.0},
        "distinct_polymers": [{"volume_fraction": 1.0, "blocks": [{"type": "A", "length": 0.5}, {"type": "B", "length": 0.5}]}],
        "langevin": {"dt": 0.8, "nbar": 100}, "saddle": {"max_iter": max_iter, "tolerance": 1e-4},
        "am": {"max_hist": 20, "start_error": 5e-1, "mix_min": 0.01, "mix_init": 0.01},
    }


def init(seed, M):
    rng = np.random.Generator(np.random.PCG64(seed))
    return {"A": rng.normal(0, 1, M), "B": rng.normal(0, 1, M)}


def ref_run(seed, nsteps, params):
    ref = refmod.load()
    if ref is None:
        pytest.skip("oracle/_ref is not built")
    from langevinfts_b200.lfts import LFTS
    sim = LFTS(params, random_seed=seed, module=ref, platform="cpu-mkl")
    it0, err0 = sim.start(init(seed, sim.M))
    hist = [(it0, err0, None, sim.w_aux.copy())]
    for _ in range(nsteps):
        it, err, h, failed = sim.step()
        hist.append((it, err, h, sim.w_aux.copy(), failed))
    return hist


def test_drop_in_driver_matches_reference():
    from langevinfts_b200 import langevinfts as L
    from langevinfts_b200.lfts import LFTS
    p = small_params()
    ref = ref_run(7, 3, p)
    sim = LFTS(p, random_seed=7, module=L, platform="cuda")
    it0, err0 = sim.start(init(7, sim.M))
    assert it0 == ref[0][0]
    assert np.max(np.abs(sim.w_aux - ref[0][3])) < 1e-8 * np.max(np.abs(ref[0][3]))
    for k in range(1, 4):
        it, err, h, failed = sim.step()
        assert it == ref[k][0], (k, it, ref[k][0])
        assert abs(h / ref[k][2] - 1) < 1e-8
        assert np.max(np.abs(sim.w_aux - ref[k][3])) < 1e-8 * np.max(np.abs(ref[k][3]))


def test_batched_replicas_follow_their_own_reference_trajectories():
    from langevinfts_b200 import langevinfts as L
    from langevinfts_b200.lfts import BatchedLFTS
    p = small_params()
    seeds = [11, 12, 13]
    refs = [ref_run(s, 2, p) for s in seeds]
    sim = BatchedLFTS(p, seeds, module=L)
    st = sim.start([init(s, sim.M) for s in seeds])
    w = sim.fields()
    for r in range(3):
        assert st["iterations"][r] == refs[r][0][0]
        assert np.max(np.abs(w[r] - refs[r][0][3])) < 1e-8 * np.max(np.abs(refs[r][0][3]))
    for k in range(1, 3):
        st = sim.step()
        w = sim.fields()
        for r in range(3):
            assert st["iterations"][r] == refs[r][k][0], (k, r)
            assert abs(st["hamiltonian"][r] / refs[r][k][2] - 1) < 1e-8
            assert np.max(np.abs(w[r] - refs[r][k][3])) < 1e-8 * np.max(np.abs(refs[r][k][3]))


@pytest.mark.parametrize("seeds", [[31, 32, 33, 34], [35]])
def test_device_saddle_control_matches_host_control(seeds):
    """The saddle loop with its per-replica control and Anderson solve on the
    device (lfts_saddle_control, lfts_am_batch_solve; no host round trip inside
    an iteration) gives the iterates of the same loop controlled from the host:
    equal iteration counts, fields and errors to 1e-12.  The device control runs
    twice: polled by the host once per iteration, and as one CUDA graph per
    Langevin step (a conditional WHILE node; Hamiltonian, pressure shift and
    restore on the device).  One replica exercises the step launches without an
    active mask."""
    from langevinfts_b200 import langevinfts as L
    from langevinfts_b200.lfts import BatchedLFTS
    p = small_params()
    runs = []
    for host, graph in ((True, False), (False, False), (False, True)):
        sim = BatchedLFTS(p, seeds, module=L)
        sim.engine.set_host_control(host)
        sim.engine.set_step_graph(graph)
        assert sim.engine.host_control() == host and sim.engine.step_graph() == graph
        st = sim.start([init(s, sim.M) for s in seeds])
        hist = [(list(st["iterations"]), np.array(st["error"]), sim.fields(), None, None)]
        for _ in range(3):
            st = sim.step()
            assert not any(st["failed"])
            hist.append((list(st["iterations"]), np.array(st["error"]), sim.fields(), np.array(st["hamiltonian"]),
                         np.array(st["partitions"])))
        runs.append(hist)
    for other in runs[1:]:
        for (ih, eh, wh, hh, qh), (idv, ed, wd, hd, qd) in zip(runs[0], other):
            assert ih == idv
            np.testing.assert_allclose(ed, eh, rtol=1e-12)
            assert np.max(np.abs(wd - wh)) <= 1e-12 * np.max(np.abs(wh))
            if hh is not None:
                np.testing.assert_allclose(hd, hh, rtol=1e-12)
                np.testing.assert_allclose(qd, qh, rtol=1e-12)


def test_step_graph_split_update_and_search():
    """The two halves of a step (langevin_update_device, then finish_step, the
    route of a learned start) as two graphs give the one-graph step's result."""
    from langevinfts_b200 import langevinfts as L
    from langevinfts_b200.lfts import BatchedLFTS
    p = small_params()
    seeds = [41, 42]
    out = []
    for split in (False, True):
        sim = BatchedLFTS(p, seeds, module=L)
        assert sim.engine.step_graph()
        sim.start([init(s, sim.M) for s in seeds])
        for _ in range(2):
            st = sim.step(start=(lambda s: None) if split else None)
        out.append((list(st["iterations"]), sim.fields(), np.array(st["hamiltonian"])))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])


@pytest.mark.parametrize("graph", [True, False])
def test_failed_saddle_point_restores_fields(graph):
    """max_iter too small: the step fails and the fields go back (lfts.py:713-730),
    with the step as one graph (restore on the device) and driven from the host."""
    from langevinfts_b200 import langevinfts as L
    from langevinfts_b200.lfts import BatchedLFTS, LFTS
    p = small_params()
    seeds = [21, 22]
    sim = BatchedLFTS(p, seeds, module=L)
    sim.start([init(s, sim.M) for s in seeds])
    before = sim.fields()
    # a new engine with max_iter=2 from the converged fields
    p2 = small_params(max_iter=2)
    sim2 = BatchedLFTS(p2, seeds, module=L)
    sim2.engine.set_step_graph(graph)
    sim2.engine.set_fields(before)
    phi2 = sim2.engine.get_concentrations(sim2.S)
    st = sim2.step()
    assert all(st["failed"]) and all(i == 2 for i in st["iterations"])
    assert np.array_equal(sim2.fields(), before)
    assert np.array_equal(sim2.engine.get_concentrations(sim2.S), phi2)
    # the drop-in driver agrees on the failure
    one = LFTS(p2, random_seed=21, module=L)
    one.w_aux = before[0].copy()
    one.phi = {t: np.full(one.M, 0.5) for t in one.monomer_types}
    one.noise_prev = np.zeros([1, one.M])
    _, _, _, failed = one.step()
    assert failed and np.array_equal(one.w_aux, before[0])


def test_two_contexts_with_different_grids_interleave():
    """Kernels are shared by every context: a second, smaller grid must not
    break the first one's launches."""
    from langevinfts_b200 import langevinfts as L
    f = L.PlatformSelector.create_factory("cuda")
    mk = []
    for nx in ([32, 32, 32], [8, 6, 4]):
        cb = f.create_computation_box(nx, [4.0, 3.0, 2.0])
        mol = f.create_molecules_information("continuous", 0.05, {"A": 1.0, "B": 1.0})
        mol.add_polymer(1.0, [["A", 0.5, 0, 1], ["B", 0.5, 1, 2]])
        pa = f.create_propagator_analyzer(mol, True)
        mk.append((f.create_pseudospectral_solver(cb, mol, pa), int(np.prod(nx))))
    am = f.create_anderson_mixing(10, 3, 0.1, 0.01, 0.1)
    rng = np.random.default_rng(0)
    out = []
    for rep in range(2):
        for s, M in mk:
            s.compute_statistics({"A": rng.normal(0, 1, M), "B": rng.normal(0, 1, M)})
            out.append(s.get_total_partition(0))
        am.calculate_new_fields(np.zeros(10), np.ones(10), 1.0, 0.9)
    assert all(np.isfinite(out)) and all(q > 0 for q in out)
