"""The reduce-memory mode (create_factory(platform, True)): every propagator
slice in pinned host memory mapped into the device, read and written in place
by the same kernels, as the reference's memory-saving platform keeps its
slices in pinned host memory (CudaComputationReduceMemoryContinuous.cu:55-80).
Results equal the all-in-HBM mode bit for bit: continuous and discrete
chains, the pseudo-spectral and the real-space method, propagators, Q,
concentrations and stress."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(reduce_memory, model, realspace=False):
    from langevinfts_b200 import langevinfts as L
    f = L.PlatformSelector.create_factory("cuda", reduce_memory)
    nx, lx = [16, 12, 10], [3.0, 2.5, 2.0]
    bc = ["reflecting", "reflecting", "periodic", "periodic", "absorbing", "absorbing"] if realspace else None
    cb = f.create_computation_box(nx, lx, bc) if bc else f.create_computation_box(nx, lx)
    mol = f.create_molecules_information(model, 1 / 30, {"A": 1.0, "B": 1.1})
    mol.add_polymer(0.6, [["A", 0.4, 0, 1], ["B", 0.3, 1, 2], ["A", 0.3, 1, 3]])
    mol.add_polymer(0.4, [["B", 0.5, 0, 1]])
    pa = f.create_propagator_analyzer(mol, True)
    sol = f.create_realspace_solver(cb, mol, pa) if realspace else f.create_pseudospectral_solver(cb, mol, pa)
    rng = np.random.default_rng(3)
    M = int(np.prod(nx))
    sol.compute_statistics({"A": rng.normal(0, 1, M), "B": rng.normal(0, 1, M)})
    out = {"Q": [sol.get_total_partition(p) for p in range(2)],
           "phi": np.array([sol.get_total_concentration(t) for t in ("A", "B")]),
           "q": np.array(sol.get_chain_propagator(0, 1, 2, 5))}
    if not realspace:
        sol.compute_stress()
        out["stress"] = np.array(sol.get_stress())
    return out


@pytest.mark.parametrize("model,realspace", [("continuous", False), ("discrete", False), ("continuous", True)])
def test_reduce_memory_mode_matches_device_mode(model, realspace):
    a, b = _run(False, model, realspace), _run(True, model, realspace)
    for k in a:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
