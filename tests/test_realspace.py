"""Real-space (Crank-Nicolson) step of the oracle against the reference's own
CPU build (oracle/_ref): the numpy restatement oracle.step_realspace follows
src/platforms/cpu/CpuSolverReal.cpp to round-off on 3D, 2D and 1D boxes with
periodic, reflecting and absorbing walls.  CPU only."""
import numpy as np
import pytest

from oracle import lfts_oracle as orc
from tests import refmod

CASES = [((10, 8, 6), (3.0, 2.5, 2.0), None),
         ((10, 8, 6), (3.0, 2.5, 2.0), ["reflecting", "reflecting", "periodic", "periodic", "absorbing", "absorbing"]),
         ((9, 7, 8), (2.0, 2.5, 3.0), ["absorbing", "absorbing", "reflecting", "reflecting", "reflecting", "absorbing"]),
         ((12, 9), (3.0, 2.5), ["absorbing", "reflecting", "periodic", "periodic"]),
         ((20,), (4.0,), ["reflecting", "absorbing"]), ((20,), (4.0,), None)]


def reference_propagators(nx, lx, bc, w, ds, nseg):
    ref = refmod.load()
    if ref is None:
        pytest.skip("oracle/_ref is not built")
    f = ref.PlatformSelector.create_factory("cpu-mkl", False)
    cb = f.create_computation_box(list(nx), list(lx), bc) if bc else f.create_computation_box(list(nx), list(lx))
    mol = f.create_molecules_information("continuous", ds, {"A": 1.0})
    mol.add_polymer(1.0, [["A", nseg * ds, 0, 1]])
    pa = f.create_propagator_analyzer(mol, False)  # the reference's solver does not keep its analyzer alive
    sol = f.create_realspace_solver(cb, mol, pa)
    sol.compute_statistics({"A": w})
    out = [np.array(sol.get_chain_propagator(0, 0, 1, n)) for n in range(1, nseg + 1)]
    del sol, pa
    return out


@pytest.mark.parametrize("nx,lx,bc", CASES, ids=[f"{len(c[0])}d-{'-'.join(c[2]) if c[2] else 'periodic'}" for c in CASES])
def test_oracle_realspace_step_matches_reference_build(nx, lx, bc):
    M, ds, nseg = int(np.prod(nx)), 0.05, 3
    w = np.random.default_rng(len(nx) * 7 + M).normal(0, 1, M)
    qs = reference_propagators(nx, lx, bc, w, ds, nseg)
    q, e = np.ones(M), np.exp(-w * ds / 2)
    for n in range(nseg):
        q = orc.step_realspace(list(nx), list(lx), q, e, 1.0, ds, bc)
        assert np.max(np.abs(q - qs[n])) <= 1e-13 * np.max(np.abs(qs[n]))
