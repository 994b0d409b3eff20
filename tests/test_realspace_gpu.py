"""Real-space (Crank-Nicolson) solver on the GPU (lfts_step_realspace, the
"realspace" method of src/platforms/cpu/CpuSolverReal.cpp and
CudaSolverReal.cu) against the CPU oracle and the reference's own build:
every step to 1e-12, and through the langevinfts API (create_realspace_solver)
Q, concentrations and propagators of a diblock to 1e-10 relative, in 3D, 2D
and 1D boxes with periodic, reflecting and absorbing walls."""
import ctypes as C

import numpy as np
import pytest

from oracle import lfts_oracle as orc
from tests import refmod

pytestmark = pytest.mark.gpu

BC3 = ["reflecting", "reflecting", "periodic", "periodic", "absorbing", "absorbing"]
ENGINE_CASES = [((16, 12, 10), (3.0, 2.5, 2.0), BC3), ((16, 12, 10), (3.0, 2.5, 2.0), None),
                ((64, 64, 64), (7.3, 7.3, 7.3), ["absorbing", "absorbing", "reflecting", "reflecting", "periodic", "periodic"]),
                ((24, 18), (3.0, 2.5), ["absorbing", "reflecting", "periodic", "periodic"]),
                ((40,), (4.0,), ["reflecting", "absorbing"]), ((40,), (4.0,), None)]


def _codes(bc, dim):
    return [orc.BC_CODES[b] for b in bc] if bc else [0] * (2 * dim)


@pytest.mark.parametrize("nx,lx,bc", ENGINE_CASES, ids=["x".join(map(str, c[0])) + ("-" + c[2][0] if c[2] else "-periodic")
                                                         for c in ENGINE_CASES])
def test_step_realspace_matches_oracle(nx, lx, bc):
    from langevinfts_b200.capi import Context, StepJob, check
    ctx = Context(nx, precision=8)
    M, dim, ds, nsteps, njobs = ctx.M, len(nx), 0.02, 3, 3
    rng = np.random.default_rng(5)
    n = ctx.lib.lfts_realspace_table_size(ctx.h)
    dx = (C.c_double * dim)(*[lx[d] / nx[d] for d in range(dim)])
    codes = (C.c_int * (2 * dim))(*_codes(bc, dim))
    tab = np.zeros(n)
    check(ctx.lib.lfts_realspace_tables(ctx.h, 1.3, ds, dim, dx, codes, tab.ctypes.data))
    tdev = ctx.upload(tab)
    jobs, w, q0 = [], [], []
    for j in range(njobs):
        w.append(rng.normal(0, 1.5, M))
        q0.append(1.0 + 0.3 * rng.random(M))
        fac = ctx.malloc(M * 8)
        check(ctx.lib.lfts_field_factors(ctx.h, ctx.upload(w[j]), -ds / 4, fac))
        q = ctx.malloc((nsteps + 1) * M * 8)
        ctx.h2d(q, q0[j])
        jobs.append(StepJob(q, M, q + M * 8, M, fac, tdev, None, ctx.malloc(2 * M * 8)))
    arr = (StepJob * njobs)(*jobs)
    jp = ctx.upload(np.frombuffer(arr, dtype=np.uint8))
    for s in range(nsteps):
        check(ctx.lib.lfts_step_realspace(ctx.h, jp, njobs, s, dim))
    ctx.sync()
    for j in range(njobs):
        got = ctx.d2h(jobs[j].in_, (nsteps + 1, M), np.float64)
        ref, e = q0[j], np.exp(-w[j] * ds / 2)
        for s in range(nsteps):
            ref = orc.step_realspace(list(nx), list(lx), ref, e, 1.3, ds, bc)
            assert np.max(np.abs(got[s + 1] - ref)) <= 1e-12 * (s + 1) * np.max(np.abs(ref)), (j, s)
    ctx.close()


API_CASES = [([16, 12, 10], [3.0, 2.5, 2.0], BC3), ([24, 18], [3.0, 2.5], ["absorbing", "reflecting", "periodic", "periodic"]),
             ([48], [4.0], ["reflecting", "absorbing"]), ([12, 12, 12], [3.0, 3.0, 3.0], None)]


def _solve(module, platform, nx, lx, bc, w, realspace=True):
    f = module.PlatformSelector.create_factory(platform, False)
    cb = f.create_computation_box(nx, lx, bc) if bc else f.create_computation_box(nx, lx)
    mol = f.create_molecules_information("continuous", 1 / 40, {"A": 1.0, "B": 1.2})
    mol.add_polymer(0.7, [["A", 0.4, 0, 1], ["B", 0.6, 1, 2]])
    mol.add_polymer(0.3, [["A", 0.5, 0, 1]])
    pa = f.create_propagator_analyzer(mol, True)
    sol = f.create_realspace_solver(cb, mol, pa) if realspace else f.create_pseudospectral_solver(cb, mol, pa)
    sol.compute_statistics(w)
    out = {"Q": [sol.get_total_partition(p) for p in range(2)],
           "phi": np.array([sol.get_total_concentration(t) for t in ("A", "B")]),
           "q": np.array(sol.get_chain_propagator(0, 1, 2, 10))}
    del sol, pa  # the reference's solver does not keep its analyzer alive
    return out


@pytest.mark.parametrize("nx,lx,bc", API_CASES, ids=[f"{len(c[0])}d" + ("-" + c[2][0] if c[2] else "-periodic") for c in API_CASES])
def test_realspace_solver_matches_reference_build(nx, lx, bc):
    from langevinfts_b200 import langevinfts as L
    ref = refmod.load()
    if ref is None:
        pytest.skip("oracle/_ref is not built")
    M = int(np.prod(nx))
    rng = np.random.default_rng(17)
    w = {"A": rng.normal(0, 1, M), "B": rng.normal(0, 1, M)}
    got, want = _solve(L, "cuda", nx, lx, bc, w), _solve(ref, "cpu-mkl", nx, lx, bc, w)
    np.testing.assert_allclose(got["Q"], want["Q"], rtol=1e-10)
    assert np.max(np.abs(got["phi"] - want["phi"])) <= 1e-10 * np.max(np.abs(want["phi"]))
    assert np.max(np.abs(got["q"] - want["q"])) <= 1e-10 * np.max(np.abs(want["q"]))


def test_realspace_solver_limits():
    """What the reference refuses, refused alike: discrete chains, stress, and
    non-periodic walls for the pseudo-spectral method; FP32 has no real-space
    step here."""
    from langevinfts_b200 import langevinfts as L
    f = L.PlatformSelector.create_factory("cuda", False)
    cb = f.create_computation_box([12, 10, 8], [3.0, 2.5, 2.0], BC3)
    mol = f.create_molecules_information("continuous", 0.05, {"A": 1.0})
    mol.add_polymer(1.0, [["A", 0.5, 0, 1]])
    pa = f.create_propagator_analyzer(mol, True)
    with pytest.raises(RuntimeError, match="pseudo-spectral method only supports periodic"):
        f.create_pseudospectral_solver(cb, mol, pa)
    sol = f.create_realspace_solver(cb, mol, pa)
    sol.compute_statistics({"A": np.zeros(12 * 10 * 8)})
    with pytest.raises(RuntimeError, match="does not support stress"):
        sol.compute_stress()
    dmol = f.create_molecules_information("discrete", 0.05, {"A": 1.0})
    dmol.add_polymer(1.0, [["A", 0.5, 0, 1]])
    with pytest.raises(RuntimeError, match="does not support discrete"):
        f.create_realspace_solver(cb, dmol, f.create_propagator_analyzer(dmol, True))
    f32 = L.PlatformSelector.create_factory("cuda-fp32", False)
    with pytest.raises(RuntimeError, match="FP64"):
        f32.create_realspace_solver(f32.create_computation_box([12, 10, 8], [3.0, 2.5, 2.0], BC3), mol, pa)
    with pytest.raises(RuntimeError, match="invalid boundary condition"):
        f.create_computation_box([8, 8], [2.0, 2.0], ["periodic", "reflecting", "periodic", "periodic"])
