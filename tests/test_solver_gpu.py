"""The drop-in `langevinfts` API on the GPU against the reference.

Two anchors: the reference's own known-answer values (tests/golden/
reference_tests.json, tolerance 1e-7 absolute as in the reference tests) and
the reference's CPU build itself (oracle/_ref, loaded through tests/refmod.py),
run on identical seeded inputs.  FP64 bar: relative 1e-10 on Q, concentrations,
stress and propagators.  FP32 platform: relative 1e-5 (Q), 1e-4 (phi, stress).
"""
import json
import os

import numpy as np
import pytest

from tests import refmod

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
KAT = json.load(open(os.path.join(HERE, "golden", "reference_tests.json")))
SCHED = {(c["molecule"]["name"], c["aggregate"]): c["molecule"] for c in json.load(open(os.path.join(HERE, "golden", "schedules.json")))}

RTOL = 1e-10


def mine():
    from langevinfts_b200 import langevinfts
    return langevinfts


def reference():
    r = refmod.load()
    if r is None:
        pytest.skip("oracle/_ref is not built")
    return r


def make(L, platform, nx, lx, model, ds, bonds, polymers, aggregate, solvents=()):
    f = L.PlatformSelector.create_factory(platform, False)
    cb = f.create_computation_box(nx, lx)
    mol = f.create_molecules_information(model, ds, bonds)
    for vf, blocks in polymers:
        mol.add_polymer(vf, blocks)
    for vf, t in solvents:
        mol.add_solvent(vf, t)
    pa = f.create_propagator_analyzer(mol, aggregate)
    return {"f": f, "cb": cb, "mol": mol, "pa": pa, "solver": f.create_pseudospectral_solver(cb, mol, pa)}


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def compare(sys_m, sys_r, types, tol_q=RTOL, tol_phi=RTOL, tol_stress=RTOL, stress=True, edges=()):
    sm, sr = sys_m["solver"], sys_r["solver"]
    P = sys_r["mol"].get_n_polymer_types()
    for p in range(P):
        assert abs(sm.get_total_partition(p) / sr.get_total_partition(p) - 1) < tol_q, p
    for t in types:
        e = rel(sm.get_total_concentration(t), sr.get_total_concentration(t))
        assert e < tol_phi, (t, e)
    for (p, v, u, n) in edges:
        e = rel(sm.get_chain_propagator(p, v, u, n), sr.get_chain_propagator(p, v, u, n))
        assert e < tol_phi, ((p, v, u, n), e)
    if stress:
        sm.compute_stress()
        sr.compute_stress()
        a, b = np.array(sm.get_stress()), np.array(sr.get_stress())
        assert np.max(np.abs(a - b)) <= tol_stress * np.max(np.abs(b)), (a, b)


@pytest.mark.parametrize("case", KAT, ids=[c["name"] for c in KAT])
def test_reference_known_answers(case):
    L, R = mine(), reference()
    for agg in ([False, True] if "Branched" in case["name"] else [False]):
        pol = [(1.0, case["blocks"])]
        sm = make(L, "cuda", case["nx"], case["lx"], case["model"], case["ds"], case["bond_lengths"], pol, agg)
        sr = make(R, "cpu-mkl", case["nx"], case["lx"], case["model"], case["ds"], case["bond_lengths"], pol, agg)
        w = {"A": np.array(case["w_a"]), "B": np.array(case["w_b"])}
        for s in (sm, sr):
            s["solver"].compute_statistics(w)
        s = sm["solver"]
        pc = sm["mol"].get_polymer(0)
        for qref in case["q_refs"]:
            v, u = qref["edge"]
            got = s.get_chain_propagator(0, v, u, pc.get_block(v, u).n_segment)
            assert np.max(np.abs(got - qref["q"])) < 1e-7
        assert abs(s.get_total_partition(0) - case["Q"]) < 1e-7
        assert np.max(np.abs(s.get_total_concentration("A") - case["phi_a"])) < 1e-7
        assert np.max(np.abs(s.get_total_concentration("B") - case["phi_b"])) < 1e-7
        assert s.check_total_partition()
        if case["stress"] is not None:
            s.compute_stress()
            assert np.max(np.abs(np.array(s.get_stress()) - case["stress"])) < 1e-7
        compare(sm, sr, ["A", "B"], edges=[(0, q["edge"][0], q["edge"][1], 1) for q in case["q_refs"]])


def test_config_diblock_32():
    """32^3 AB diblock, f=0.5, N=100, L=4, w ~ Normal(0,1) from PCG64(1)."""
    L, R = mine(), reference()
    mol = SCHED[("diblock_f0.5_N100", True)]
    nx, lx = [32, 32, 32], [4.0, 4.0, 4.0]
    rng = np.random.Generator(np.random.PCG64(1))
    M = 32 ** 3
    w = {"A": rng.normal(0, 1, M), "B": rng.normal(0, 1, M)}
    pol = [(p["vf"], p["blocks"]) for p in mol["polymers"]]
    sm = make(L, "cuda", nx, lx, mol["model"], mol["ds"], mol["bonds"], pol, True)
    sr = make(R, "cpu-mkl", nx, lx, mol["model"], mol["ds"], mol["bonds"], pol, True)
    for s in (sm, sr):
        s["solver"].compute_statistics(w)
    compare(sm, sr, ["A", "B"], edges=[(0, 0, 1, 50), (0, 1, 2, 50), (0, 2, 1, 50), (0, 1, 0, 50), (0, 1, 0, 17)])
    # second call with new fields reuses the captured graph
    w2 = {"A": rng.normal(0, 1, M), "B": rng.normal(0, 1, M)}
    for s in (sm, sr):
        s["solver"].compute_statistics(w2)
    compare(sm, sr, ["A", "B"], stress=False)


def test_config_branched_mixture_48_discrete():
    """48^3 discrete mixture: ABC star, A-B bottlebrush, A homopolymer, Normal(0,2) fields from PCG64(3)."""
    L, R = mine(), reference()
    mol = SCHED[("branched_mixture_discrete", True)]
    nx, lx = [48, 48, 48], [5.0, 5.0, 5.0]
    rng = np.random.Generator(np.random.PCG64(3))
    M = 48 ** 3
    w = {t: rng.normal(0, 2.0, M) for t in ("A", "B", "C")}
    pol = [(p["vf"], p["blocks"]) for p in mol["polymers"]]
    sm = make(L, "cuda", nx, lx, mol["model"], mol["ds"], mol["bonds"], pol, True)
    sr = make(R, "cpu-mkl", nx, lx, mol["model"], mol["ds"], mol["bonds"], pol, True)
    for s in (sm, sr):
        s["solver"].compute_statistics(w)
    compare(sm, sr, ["A", "B", "C"])


@pytest.mark.parametrize("name", ["TestPseudoBranchedMixtureContinuous3D", "TestPseudoBranchedMixtureDiscrete3D",
                                  "ABA_triblock_discrete", "star9_continuous", "TestPseudoBranchedContinuous3D",
                                  "TestPseudoBranchedDiscrete3D"])
@pytest.mark.parametrize("agg", [False, True])
def test_molecules_vs_reference(name, agg):
    L, R = mine(), reference()
    mol = SCHED[(name, agg)]
    nx, lx = [8, 6, 10], [3.0, 2.5, 3.5]
    rng = np.random.default_rng(4)
    w = {t: rng.normal(0, 1.0, int(np.prod(nx))) for t in mol["bonds"]}
    pol = [(p["vf"], p["blocks"]) for p in mol["polymers"]]
    sm = make(L, "cuda", nx, lx, mol["model"], mol["ds"], mol["bonds"], pol, agg)
    sr = make(R, "cpu-mkl", nx, lx, mol["model"], mol["ds"], mol["bonds"], pol, agg)
    for s in (sm, sr):
        s["solver"].compute_statistics(w)
    compare(sm, sr, sorted(mol["bonds"]), tol_stress=1e-9)
    if not agg:
        for p in range(len(pol)):
            assert rel(sm["solver"].get_block_concentration(p), sr["solver"].get_block_concentration(p)) < RTOL


@pytest.mark.parametrize("model", ["continuous", "discrete"])
@pytest.mark.parametrize("dims", [1, 2, 3])
def test_solvent_and_low_dimensions(model, dims):
    L, R = mine(), reference()
    nx = [[40], [24, 20], [10, 12, 9]][dims - 1]
    lx = [[4.0], [3.0, 2.5], [2.5, 3.0, 2.0]][dims - 1]
    ds = 0.05
    bonds = {"A": 1.0, "B": 1.2, "S": 1.0}
    pol = [(0.8, [["A", 0.4, 0, 1], ["B", 0.6, 1, 2]])]
    rng = np.random.default_rng(9)
    w = {t: rng.normal(0, 1.0, int(np.prod(nx))) for t in bonds}
    sm = make(L, "cuda", nx, lx, model, ds, bonds, pol, True, solvents=[(0.2, "S")])
    sr = make(R, "cpu-mkl", nx, lx, model, ds, bonds, pol, True, solvents=[(0.2, "S")])
    for s in (sm, sr):
        s["solver"].compute_statistics(w)
    compare(sm, sr, ["A", "B", "S"], tol_stress=1e-9)
    assert abs(sm["solver"].get_solvent_partition(0) / sr["solver"].get_solvent_partition(0) - 1) < RTOL
    assert rel(sm["solver"].get_solvent_concentration(0), sr["solver"].get_solvent_concentration(0)) < RTOL
    a = sm["solver"].get_total_concentration_gce(1.3, 0, "A")
    b = sr["solver"].get_total_concentration_gce(1.3, 0, "A")
    assert rel(a, b) < RTOL


def test_fp32_platform_error_vs_fp64_reference():
    L, R = mine(), reference()
    mol = SCHED[("diblock_f0.5_N100", True)]
    nx, lx = [32, 32, 32], [4.0, 4.0, 4.0]
    rng = np.random.Generator(np.random.PCG64(1))
    M = 32 ** 3
    w = {"A": rng.normal(0, 1, M), "B": rng.normal(0, 1, M)}
    pol = [(p["vf"], p["blocks"]) for p in mol["polymers"]]
    sm = make(L, "cuda-fp32", nx, lx, mol["model"], mol["ds"], mol["bonds"], pol, True)
    sr = make(R, "cpu-mkl", nx, lx, mol["model"], mol["ds"], mol["bonds"], pol, True)
    for s in (sm, sr):
        s["solver"].compute_statistics(w)
    compare(sm, sr, ["A", "B"], tol_q=1e-5, tol_phi=1e-4, tol_stress=1e-3)


def test_anderson_mixing_vs_reference():
    L, R = mine(), reference()
    n = 5000
    am_m = L.PlatformSelector.create_factory("cuda").create_anderson_mixing(n, 6, 0.3, 0.01, 0.1)
    am_r = R.PlatformSelector.create_factory("cpu-mkl").create_anderson_mixing(n, 6, 0.3, 0.01, 0.1)
    rng = np.random.default_rng(2)
    for trial in range(2):
        am_m.reset_count()
        am_r.reset_count()
        w = rng.random(n)
        err_old = 1e20
        for it in range(16):
            d = np.sin(w * (it + 1)) * 0.7 ** it
            err = 0.9 * 0.65 ** it
            a = am_m.calculate_new_fields(w, d, err_old, err)
            b = am_r.calculate_new_fields(w, d, err_old, err)
            assert rel(a, b) < 1e-10, (trial, it, rel(a, b))
            w, err_old = b, err


def test_box_relaxation_scft_iterations():
    """A few SCFT iterations with stress-driven box updates (scft.py:617-736 logic)
    run through both modules: fields, box and free energy stay together."""
    L, R = mine(), reference()
    nx, lx0, ds, f = [16, 16, 16], [3.6, 3.6, 3.6], 0.01, 0.36
    bonds = {"A": 1.0, "B": 1.0}
    pol = [(1.0, [["A", f, 0, 1], ["B", 1 - f, 1, 2]])]
    chin = 20.0
    M = int(np.prod(nx))
    x = np.arange(nx[0]) * 2 * np.pi / nx[0]
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    g = (np.sin(X) * np.cos(Y) + np.sin(Y) * np.cos(Z) + np.sin(Z) * np.cos(X)).reshape(-1)
    rng = np.random.Generator(np.random.PCG64(2))
    w0 = np.array([chin * g + 0.1 * rng.normal(0, 1, M), -chin * g + 0.1 * rng.normal(0, 1, M)])
    runs = []
    for mod, plat in ((L, "cuda"), (R, "cpu-mkl")):
        s = make(mod, plat, nx, lx0, "continuous", ds, bonds, pol, True)
        am = s["f"].create_anderson_mixing(2 * M + 3, 20, 1e-1, 0.1, 0.1)
        w = w0.copy()
        hist = []
        err_old = 1e20
        for it in range(12):
            s["solver"].compute_statistics({"A": w[0], "B": w[1]})
            phi = [s["solver"].get_total_concentration(t) for t in "AB"]
            wd = np.array([chin * phi[1] - 0.5 * (w[0] - w[1]), chin * phi[0] - 0.5 * (w[1] - w[0])])
            wd -= wd.mean(axis=1, keepdims=True)
            s["solver"].compute_stress()
            st = np.array(s["solver"].get_stress())
            err = np.sqrt(np.sum(wd ** 2) / (1 + np.sum(w ** 2))) + np.sqrt(np.sum(st ** 2))
            hist.append((s["solver"].get_total_partition(0), err, np.array(s["cb"].get_lx())))
            cur = np.concatenate([w.reshape(-1), s["cb"].get_lx()])
            dif = np.concatenate([wd.reshape(-1), -0.1 * st])
            new = am.calculate_new_fields(cur, dif, err_old, err)
            err_old = err
            w = new[:2 * M].reshape(2, M)
            old = np.array(s["cb"].get_lx())
            lx = (1 + np.clip((new[-3:] - old) / old, -0.1, 0.1)) * old
            s["cb"].set_lx(list(lx))
            s["solver"].update_laplacian_operator()
            w -= w.mean(axis=1, keepdims=True)
        runs.append(hist)
    for (qm, em, lm), (qr, er, lr) in zip(*runs):
        assert abs(qm / qr - 1) < 1e-9 and abs(em / er - 1) < 1e-8 and np.max(np.abs(lm - lr)) < 1e-10
