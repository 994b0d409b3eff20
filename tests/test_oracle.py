"""The CPU oracle: the numpy restatement against the reference's known-answer
values and against the compiled reference itself (oracle/_ref)."""
import json
import os

import numpy as np
import pytest

from oracle import lfts_oracle as orc
from tests import refmod

HERE = os.path.dirname(os.path.abspath(__file__))
KAT = json.load(open(os.path.join(HERE, "golden", "reference_tests.json")))
SCHED = {(c["molecule"]["name"], c["aggregate"]): c for c in json.load(open(os.path.join(HERE, "golden", "schedules.json")))}


def _analyzer_tables(model, ds, bonds, polymers, aggregate):
    ref = refmod.load()
    if ref is None:
        pytest.skip("oracle/_ref not built")
    import subprocess
    lines = ["model " + model, "ds %.17g" % ds, "aggregate %d" % int(aggregate), "streams 4"]
    lines += ["bond %s %.17g" % kv for kv in bonds.items()]
    for vf, blocks in polymers:
        lines.append("polymer %.17g" % vf)
        lines += ["block %s %.17g %d %d" % tuple(b) for b in blocks]
    out = subprocess.run([os.path.join(refmod.ROOT, "oracle", "_ref", "ref_schedule_dump")], input="\n".join(lines) + "\n",
                         capture_output=True, text=True, check=True).stdout
    return json.loads(out)


@pytest.mark.parametrize("case", KAT, ids=[c["name"] for c in KAT])
def test_oracle_matches_reference_known_answers(case):
    aggs = [False, True] if "Branched" in case["name"] else [False]
    for agg in aggs:
        pol = [(1.0, 1.0 * sum(b[1] for b in case["blocks"]))]
        tables = _analyzer_tables(case["model"], case["ds"], case["bond_lengths"], [(1.0, case["blocks"])], agg)
        s = orc.PropagatorSolver(case["nx"], case["lx"], case["model"], case["ds"], case["bond_lengths"], pol, tables)
        s.compute_propagators({"A": np.array(case["w_a"]), "B": np.array(case["w_b"])})
        s.compute_concentrations()
        assert abs(s.Q[0] - case["Q"]) < 1e-7
        assert np.max(np.abs(s.get_total_concentration("A") - case["phi_a"])) < 1e-7
        assert np.max(np.abs(s.get_total_concentration("B") - case["phi_b"])) < 1e-7
        if case["stress"] is not None:
            assert np.max(np.abs(s.compute_stress() - np.array(case["stress"]))) < 1e-7


def _ref_solver(ref, nx, lx, model, ds, bonds, polymers, aggregate, solvents=()):
    f = ref.PlatformSelector.create_factory("cpu-mkl", False)
    cb = f.create_computation_box(nx, lx)
    mol = f.create_molecules_information(model, ds, bonds)
    for vf, blocks in polymers:
        mol.add_polymer(vf, blocks)
    for vf, t in solvents:
        mol.add_solvent(vf, t)
    pa = f.create_propagator_analyzer(mol, aggregate)
    return f, cb, mol, pa, f.create_pseudospectral_solver(cb, mol, pa)


@pytest.mark.parametrize("name,agg", [("TestPseudoBranchedMixtureContinuous3D", True), ("TestPseudoBranchedMixtureDiscrete3D", False),
                                      ("branched_mixture_discrete", True), ("ABA_triblock_discrete", True), ("star9_continuous", True)])
def test_oracle_matches_compiled_reference(name, agg):
    ref = refmod.load()
    if ref is None:
        pytest.skip("oracle/_ref not built")
    mol = SCHED[(name, agg)]["molecule"]
    nx, lx = [6, 5, 4], [3.0, 2.5, 2.0]
    polymers = [(p["vf"], p["blocks"]) for p in mol["polymers"]]
    _, cb, m, pa, solver = _ref_solver(ref, nx, lx, mol["model"], mol["ds"], mol["bonds"], polymers, agg)
    rng = np.random.default_rng(1)
    M = int(np.prod(nx))
    w = {t: rng.normal(0, 1.0, M) for t in mol["bonds"]}
    solver.compute_statistics(w)
    solver.compute_stress()
    alphas = [(p["vf"], sum(b[1] for b in p["blocks"])) for p in mol["polymers"]]
    s = orc.PropagatorSolver(nx, lx, mol["model"], mol["ds"], mol["bonds"], alphas, SCHED[(name, agg)]["reference"])
    s.compute_propagators(w)
    s.compute_concentrations()
    for p in range(len(polymers)):
        assert abs(s.Q[p] / solver.get_total_partition(p) - 1) < 1e-11
    for t in mol["bonds"]:
        r = solver.get_total_concentration(t)
        assert np.max(np.abs(s.get_total_concentration(t) - r)) < 1e-11 * np.max(np.abs(r))
    st_ref = np.array(solver.get_stress())
    assert np.max(np.abs(s.compute_stress() - st_ref)) < 1e-9 * max(np.max(np.abs(st_ref)), 1e-12)


def test_oracle_anderson_mixing_matches_reference():
    ref = refmod.load()
    if ref is None:
        pytest.skip("oracle/_ref not built")
    n = 257
    am_r = ref.PlatformSelector.create_factory("cpu-mkl", False).create_anderson_mixing(n, 5, 0.3, 0.01, 0.1)
    am_o = orc.AndersonMixing(n, 5, 0.3, 0.01, 0.1)
    rng = np.random.default_rng(2)
    w = rng.random(n)
    err_old = 1e20
    for it in range(14):
        d = np.sin(w * (it + 1)) * 0.5 ** it
        err = 1.0 * 0.6 ** it
        a = am_r.calculate_new_fields(w, d, err_old, err)
        b = am_o.calculate_new_fields(w, d, err_old, err)
        assert np.max(np.abs(a - b)) < 1e-12 * max(1.0, np.max(np.abs(a)))
        w, err_old = a, err
