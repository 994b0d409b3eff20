"""Host-side dedup / aggregation / schedule against the reference's own host
code (fixtures from oracle/_ref/ref_schedule_dump, tests/golden/schedules.json).
Exact (string and integer) equality."""
import json
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = json.load(open(os.path.join(HERE, "golden", "schedules.json")))


def _mod():
    from langevinfts_b200 import langevinfts
    return langevinfts


def _build(L, mol, aggregate):
    m = L.Molecules(mol["model"], mol["ds"], mol["bonds"])
    for p in mol["polymers"]:
        m.add_polymer(p["vf"], p["blocks"])
    return m, L.PropagatorAnalyzer if False else None


@pytest.mark.parametrize("case", CASES, ids=[c["molecule"]["name"] + ("-agg" if c["aggregate"] else "") for c in CASES])
def test_analyzer_and_schedule_match_reference(case):
    L = _mod()
    mol = case["molecule"]
    factory = L.PlatformSelector.create_factory("cuda", False)
    m = factory.create_molecules_information(mol["model"], mol["ds"], mol["bonds"])
    for p in mol["polymers"]:
        m.add_polymer(p["vf"], p["blocks"])
    pa = factory.create_propagator_analyzer(m, case["aggregate"])
    ref = case["reference"]
    mine = pa.get_computation_propagators()
    assert [k for k, _ in mine] == [p["key"] for p in ref["propagators"]]
    for (k, e), r in zip(mine, ref["propagators"]):
        assert e["max_n_segment"] == r["max_n_segment"], k
        assert e["monomer_type"] == r["monomer_type"], k
        assert e["height"] == r["height"], k
        assert [list(d) for d in e["deps"]] == r["deps"], k
        assert e["junction_ends"] == r["junction_ends"], k
    blocks = pa.get_computation_blocks()
    assert len(blocks) == len(ref["blocks"])
    for (key, b), r in zip(blocks, ref["blocks"]):
        assert list(key) == [r["polymer"], r["key_left"], r["key_right"]]
        assert b["monomer_type"] == r["monomer_type"]
        assert (b["n_segment_left"], b["n_segment_right"], b["n_repeated"]) == (r["n_segment_left"], r["n_segment_right"], r["n_repeated"])
        assert [list(x) for x in b["v_u"]] == r["v_u"]
    sched = pa.get_schedule(case["n_streams"])
    assert [[list(j) for j in slot] for slot in sched] == ref["schedule"]


def test_polymer_validation_errors():
    L = _mod()
    m = L.Molecules("Continuous", 0.01, {"A": 1.0, "B": 1.0})
    with pytest.raises(Exception, match="is not an integer"):
        m.add_polymer(1.0, [["A", 0.333, 0, 1]])
    with pytest.raises(Exception, match="cycle"):
        m.add_polymer(1.0, [["A", 0.1, 0, 1], ["A", 0.1, 1, 2], ["A", 0.1, 2, 0]])
    with pytest.raises(Exception, match="not in bond_lengths"):
        m.add_polymer(1.0, [["C", 0.1, 0, 1]])
    with pytest.raises(Exception, match="no route"):
        m.add_polymer(1.0, [["A", 0.1, 0, 1], ["A", 0.1, 2, 3]])
    with pytest.raises(Exception, match="invalid chain model"):
        L.Molecules("gaussian", 0.01, {"A": 1.0})


def test_keys_and_polymer_getters():
    L = _mod()
    m = L.Molecules("continuous", 0.01, {"A": 1.0, "B": 2.0})
    m.add_polymer(0.7, [["A", 0.4, 0, 1], ["B", 0.6, 1, 2]])
    pc = m.get_polymer(0)
    assert pc.get_propagator_key(0, 1) == "A"
    assert pc.get_propagator_key(1, 0) == "(B60)A"
    assert pc.get_n_segment_total() == 100
    assert abs(pc.get_alpha() - 1.0) < 1e-15 and pc.get_volume_fraction() == 0.7
    f = L.PlatformSelector.create_factory("cuda")
    pa = f.create_propagator_analyzer(m, True)
    assert pa.get_deps_from_key("[(A4)B2,(C5)B2:3]B") == [("(A4)B", 2, 1), ("(C5)B", 2, 3)]
    assert pa.get_monomer_type_from_key("((A4)B2(C5)B2)B") == "B"


def test_box():
    L = _mod()
    f = L.PlatformSelector.create_factory("cuda")
    cb = f.create_computation_box([4, 5, 6], [2.0, 2.5, 3.0])
    import numpy as np
    g = np.arange(120, dtype=float)
    assert abs(cb.integral(g) - g.sum() * 0.5 ** 3) < 1e-9
    assert cb.get_volume() == 15.0 and cb.get_n_grid() == 120 and cb.get_dim() == 3
    with pytest.raises(Exception, match="must match"):
        cb.integral(np.zeros(7))
    with pytest.raises(Exception, match="not supported"):
        f.create_computation_box([4, 5, 6], [2.0, 2.5, 3.0], mask=np.ones(120))
    assert "cuda" in L.PlatformSelector.avail_platforms()
