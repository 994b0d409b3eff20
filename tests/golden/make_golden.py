"""Generate the committed golden fixtures of tests/golden/ (run here, not on the GPU box).

  reference_tests.json  inputs and expected values of the reference's own
                        known-answer tests (TestPseudoLinear{Continuous,Discrete}3D,
                        TestPseudoBranched{Continuous,Discrete}3D), read from
                        the test sources as text
  schedules.json        propagator table, computation blocks and stream
                        schedule produced by the reference's own host code
                        (oracle/_ref/ref_schedule_dump) for a set of molecules

Usage:  python tests/golden/make_golden.py /path/to/reference
        (or set LFTS_REFERENCE to the reference checkout)
Needs the oracle build (make -C oracle).
"""
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LFTS_REFERENCE", "")
if not REF:
    raise SystemExit("usage: make_golden.py <reference checkout> (or set LFTS_REFERENCE)")
DUMP = os.path.join(ROOT, "oracle", "_ref", "ref_schedule_dump")

NUM = r"[-+]?\d*\.?\d+(?:[eE][-+]?\d+)?"


def read(name):
    with open(os.path.join(REF, "tests", name)) as f:
        return f.read()


def array(src, name):
    m = re.search(r"double\s+" + re.escape(name) + r"\[M\]\s*=\s*\{(.*?)\};", src, re.S)
    return [float(x) for x in re.findall(NUM, m.group(1))]


def block_lists(src):
    out = {}
    for m in re.finditer(r"std::vector<BlockInput>\s+(\w+)\s*=\s*\{(.*?)\};", src, re.S):
        blocks = []
        for b in re.finditer(r"\{\s*\"(\w+)\"\s*,\s*(" + NUM + r")\s*,\s*(\d+)\s*,\s*(\d+)\s*\}", m.group(2)):
            blocks.append([b.group(1), float(b.group(2)), int(b.group(3)), int(b.group(4))])
        out[m.group(1)] = blocks
    return out


def bond_lengths(src):
    m = re.search(r"bond_lengths\s*=\s*\{(.*?)\};", src, re.S)
    return {k: float(v) for k, v in re.findall(r"\{\"(\w+)\"\s*,\s*(" + NUM + r")\}", m.group(1))}


def known_answer_tests():
    cases = []
    spec = [
        ("TestPseudoLinearContinuous3D.cpp", "continuous", 1.0 / 4, ["q1_last_ref", "q2_last_ref"], [(1, 2), (1, 0)]),
        ("TestPseudoLinearDiscrete3D.cpp", "discrete", None, ["q1_last_ref", "q2_last_ref"], [(1, 2), (1, 0)]),
        ("TestPseudoBranchedContinuous3D.cpp", "continuous", 0.15, ["q_1_4_last_ref", "q_1_0_last_ref"], [(1, 4), (1, 0)]),
        ("TestPseudoBranchedDiscrete3D.cpp", "discrete", 0.15, ["q_1_4_last_ref", "q_1_0_last_ref"], [(1, 4), (1, 0)]),
    ]
    for fname, model, ds, qnames, edges in spec:
        src = read(fname)
        if ds is None:  # discrete linear test: ds = 1.0/N with const int N
            ds = 1.0 / int(re.search(r"const int N\{(\d+)\}", src).group(1))
        nx = [int(re.search(r"const int %s\{(\d+)\}" % k, src).group(1)) for k in ("II", "JJ", "KK")]
        lx = [float(re.search(r"%s = (%s);" % (k, NUM), src).group(1)) for k in ("Lx", "Ly", "Lz")]
        blocks = block_lists(src)["blocks"]
        if "f = " in src and any(isinstance(b[1], float) for b in blocks):
            pass
        m = re.search(r"std::vector<BlockInput> blocks\s*=\s*\{(.*?)\};", src, re.S)
        if re.search(r"\{\"A\",\s*f,", m.group(1)):  # linear tests use {"A", f, 0, 1}, {"B", 1.0-f, 1, 2}
            f = float(re.search(r"\bf = (%s);" % NUM, src).group(1))
            blocks = [["A", f, 0, 1], ["B", 1.0 - f, 1, 2]]
        Q = float(re.search(r"std::abs\(QQ-(%s)/\(Lx\*Ly\*Lz\)\)" % NUM, src).group(1)) / (lx[0] * lx[1] * lx[2])
        stress = [None, None, None]
        for d, v in re.findall(r"std::abs\(stress\[(\d)\] \+ (%s)\)" % NUM, src):
            stress[int(d)] = -float(v)
        cases.append({
            "name": fname[:-4], "model": model, "ds": ds, "nx": nx, "lx": lx,
            "bond_lengths": bond_lengths(src), "blocks": blocks,
            "w_a": array(src, "w_a"), "w_b": array(src, "w_b"),
            "q_refs": [{"edge": list(e), "q": array(src, q)} for q, e in zip(qnames, edges)],
            "phi_a": array(src, "phi_a_ref"), "phi_b": array(src, "phi_b_ref"),
            "Q": Q, "stress": stress if stress[0] is not None else None,
        })
    return cases


def mixture_molecules():
    out = []
    for fname, model in (("TestPseudoBranchedMixtureContinuous3D.cpp", "continuous"),
                         ("TestPseudoBranchedMixtureDiscrete3D.cpp", "discrete")):
        src = read(fname)
        lists = block_lists(src)
        vfs = [float(x) for x in re.findall(r"volume_fraction\.push_back\((%s)\)" % NUM, src)]
        polys = [v for k, v in lists.items() if k.startswith("block_input")]
        out.append({"name": fname[:-4], "model": model, "ds": 0.15, "bonds": bond_lengths(src),
                    "polymers": [{"vf": vf, "blocks": b} for vf, b in zip(vfs, polys)]})
    return out


def config_molecules():
    """Schedule fixtures: the benchmark diblocks (N 100 and 90, conformationally
    asymmetric f 0.36), a discrete branched mixture, an ABA triblock blend and
    a nine-arm star."""
    eps = 1.2
    f2 = 0.36
    bb = [["B", 5 / 60, i, i + 1] for i in range(8)] + [["A", 6 / 60, i, 8 + i] for i in range(1, 9)]
    return [
        {"name": "diblock_f0.5_N100", "model": "continuous", "ds": 0.01, "bonds": {"A": 1.0, "B": 1.0},
         "polymers": [{"vf": 1.0, "blocks": [["A", 0.5, 0, 1], ["B", 0.5, 1, 2]]}]},
        {"name": "diblock_f0.36_N100_eps1.2", "model": "continuous", "ds": 0.01,
         "bonds": {"A": (eps * eps / (eps * eps * f2 + (1 - f2))) ** 0.5, "B": (1.0 / (eps * eps * f2 + (1 - f2))) ** 0.5},
         "polymers": [{"vf": 1.0, "blocks": [["A", 0.36, 0, 1], ["B", 0.64, 1, 2]]}]},
        {"name": "branched_mixture_discrete", "model": "discrete", "ds": 1 / 60, "bonds": {"A": 1.0, "B": 1.0, "C": 1.0},
         "polymers": [{"vf": 0.5, "blocks": [["A", 20 / 60, 0, 1], ["B", 20 / 60, 0, 2], ["C", 20 / 60, 0, 3]]},
                      {"vf": 0.3, "blocks": bb},
                      {"vf": 0.2, "blocks": [["A", 30 / 60, 0, 1]]}]},
        {"name": "diblock_f0.5_N90", "model": "continuous", "ds": 1 / 90, "bonds": {"A": 1.0, "B": 1.0},
         "polymers": [{"vf": 1.0, "blocks": [["A", 0.5, 0, 1], ["B", 0.5, 1, 2]]}]},
        {"name": "diblock_f0.4_N90", "model": "continuous", "ds": 1 / 90, "bonds": {"A": 1.0, "B": 1.0},
         "polymers": [{"vf": 1.0, "blocks": [["A", 0.4, 0, 1], ["B", 0.6, 1, 2]]}]},
        {"name": "ABA_triblock_discrete", "model": "discrete", "ds": 1 / 20, "bonds": {"A": 1.0, "B": 1.3},
         "polymers": [{"vf": 0.7, "blocks": [["A", 0.25, 0, 1], ["B", 0.5, 1, 2], ["A", 0.25, 2, 3]]},
                      {"vf": 0.3, "blocks": [["A", 0.5, 0, 1]]}]},
        {"name": "star9_continuous", "model": "continuous", "ds": 1 / 40, "bonds": {"A": 1.0, "B": 1.0},
         "polymers": [{"vf": 1.0, "blocks": [["A" if i % 2 else "B", 0.25 + 0.025 * (i % 3), 0, i + 1] for i in range(9)]}]},
    ]


def reference_molecules():
    mols = config_molecules() + mixture_molecules()
    for fname, model in (("TestPseudoBranchedContinuous3D.cpp", "continuous"), ("TestPseudoBranchedDiscrete3D.cpp", "discrete")):
        src = read(fname)
        mols.append({"name": fname[:-4], "model": model, "ds": 0.15, "bonds": bond_lengths(src),
                     "polymers": [{"vf": 1.0, "blocks": block_lists(src)["blocks"]}]})
    return mols


def dump(mol, aggregate, streams=4):
    lines = ["model " + mol["model"], "ds %.17g" % mol["ds"], "aggregate %d" % int(aggregate), "streams %d" % streams]
    for k, v in mol["bonds"].items():
        lines.append("bond %s %.17g" % (k, v))
    for p in mol["polymers"]:
        lines.append("polymer %.17g" % p["vf"])
        for b in p["blocks"]:
            lines.append("block %s %.17g %d %d" % (b[0], b[1], b[2], b[3]))
    r = subprocess.run([DUMP], input="\n".join(lines) + "\n", capture_output=True, text=True, check=True)
    return json.loads(r.stdout)


def main():
    with open(os.path.join(HERE, "reference_tests.json"), "w") as f:
        json.dump(known_answer_tests(), f)
    sched = []
    for mol in reference_molecules():
        for agg in (False, True):
            sched.append({"molecule": mol, "aggregate": agg, "n_streams": 4, "reference": dump(mol, agg)})
    with open(os.path.join(HERE, "schedules.json"), "w") as f:
        json.dump(sched, f)
    print("wrote", len(sched), "schedule cases")


if __name__ == "__main__":
    main()
