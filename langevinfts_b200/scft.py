"""Device-resident SCFT driver.

Takes the params dict of the reference's SCFT driver and runs its iteration
(examples/scft/scft.py:617-736): statistics, self-consistency residual
w_diff_i = sum_j chi_ij phi_j - P_ij w_j, error level, stress-driven box
updates and the Anderson-mixing or Adam step.  The fields, residuals and
optimizer history stay on the device (langevinfts.DeviceScft); only scalars
reach the host each iteration.
"""
import itertools
import re

import numpy as np

from .lfts import SymmetricPolymerTheory


def build_system(params, module, platform):
    """Monomer types, chiN, field theory, factory, box, molecules and analyzer of
    a params dict, through any langevinfts-compatible module."""
    monomer_types = sorted(params["segment_lengths"].keys())
    chi_n = {}
    for pair, v in params["chi_n"].items():
        mp = sorted(re.split(",| |_|/", pair))
        chi_n[mp[0] + "," + mp[1]] = v
    for mp in itertools.combinations(monomer_types, 2):
        chi_n.setdefault(",".join(sorted(mp)), 0.0)
    mpt = SymmetricPolymerTheory(monomer_types, chi_n)
    factory = module.PlatformSelector.create_factory(platform, False)
    cb = factory.create_computation_box(params["nx"], params["lx"])
    molecules = factory.create_molecules_information(params["chain_model"], params["ds"], params["segment_lengths"])
    for polymer in params["distinct_polymers"]:
        blocks = []
        for b in polymer["blocks"]:
            if "v" in b:
                blocks.append([b["type"], b["length"], b["v"], b["u"]])
            else:
                blocks.append([b["type"], b["length"], len(blocks), len(blocks) + 1])
        molecules.add_polymer(polymer["volume_fraction"], blocks)
    analyzer = factory.create_propagator_analyzer(molecules, params.get("aggregate_propagator_computation", True))
    return monomer_types, chi_n, mpt, factory, cb, molecules, analyzer


class SCFT:
    def __init__(self, params, module=None, platform="cuda"):
        if module is None:
            from langevinfts_b200 import langevinfts as module
        self.params = params
        (self.monomer_types, self.chi_n, self.mpt, self.factory, self.cb, self.molecules,
         self.analyzer) = build_system(params, module, platform)
        opt = params.get("optimizer", {"name": "am", "max_hist": 20, "start_error": 1e-2, "mix_min": 0.1, "mix_init": 0.1})
        cfg = {
            "monomer_types": self.monomer_types,
            "matrix_chi": list(np.asarray(self.mpt.matrix_chi, dtype=float).reshape(-1)),
            "matrix_p": list(np.asarray(self.mpt.matrix_p, dtype=float).reshape(-1)),
            "matrix_a_inv": list(np.asarray(self.mpt.matrix_a_inv, dtype=float).reshape(-1)),
            "box_is_altering": bool(params.get("box_is_altering", False)),
            "scale_stress": float(params.get("scale_stress", 1.0)),
            "optimizer": opt["name"],
        }
        if opt["name"] == "am":
            cfg.update({"am_max_hist": int(opt["max_hist"]), "am_start_error": float(opt["start_error"]),
                        "am_mix_min": float(opt["mix_min"]), "am_mix_init": float(opt["mix_init"])})
        else:
            cfg.update({"adam_lr": float(opt.get("lr", 1e-2)), "adam_gamma": float(opt.get("gamma", 1.0))})
        self.engine = module.DeviceScft(self.factory, self.cb, self.molecules, self.analyzer, cfg)
        self.max_iter = int(params.get("max_iter", 2000))
        self.tolerance = float(params.get("tolerance", 1e-8))

    def compute_hamiltonian(self, stats):
        """The SCFT free energy per site (scft.py:206-222) from the field averages
        and partition functions that evaluate() returns."""
        S = len(self.monomer_types)
        h = -stats["aux_mean"][S - 1]
        for i in range(S - 1):
            h += self.mpt.h_coef_mu2[i] * stats["aux_msq"][i] + self.mpt.h_coef_mu1[i] * stats["aux_mean"][i]
        for p in range(self.molecules.get_n_polymer_types()):
            pol = self.molecules.get_polymer(p)
            h -= pol.get_volume_fraction() / pol.get_alpha() * np.log(stats["partitions"][p])
        return h

    def run(self, initial_fields, verbose=False):
        """Iterate from {monomer type: field} until the error level is below the
        tolerance or max_iter iterations have run.  Returns the last iteration's
        statistics with "iterations" and "energy"; phi and w are then in
        self.phi and self.w."""
        M = self.cb.get_n_grid()
        w = np.array([np.reshape(initial_fields[t], M) for t in self.monomer_types], dtype=np.float64)
        self.engine.set_fields(w)
        self.engine.reset()
        history = []
        for it in range(1, self.max_iter + 1):
            st = self.engine.evaluate()
            st["energy"] = self.compute_hamiltonian(st)
            st["iterations"] = it
            history.append((st["error_level"], st["energy"]))
            if verbose:
                print("%8d %12.3E [ %s ] %15.9f %15.7E %s" % (
                    it, st["mass_error"], " ".join("%13.7E" % q for q in st["partitions"]), st["energy"],
                    st["error_level"], "[" + ",".join("%10.7f" % x for x in st["lx"]) + "]" if st["stress"] else ""))
            if st["error_level"] < self.tolerance:
                break
            self.engine.update()
        phi = self.engine.get_concentrations()
        self.phi = {t: phi[i] for i, t in enumerate(self.monomer_types)}
        self.w = self.engine.get_fields()
        st["history"] = history
        return st
