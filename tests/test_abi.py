"""The C ABI library loads and exports every entry point include/lfts_b200.h
declares (no GPU work is done here)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "lfts_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lfts_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    assert "lfts_step_continuous" in names and "lfts_stress" in names and len(names) >= 30


def test_library_exports_every_declared_symbol():
    from langevinfts_b200 import capi
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(set(capi.declared_symbols())) == declared()


def test_pybind_module_surface():
    from langevinfts_b200 import langevinfts as L
    for cls, methods in {
        "PropagatorComputation": ["compute_propagators", "compute_concentrations", "compute_statistics", "get_total_concentration",
                                  "get_total_concentration_gce", "get_block_concentration", "get_total_partition",
                                  "get_solvent_partition", "get_solvent_concentration", "get_chain_propagator", "compute_stress",
                                  "get_stress", "get_stress_gce", "check_total_partition", "update_laplacian_operator"],
        "AndersonMixing": ["reset_count", "calculate_new_fields"],
        "AbstractFactory": ["create_computation_box", "create_molecules_information", "create_propagator_analyzer",
                            "create_pseudospectral_solver", "create_realspace_solver", "create_anderson_mixing", "display_info",
                            "get_model_name", "create_array"],
        "ComputationBox": ["get_dim", "get_nx", "get_lx", "get_dx", "get_dv", "get_n_grid", "get_volume", "set_lx", "integral",
                           "inner_product"],
        "PropagatorAnalyzer": ["get_computation_propagators()", "get_computation_propagator", "get_computation_blocks",
                               "get_computation_block", "display_propagators", "display_blocks", "get_deps_from_key",
                               "get_monomer_type_from_key"],
        "Molecules": ["get_model_name", "get_ds", "get_bond_lengths", "get_n_polymer_types", "add_polymer", "get_polymer",
                      "get_n_solvent_types", "add_solvent"],
        "PlatformSelector": ["avail_platforms", "create_factory"],
    }.items():
        c = getattr(L, cls)
        for m in methods:
            assert hasattr(c, m), (cls, m)
