// pybind11 module `langevinfts`: the reference's Python-facing API
// (src/pybind11/langevinfts.cpp:24-463) over the B200 engine.
// Same class and method names, argument meaning, size checks and errors; the
// platform is "cuda" (FP64) or "cuda-fp32" (FP32 propagators and FFTs, FP64
// reductions).
#include <pybind11/numpy.h>
#include <pybind11/complex.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <iostream>

#include "lfts_computation.h"
#include "lfts_host.h"
#include "lfts_langevin.h"
#include "lfts_scft.h"

namespace py = pybind11;
using namespace lfts;

namespace {

struct Factory {
    int precision = 8;
    bool reduce_memory = false;
    int device = 0;
    std::string name = "cuda";
};

struct PlatformSelector {
    static std::vector<std::string> avail_platforms() { return {"cuda", "cuda-fp32"}; }
    static Factory *create_factory(const std::string &platform, bool reduce_memory) {
        Factory *f = new Factory();
        if (platform == "cuda") {
            f->precision = 8;
        } else if (platform == "cuda-fp32") {
            f->precision = 4;
        } else {
            delete f;
            LFTS_THROW("Could not find platform '" + platform + "'");
        }
        f->name = platform;
        f->reduce_memory = reduce_memory;
        return f;
    }
};

void size_check(const py::buffer_info &b, long long n, const std::string &what, const std::string &against) {
    if (b.size != n)
        throw std::runtime_error("Size of input " + what + "(" + std::to_string(b.size) + ") and '" + against + "' (" +
                                 std::to_string(n) + ") must match");
}

std::map<std::string, const double *> field_map(std::map<std::string, py::array_t<double, py::array::c_style | py::array::forcecast>> &in,
                                                long long M, const char *tag) {
    std::map<std::string, const double *> out;
    for (auto &kv : in) {
        py::buffer_info b = kv.second.request();
        size_check(b, M, std::string(tag) + "[" + kv.first + "] ", "n_grid");
        out[kv.first] = (const double *)b.ptr;
    }
    return out;
}

using Arr = py::array_t<double, py::array::c_style | py::array::forcecast>;

}  // namespace

static py::dict stats_dict(const lfts::SaddleStats &s) {
    py::dict d;
    d["iterations"] = s.iterations; d["error"] = s.error; d["hamiltonian"] = s.hamiltonian;
    d["failed"] = s.failed; d["partitions"] = s.partitions;
    d["aux_mean"] = s.aux_mean; d["aux_msq"] = s.aux_msq;
    return d;
}

PYBIND11_MODULE(langevinfts, m) {
    m.doc() = "langevinfts chain-propagator solver on NVIDIA B200 (sm_100a)";

    py::class_<ComputationBox>(m, "ComputationBox")
        .def("get_dim", &ComputationBox::get_dim)
        .def("get_nx", py::overload_cast<>(&ComputationBox::get_nx, py::const_))
        .def("get_nx", py::overload_cast<int>(&ComputationBox::get_nx, py::const_))
        .def("get_lx", py::overload_cast<>(&ComputationBox::get_lx, py::const_))
        .def("get_lx", py::overload_cast<int>(&ComputationBox::get_lx, py::const_))
        .def("get_dx", py::overload_cast<>(&ComputationBox::get_dx, py::const_))
        .def("get_dx", py::overload_cast<int>(&ComputationBox::get_dx, py::const_))
        .def("get_dv", &ComputationBox::get_dv)
        .def("get_n_grid", &ComputationBox::get_n_grid)
        .def("get_volume", &ComputationBox::get_volume)
        .def("set_lx", &ComputationBox::set_lx)
        .def("integral", [](ComputationBox &cb, Arr g) {
            py::buffer_info b = g.request();
            size_check(b, cb.get_n_grid(), "", "n_grid");
            return cb.integral((const double *)b.ptr);
        })
        .def("inner_product", [](ComputationBox &cb, Arr g, Arr h) {
            py::buffer_info bg = g.request(), bh = h.request();
            size_check(bg, cb.get_n_grid(), "", "n_grid");
            size_check(bh, cb.get_n_grid(), "", "n_grid");
            return cb.inner_product((const double *)bg.ptr, (const double *)bh.ptr);
        });

    py::class_<Block>(m, "Block")
        .def_readonly("monomer_type", &Block::monomer_type)
        .def_readonly("n_segment", &Block::n_segment)
        .def_readonly("contour_length", &Block::contour_length)
        .def_readonly("v", &Block::v)
        .def_readonly("u", &Block::u);

    py::class_<Polymer>(m, "Polymer")
        .def("get_alpha", &Polymer::get_alpha)
        .def("get_volume_fraction", &Polymer::get_volume_fraction)
        .def("get_n_blocks", &Polymer::get_n_blocks)
        .def("get_blocks", &Polymer::get_blocks, py::return_value_policy::reference_internal)
        .def("get_block", &Polymer::get_block, py::return_value_policy::reference_internal)
        .def("get_n_segment_total", &Polymer::get_n_segment_total)
        .def("get_n_segment", &Polymer::get_n_segment)
        .def("get_block_index_from_edge", &Polymer::get_block_index_from_edge)
        .def("get_adjacent_nodes", &Polymer::get_adjacent_nodes)
        .def("get_block_indexes", &Polymer::get_block_indexes)
        .def("get_propagator_key", &Polymer::get_propagator_key);

    auto blocks_from_py = [](const std::vector<std::vector<py::object>> &list) {
        std::vector<BlockInput> out;
        for (const auto &b : list) {
            if (b.size() < 4) throw std::runtime_error("each block must be [monomer_type, contour_length, v, u]");
            out.push_back({py::cast<std::string>(b[0]), py::cast<double>(b[1]), py::cast<int>(b[2]), py::cast<int>(b[3])});
        }
        return out;
    };
    py::class_<Molecules>(m, "Molecules")
        .def(py::init<std::string, double, std::map<std::string, double>>())
        .def("get_model_name", &Molecules::get_model_name)
        .def("get_ds", &Molecules::get_ds)
        .def("get_bond_lengths", &Molecules::get_bond_lengths)
        .def("get_n_polymer_types", &Molecules::get_n_polymer_types)
        .def("add_polymer", [blocks_from_py](Molecules &mol, double vf, std::vector<std::vector<py::object>> blocks) {
            mol.add_polymer(vf, blocks_from_py(blocks), {});
        })
        .def("add_polymer", [blocks_from_py](Molecules &mol, double vf, std::vector<std::vector<py::object>> blocks,
                                             std::map<int, std::string> q_init) {
            mol.add_polymer(vf, blocks_from_py(blocks), q_init);
        })
        .def("get_polymer", &Molecules::get_polymer, py::return_value_policy::reference_internal)
        .def("get_n_solvent_types", &Molecules::get_n_solvent_types)
        .def("add_solvent", &Molecules::add_solvent);

    auto edge_dict = [](const ComputationEdge &e) {
        py::dict d;
        d["max_n_segment"] = e.max_n_segment;
        d["monomer_type"] = e.monomer_type;
        d["deps"] = e.deps;
        d["height"] = e.height;
        d["junction_ends"] = std::vector<int>(e.junction_ends.begin(), e.junction_ends.end());
        return d;
    };
    auto block_dict = [](const ComputationBlock &b) {
        py::dict d;
        d["monomer_type"] = b.monomer_type;
        d["n_segment_left"] = b.n_segment_left;
        d["n_segment_right"] = b.n_segment_right;
        d["n_repeated"] = b.n_repeated;
        d["v_u"] = b.v_u;
        return d;
    };
    py::class_<PropagatorAnalyzer>(m, "PropagatorAnalyzer")
        .def("get_computation_propagators()", [edge_dict](PropagatorAnalyzer &pa) {
            py::list out;  // keeps the analyzer's key order
            for (const auto &it : pa.get_computation_propagators()) out.append(py::make_tuple(it.first, edge_dict(it.second)));
            return out;
        })
        .def("get_computation_propagators", [edge_dict](PropagatorAnalyzer &pa) {
            py::list out;
            for (const auto &it : pa.get_computation_propagators()) out.append(py::make_tuple(it.first, edge_dict(it.second)));
            return out;
        })
        .def("get_computation_propagator", [edge_dict](PropagatorAnalyzer &pa, const std::string &key) {
            return edge_dict(pa.get_computation_propagator(key));
        })
        .def("get_computation_blocks", [block_dict](PropagatorAnalyzer &pa) {
            py::list out;
            for (const auto &it : pa.get_computation_blocks()) out.append(py::make_tuple(it.first, block_dict(it.second)));
            return out;
        })
        .def("get_computation_block", [block_dict](PropagatorAnalyzer &pa, std::tuple<int, std::string, std::string> key) {
            return block_dict(pa.get_computation_block(key));
        })
        .def("display_propagators", &PropagatorAnalyzer::display_propagators)
        .def("display_blocks", &PropagatorAnalyzer::display_blocks)
        .def("get_deps_from_key", [](PropagatorAnalyzer &, const std::string &key) { return code::deps_from_key(key); })
        .def("get_monomer_type_from_key", [](PropagatorAnalyzer &, const std::string &key) { return code::monomer_type_from_key(key); })
        .def("get_schedule", [](PropagatorAnalyzer &pa, int n_streams) {
            Scheduler s(pa.get_computation_propagators(), n_streams);
            return s.get_schedule();
        }, py::arg("n_streams") = 4);

    py::class_<GpuComputation>(m, "PropagatorComputation")
        .def("update_laplacian_operator", &GpuComputation::update_laplacian_operator)
        .def("compute_propagators", [](GpuComputation &c, std::map<std::string, Arr> w, py::object q_init) {
            const long long M = c.get_n_grid();
            auto wm = field_map(w, M, "w");
            std::map<std::string, Arr> qi;
            if (!q_init.is_none()) qi = q_init.cast<std::map<std::string, Arr>>();
            auto qm = field_map(qi, M, "q");
            py::gil_scoped_release nogil;
            c.compute_propagators(wm, qm);
        }, py::arg("w_input"), py::arg("q_init") = py::none())
        .def("compute_concentrations", [](GpuComputation &c) {
            py::gil_scoped_release nogil;
            c.compute_concentrations();
        })
        .def("compute_statistics", [](GpuComputation &c, std::map<std::string, Arr> w, py::object q_init) {
            const long long M = c.get_n_grid();
            auto wm = field_map(w, M, "w");
            std::map<std::string, Arr> qi;
            if (!q_init.is_none()) qi = q_init.cast<std::map<std::string, Arr>>();
            auto qm = field_map(qi, M, "q");
            py::gil_scoped_release nogil;
            c.compute_statistics(wm, qm);
        }, py::arg("w_input"), py::arg("q_init") = py::none())
        .def("get_total_concentration", [](GpuComputation &c, const std::string &type) {
            py::array_t<double> phi(c.get_n_grid());
            c.get_total_concentration(type, (double *)phi.request().ptr);
            return phi;
        })
        .def("get_total_concentration", [](GpuComputation &c, int p, const std::string &type) {
            py::array_t<double> phi(c.get_n_grid());
            c.get_total_concentration(p, type, (double *)phi.request().ptr);
            return phi;
        })
        .def("get_total_concentration_gce", [](GpuComputation &c, double fugacity, int p, const std::string &type) {
            py::array_t<double> phi(c.get_n_grid());
            c.get_total_concentration_gce(fugacity, p, type, (double *)phi.request().ptr);
            return phi;
        })
        .def("get_block_concentration", [](GpuComputation &c, int p) {
            py::array_t<double> phi({(py::ssize_t)c.get_n_blocks(p), (py::ssize_t)c.get_n_grid()});
            c.get_block_concentration(p, (double *)phi.request().ptr);
            return phi;
        })
        .def("get_total_partition", &GpuComputation::get_total_partition)
        .def("get_solvent_partition", &GpuComputation::get_solvent_partition)
        .def("get_solvent_concentration", [](GpuComputation &c, int s) {
            py::array_t<double> phi(c.get_n_grid());
            c.get_solvent_concentration(s, (double *)phi.request().ptr);
            return phi;
        })
        .def("get_chain_propagator", [](GpuComputation &c, int p, int v, int u, int n) {
            py::array_t<double> q(c.get_n_grid());
            c.get_chain_propagator((double *)q.request().ptr, p, v, u, n);
            return q;
        })
        .def("compute_stress", [](GpuComputation &c) {
            py::gil_scoped_release nogil;
            c.compute_stress();
        })
        .def("get_stress", &GpuComputation::get_stress)
        .def("get_stress_gce", &GpuComputation::get_stress_gce)
        .def("check_total_partition", &GpuComputation::check_total_partition)
        .def("get_n_grid", &GpuComputation::get_n_grid)
        .def("get_precision", &GpuComputation::get_precision);

    py::class_<GpuAndersonMixing>(m, "AndersonMixing")
        .def("reset_count", &GpuAndersonMixing::reset_count)
        .def("get_n_var", &GpuAndersonMixing::get_n_var)
        .def("calculate_new_fields", [](GpuAndersonMixing &am, Arr w_current, Arr w_deriv, double old_err, double err) {
            const long long n = am.get_n_var();
            py::array_t<double> w_new(n);
            py::buffer_info bc = w_current.request(), bd = w_deriv.request();
            size_check(bc, n, "w_current ", "n_var");
            size_check(bd, n, "w_deriv ", "n_var");
            double *out = (double *)w_new.request().ptr;
            {
                py::gil_scoped_release nogil;
                am.calculate_new_fields(out, (const double *)bc.ptr, (const double *)bd.ptr, old_err, err);
            }
            return w_new;
        });

    py::class_<Factory>(m, "AbstractFactory")
        .def("create_array", [](Factory &, unsigned int) -> py::object {
            throw std::runtime_error("Array is not part of this module (the solver API works on numpy arrays)");
        })
        .def("create_computation_box", [](Factory &, std::vector<int> nx, std::vector<double> lx, py::object bc, py::object mask) {
            std::vector<std::string> bcv;
            if (!bc.is_none()) bcv = bc.cast<std::vector<std::string>>();
            if (!mask.is_none()) throw std::runtime_error("mask (impenetrable regions) is not supported by this module");
            return new ComputationBox(nx, lx, bcv);
        }, py::arg("nx"), py::arg("lx"), py::arg("bc") = py::none(), py::arg("mask") = py::none())
        .def("create_molecules_information", [](Factory &, std::string model, double ds, std::map<std::string, double> bonds) {
            return new Molecules(model, ds, bonds);
        })
        .def("create_propagator_analyzer", [](Factory &, Molecules *mol, bool aggregate) {
            return new PropagatorAnalyzer(mol, aggregate);
        }, py::keep_alive<0, 2>())
        .def("create_pseudospectral_solver", [](Factory &f, ComputationBox *cb, Molecules *mol, PropagatorAnalyzer *pa) {
            if (pa->get_model_name() != mol->get_model_name())
                throw std::runtime_error("molecules and propagator analyzer use different chain models");
            return new GpuComputation(cb, mol, pa, f.precision, f.device, 1, "pseudospectral", f.reduce_memory);
        }, py::keep_alive<0, 2>(), py::keep_alive<0, 3>(), py::keep_alive<0, 4>())
        .def("create_realspace_solver", [](Factory &f, ComputationBox *cb, Molecules *mol, PropagatorAnalyzer *pa) {
            if (pa->get_model_name() != mol->get_model_name())
                throw std::runtime_error("molecules and propagator analyzer use different chain models");
            return new GpuComputation(cb, mol, pa, f.precision, f.device, 1, "realspace", f.reduce_memory);
        }, py::keep_alive<0, 2>(), py::keep_alive<0, 3>(), py::keep_alive<0, 4>())
        .def("create_anderson_mixing", [](Factory &f, int n_var, int max_hist, double start_error, double mix_min, double mix_init) {
            return new GpuAndersonMixing(n_var, max_hist, start_error, mix_min, mix_init, f.device);
        })
        .def("display_info", [](Factory &f) {
            std::cout << "==================== B200 engine ====================" << std::endl;
            std::cout << "Platform: " << f.name << " (" << (f.precision == 8 ? "FP64" : "FP32 propagators, FP64 reductions")
                      << "), device " << f.device << std::endl;
        })
        .def("get_model_name", [](Factory &) { return std::string(""); });

    // Device-resident SCFT iteration (fields, residuals and optimizer in HBM).
    py::class_<DeviceScft>(m, "DeviceScft")
        .def(py::init([](Factory &f, ComputationBox *cb, Molecules *mol, PropagatorAnalyzer *pa, py::dict c) {
            ScftConfig cfg;
            cfg.monomer_types = c["monomer_types"].cast<std::vector<std::string>>();
            cfg.chi = c["matrix_chi"].cast<std::vector<double>>();
            cfg.P = c["matrix_p"].cast<std::vector<double>>();
            cfg.A_inv = c["matrix_a_inv"].cast<std::vector<double>>();
            cfg.box_altering = c["box_is_altering"].cast<bool>();
            cfg.scale_stress = c["scale_stress"].cast<double>();
            cfg.optimizer = c["optimizer"].cast<std::string>();
            if (c.contains("am_max_hist")) cfg.am_max_hist = c["am_max_hist"].cast<int>();
            if (c.contains("am_start_error")) cfg.am_start_error = c["am_start_error"].cast<double>();
            if (c.contains("am_mix_min")) cfg.am_mix_min = c["am_mix_min"].cast<double>();
            if (c.contains("am_mix_init")) cfg.am_mix_init = c["am_mix_init"].cast<double>();
            if (c.contains("adam_lr")) cfg.adam_lr = c["adam_lr"].cast<double>();
            if (c.contains("adam_gamma")) cfg.adam_gamma = c["adam_gamma"].cast<double>();
            return new DeviceScft(cb, mol, pa, f.precision, f.device, cfg);
        }), py::keep_alive<1, 3>(), py::keep_alive<1, 4>(), py::keep_alive<1, 5>())
        .def("set_fields", [](DeviceScft &d, Arr w) {
            py::buffer_info bi = w.request();
            size_check(bi, (long long)d.n_types() * d.n_grid(), "w ", "S*n_grid");
            d.set_fields((const double *)bi.ptr);
        })
        .def("get_fields", [](DeviceScft &d) {
            py::array_t<double> w({(py::ssize_t)d.n_types(), (py::ssize_t)d.n_grid()});
            d.get_fields((double *)w.request().ptr);
            return w;
        })
        .def("get_concentrations", [](DeviceScft &d) {
            py::array_t<double> phi({(py::ssize_t)d.n_types(), (py::ssize_t)d.n_grid()});
            d.get_concentrations((double *)phi.request().ptr);
            return phi;
        })
        .def("evaluate", [](DeviceScft &d) {
            ScftStats s;
            {
                py::gil_scoped_release nogil;
                s = d.evaluate();
            }
            py::dict r;
            r["error_level"] = s.error_level; r["mass_error"] = s.mass_error; r["partitions"] = s.partitions;
            r["stress"] = s.stress; r["lx"] = s.lx; r["aux_mean"] = s.aux_mean; r["aux_msq"] = s.aux_msq;
            return r;
        })
        .def("update", [](DeviceScft &d) {
            py::gil_scoped_release nogil;
            d.update();
        })
        .def("reset", &DeviceScft::reset);

    // Batched L-FTS engine: n_replicas independent systems on the device.

    py::class_<BatchedLangevin>(m, "BatchedLangevin")
        .def(py::init([](Factory &f, ComputationBox *cb, Molecules *mol, PropagatorAnalyzer *pa, int n_replicas, py::dict c) {
            LangevinConfig cfg;
            cfg.monomer_types = c["monomer_types"].cast<std::vector<std::string>>();
            cfg.A = c["matrix_a"].cast<std::vector<double>>();
            cfg.h_coef_mu1 = c["h_coef_mu1"].cast<std::vector<double>>();
            cfg.h_coef_mu2 = c["h_coef_mu2"].cast<std::vector<double>>();
            cfg.h_const = c["h_const"].cast<double>();
            cfg.real_idx = c["real_idx"].cast<std::vector<int>>();
            cfg.imag_idx = c["imag_idx"].cast<std::vector<int>>();
            cfg.dt_scaling = c["dt_scaling"].cast<std::vector<double>>();
            cfg.dt = c["dt"].cast<double>();
            cfg.tolerance = c["tolerance"].cast<double>();
            cfg.max_iter = c["max_iter"].cast<int>();
            cfg.am_max_hist = c["am_max_hist"].cast<int>();
            cfg.am_start_error = c["am_start_error"].cast<double>();
            cfg.am_mix_min = c["am_mix_min"].cast<double>();
            cfg.am_mix_init = c["am_mix_init"].cast<double>();
            return new BatchedLangevin(cb, mol, pa, f.precision, f.device, n_replicas, cfg);
        }), py::keep_alive<1, 3>(), py::keep_alive<1, 4>(), py::keep_alive<1, 5>())
        .def("n_replicas", &BatchedLangevin::n_replicas)
        .def("set_host_control", &BatchedLangevin::set_host_control)
        .def("set_step_graph", &BatchedLangevin::set_step_graph)
        .def("step_graph", &BatchedLangevin::step_graph)
        .def("set_noise_streams", [](BatchedLangevin &b, py::array_t<unsigned long long, py::array::c_style | py::array::forcecast> st) {
            py::buffer_info bi = st.request();
            if (bi.size != 4LL * b.n_replicas()) throw std::runtime_error("noise streams must be an n_replicas x 4 uint64 array");
            b.set_noise_streams((const unsigned long long *)bi.ptr);
        })
        .def("get_noise_streams", [](BatchedLangevin &b) {
            py::array_t<unsigned long long> st({(py::ssize_t)b.n_replicas(), (py::ssize_t)4});
            b.get_noise_streams((unsigned long long *)st.request().ptr);
            return st;
        })
        .def("has_noise_streams", &BatchedLangevin::has_noise_streams)
        .def("w_aux_ptr", [](BatchedLangevin &b) { return (std::uintptr_t)b.w_aux_device(); })
        .def("langevin_update_device", [](BatchedLangevin &b, std::uintptr_t noise_dev) {
            py::gil_scoped_release nogil;
            b.langevin_update_device((const double *)noise_dev);
        })
        .def("langevin_update_rng", [](BatchedLangevin &b, double sigma) {
            py::gil_scoped_release nogil;
            b.langevin_update_rng(sigma);
        }, py::arg("sigma"))
        .def("finish_step", [](BatchedLangevin &b) {
            SaddleStats s;
            {
                py::gil_scoped_release nogil;
                s = b.find_saddle_point(true);
            }
            return stats_dict(s);
        })
        .def("step_rng", [](BatchedLangevin &b, double sigma) {
            SaddleStats s;
            {
                py::gil_scoped_release nogil;
                s = b.step_device_rng(sigma);
            }
            return stats_dict(s);
        }, py::arg("sigma"))
        .def("autotune", [](BatchedLangevin &b, int reps) {
            py::gil_scoped_release nogil;
            return b.computation().autotune(reps);
        }, py::arg("reps") = 5)
        .def("step_implementation", [](BatchedLangevin &b) {
            char buf[64];
            check_rc(lfts_step_impl(b.computation().context(), buf, sizeof buf));
            return std::string(buf);
        })
        .def("host_control", &BatchedLangevin::host_control)
        .def("stream_ptr", [](BatchedLangevin &b) { return (std::uintptr_t)b.stream(); })
        .def("kernel_launches", [](BatchedLangevin &b) { return b.computation().kernel_launches(); })
        .def("context_ptr", [](BatchedLangevin &b) { return (std::uintptr_t)b.computation().context(); })
        .def("step_device", [](BatchedLangevin &b, std::uintptr_t noise_dev) {
            SaddleStats s;
            {
                py::gil_scoped_release nogil;
                s = b.step_device((const double *)noise_dev);
            }
            return stats_dict(s);
        })
        .def("set_fields", [](BatchedLangevin &b, Arr w) {
            py::buffer_info bi = w.request();
            size_check(bi, (long long)b.n_replicas() * b.n_grid() * (long long)(bi.size / ((long long)b.n_replicas() * b.n_grid())),
                       "w_aux ", "n_replicas*S*n_grid");
            b.set_fields((const double *)bi.ptr);
        })
        .def("get_fields", [](BatchedLangevin &b, int S) {
            py::array_t<double> w({(py::ssize_t)b.n_replicas(), (py::ssize_t)S, (py::ssize_t)b.n_grid()});
            b.get_fields((double *)w.request().ptr);
            return w;
        })
        .def("get_concentrations", [](BatchedLangevin &b, int S) {
            py::array_t<double> phi({(py::ssize_t)b.n_replicas(), (py::ssize_t)S, (py::ssize_t)b.n_grid()});
            b.get_concentrations((double *)phi.request().ptr);
            return phi;
        })
        .def("find_saddle_point", [](BatchedLangevin &b) {
            SaddleStats s;
            {
                py::gil_scoped_release nogil;
                s = b.find_saddle_point(false);
            }
            return stats_dict(s);
        })
        .def("get_noise_prev", [](BatchedLangevin &b) {
            py::array_t<double> xi({(py::ssize_t)b.n_replicas(), (py::ssize_t)b.n_real(), (py::ssize_t)b.n_grid()});
            b.get_noise_prev((double *)xi.request().ptr);
            return xi;
        })
        .def("set_noise_prev", [](BatchedLangevin &b, Arr xi) {
            py::buffer_info bi = xi.request();
            size_check(bi, (long long)b.n_replicas() * b.n_real() * b.n_grid(), "normal_noise_prev ", "n_replicas*n_real*n_grid");
            b.set_noise_prev((const double *)bi.ptr);
        })
        .def("sf_accumulate", [](BatchedLangevin &b, Arr coef, std::vector<int> pairs) {
            py::buffer_info bi = coef.request();
            if (bi.ndim != 2) throw std::runtime_error("coef must be a (S-1) x S array");
            py::gil_scoped_release nogil;
            b.sf_accumulate((const double *)bi.ptr, pairs);
        }, py::arg("coef"), py::arg("pairs"))
        .def("get_structure_function", [](BatchedLangevin &b, std::vector<py::ssize_t> shape_k, bool reset) {
            std::vector<py::ssize_t> shape = {(py::ssize_t)b.n_replicas(), (py::ssize_t)b.sf_npairs()};
            long long n = 1;
            for (auto e : shape_k) { shape.push_back(e); n *= e; }
            if (n != b.n_complex_grid()) throw std::runtime_error("shape_k must describe the half spectrum (nx, ny, nz/2+1)");
            py::array_t<std::complex<double>> out(shape);
            b.sf_get((double *)out.request().ptr, reset);
            return out;
        }, py::arg("shape_k"), py::arg("reset") = true)
        .def("step", [](BatchedLangevin &b, Arr noise) {
            py::buffer_info bi = noise.request();
            size_check(bi, (long long)b.n_replicas() * b.n_real() * b.n_grid(), "noise ", "n_replicas*n_real*n_grid");
            SaddleStats s;
            {
                py::gil_scoped_release nogil;
                s = b.step((const double *)bi.ptr);
            }
            return stats_dict(s);
        });

    py::class_<PlatformSelector>(m, "PlatformSelector")
        .def(py::init<>())
        .def_static("avail_platforms", &PlatformSelector::avail_platforms)
        .def_static("create_factory", [](const std::string &p) { return PlatformSelector::create_factory(p, false); })
        .def_static("create_factory", &PlatformSelector::create_factory);
}
