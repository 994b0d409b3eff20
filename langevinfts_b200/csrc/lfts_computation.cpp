// GPU propagator computation and Anderson mixing (host side).
// Reference behaviour followed (Langevin_FTS paths):
//   continuous  src/platforms/cpu/CpuComputationContinuous.cpp:9-816
//   discrete    src/platforms/cpu/CpuComputationDiscrete.cpp:8-1089
//   stress/Q    src/common/PropagatorComputation.cpp:35-70
//   AM          src/platforms/cpu/CpuAndersonMixing.cpp:76-161, src/common/AndersonMixing.cpp:19-47
#include "lfts_computation.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>

namespace lfts {

void check_rc(int rc) {
    if (rc != 0) throw std::runtime_error(std::string("liblfts_b200: ") + lfts_last_error());
}

void DevBuf::alloc(lfts_ctx c, size_t bytes) {
    release();
    ctx_ = c;
    n_ = bytes;
    check_rc(lfts_malloc(c, &p_, bytes));
}
void DevBuf::alloc_host(lfts_ctx c, size_t bytes) {
    release();
    ctx_ = c;
    n_ = bytes;
    check_rc(lfts_malloc_host(c, &p_, bytes));
    host_ = true;
}
void DevBuf::release() {
    if (p_ && ctx_) {
        if (host_) lfts_free_host(ctx_, p_);
        else lfts_free(ctx_, p_);
    }
    p_ = nullptr;
    n_ = 0;
    host_ = false;
}

static std::vector<double> simpson(int N) {
    // Simpson 1/3 rule with a 3/8 tail for odd N, trapezoid for N = 1 (SimpsonRule.h:10-59)
    std::vector<double> c;
    if (N == 0) return {1.0};
    if (N == 1) return {0.5, 0.5};
    if (N == 3) return {3.0 / 8.0, 9.0 / 8.0, 9.0 / 8.0, 3.0 / 8.0};
    c.push_back(1.0 / 3.0);
    const int inner_end = (N % 2 == 0) ? N - 1 : N - 4;
    for (int n = 1; n <= inner_end; n++) c.push_back(n % 2 == 1 ? 4.0 / 3.0 : 2.0 / 3.0);
    if (N % 2 == 0) {
        c.push_back(1.0 / 3.0);
    } else {
        c.push_back(3.0 / 8.0 + 1.0 / 3.0);
        c.push_back(9.0 / 8.0);
        c.push_back(9.0 / 8.0);
        c.push_back(3.0 / 8.0);
    }
    return c;
}

// arena of host-built job arrays, uploaded once; offsets are 64-byte aligned
template <typename T>
static size_t arena_push(std::vector<unsigned char> &a, const std::vector<T> &v) {
    size_t off = (a.size() + 63) / 64 * 64;
    a.resize(off + sizeof(T) * std::max<size_t>(v.size(), 1));
    if (!v.empty()) std::memcpy(a.data() + off, v.data(), sizeof(T) * v.size());
    return off;
}

GpuComputation::GpuComputation(ComputationBox *cb, Molecules *mol, PropagatorAnalyzer *pa, int precision, int device,
                               int n_replicas, const std::string &method, bool reduce_memory)
    : cb_(cb), mol_(mol), pa_(pa), prec_(precision), R_(n_replicas), esz_(precision) {
    if (!cb || !mol || !pa) LFTS_THROW("null ComputationBox, Molecules or PropagatorAnalyzer");
    if (n_replicas < 1) LFTS_THROW("n_replicas must be positive");
    if (pa->get_computation_propagators().empty()) LFTS_THROW("There is no propagator code. Add polymers first.");
    if (pa->get_computation_blocks().empty()) LFTS_THROW("There is no block. Add polymers first.");
    continuous_ = mol->get_model_name() == "continuous";
    if (method == "realspace") {
        // src/platforms/cpu/MklFactory.cpp:62-80, CpuSolverReal.cpp:15-16
        if (!continuous_) LFTS_THROW("The real-space solver does not support discrete chain model.");
        if (precision != 8) LFTS_THROW("The real-space solver runs in FP64 (platform \"cuda\") only.");
        realspace_ = true;
    } else if (method != "pseudospectral") {
        LFTS_THROW("unknown propagator method " + method);
    } else if (!cb->is_periodic()) {
        LFTS_THROW("Currently, pseudo-spectral method only supports periodic boundary conditions");  // Pseudo.cpp:49-50
    }
    const std::vector<int> nx = cb->get_nx();
    check_rc(lfts_ctx_create(&ctx_, device, (int)nx.size(), nx.data(), precision));
    check_rc(lfts_ctx_info(ctx_, &M_, &Mc_, nullptr));
    if (const char *e = std::getenv("LFTS_NO_GRAPH")) use_graph_ = std::string(e) != "1";
    const size_t RM = (size_t)R_ * M_;

    for (const auto &kv : mol->get_bond_lengths()) {
        TypeStore &t = types_[kv.first];
        t.w.alloc(ctx_, sizeof(double) * RM);
        t.fac.alloc(ctx_, esz_ * RM);
        t.bond.alloc(ctx_, std::max<size_t>(esz_ * Mc_, sizeof(double) * (size_t)lfts_realspace_table_size(ctx_)));
        t.bond_half.alloc(ctx_, esz_ * Mc_);
        phi_type_[kv.first].alloc(ctx_, sizeof(double) * RM);
    }
    for (const auto &it : pa->get_computation_propagators()) {
        KeyStore &ks = keys_[it.first];
        auto slices = [&](DevBuf &b, size_t bytes) {
            if (reduce_memory) b.alloc_host(ctx_, bytes);
            else b.alloc(ctx_, bytes);
        };
        slices(ks.q, esz_ * RM * (it.second.max_n_segment + 1));
        if (!continuous_) {
            if (!it.second.deps.empty()) slices(ks.half[0], esz_ * RM);
            for (int n : it.second.junction_ends)
                if (n >= 1 && n <= it.second.max_n_segment && !ks.half.count(n)) slices(ks.half[n], esz_ * RM);
        }
        if (it.first[0] == '{') {
            const std::string name = code::q_input_from_key(it.first);
            if (!q_init_.count(name)) q_init_[name].alloc(ctx_, esz_ * RM);
        }
    }
    for (const auto &it : pa->get_computation_blocks()) {
        phi_block_[it.first].alloc(ctx_, sizeof(double) * RM);
        block_order_.push_back(it.first);
    }
    for (int s = 0; s < mol->get_n_solvent_types(); s++) phi_solvent_.emplace_back(ctx_, sizeof(double) * RM);
    phi_tmp_.alloc(ctx_, sizeof(double) * M_);
    const int P = mol->get_n_polymer_types();
    q_poly_.assign((size_t)R_ * P, 0.0);
    q_solvent_.assign(mol->get_n_solvent_types(), 0.0);
    dq_dl_.assign(P, {0.0, 0.0, 0.0});
    dev_scalars_.alloc(ctx_, sizeof(double) * ((size_t)R_ * P + 64 + mol->get_n_solvent_types()));
    basis_.alloc(ctx_, sizeof(double) * 3 * Mc_);
    active_.alloc(ctx_, sizeof(int) * R_);
    {
        std::vector<int> ones(R_, 1);
        check_rc(lfts_memcpy_h2d(ctx_, active_.get(), ones.data(), sizeof(int) * R_));
    }

    // the reference's lane count: OMP_NUM_THREADS, default 4
    int n_streams = 4;
    if (const char *e = std::getenv("OMP_NUM_THREADS")) {
        try { n_streams = std::max(1, std::stoi(e)); } catch (...) { n_streams = 4; }
    }
    sched_ = new Scheduler(pa->get_computation_propagators(), n_streams);
    build_plan();
    build_dot_jobs();
    build_phi_jobs();
    build_stress_jobs();
    arena_.alloc(ctx_, std::max<size_t>(arena_host_.size(), 64));
    check_rc(lfts_memcpy_h2d(ctx_, arena_.get(), arena_host_.data(), arena_host_.size()));
    update_laplacian_operator();
}

GpuComputation::~GpuComputation() {
    if (graph_) lfts_graph_destroy(graph_);
    if (stats_graph_) lfts_graph_destroy(stats_graph_);
    delete sched_;
    keys_.clear();
    types_.clear();
    q_init_.clear();
    phi_block_.clear();
    phi_type_.clear();
    phi_solvent_.clear();
    active_.release(); phi_tmp_.release(); spec_.release(); arena_.release(); dev_scalars_.release(); basis_.release();
    phi_jobs_.release(); coefs_.release(); stress_jobs_.release(); stress_out_.release(); stress_spec_.release();
    if (ctx_) lfts_ctx_destroy(ctx_);
}

void *GpuComputation::slice(const std::string &key, int n, int r) const {
    const KeyStore &ks = keys_.at(key);
    const size_t nslices = ks.q.size() / (esz_ * M_ * R_);
    return (char *)ks.q.get() + esz_ * M_ * ((size_t)r * nslices + (size_t)n);
}
void *GpuComputation::half_slice(const std::string &key, int n, int r) const {
    const KeyStore &ks = keys_.at(key);
    auto it = ks.half.find(n);
    if (it == ks.half.end()) LFTS_THROW("missing half-bond slice " + std::to_string(n) + " of " + key);
    return (char *)it->second.get() + esz_ * M_ * (size_t)r;
}

double *GpuComputation::w_device(const std::string &type) { return types_.at(type).w.as<double>(); }
double *GpuComputation::phi_type_device(const std::string &type) { return phi_type_.at(type).as<double>(); }
double *GpuComputation::partition_device() { return dev_scalars_.as<double>(); }

// Translate the schedule into batched launches: every slot's junction starts,
// then its steps in lock-step (one launch per step index for all jobs of all
// replicas).
void GpuComputation::build_plan() {
    auto &props = pa_->get_computation_propagators();
    int max_jobs = 1;
    const long long Ml = M_;
    auto step_job = [&](const void *in, long long is, void *out, long long os, const std::string &type, int r) {
        const TypeStore &t = types_.at(type);
        lfts_step_job j;
        j.in = in;
        j.in_stride = is;
        j.out = out;
        j.out_stride = os;
        j.fac = (const char *)t.fac.get() + esz_ * Ml * r;
        j.bond = t.bond.get();
        j.bond_half = t.bond_half.get();
        j.spec = nullptr;  // patched to a device address once spec_ exists
        j.active = R_ > 1 ? active_.as<int>() : nullptr;
        j.replica = r;
        j.pad = 0;
        return j;
    };
    struct PendingSteps {
        int kind, nsteps, half, with_fac;
        std::vector<lfts_step_job> jobs;
    };
    for (const auto &slot : sched_->get_schedule()) {
        std::vector<lfts_junction_job> jj;
        std::vector<const void *> deps;
        std::vector<double> wts;
        std::vector<Launch> copies;
        std::vector<PendingSteps> steps;
        std::map<std::tuple<int, int, int, int>, size_t> groups;  // (kind, nsteps, half, fac) -> index
        auto add_step = [&](int kind, int nsteps, int half, int wf, const lfts_step_job &j) {
            auto key = std::make_tuple(kind, nsteps, half, wf);
            auto g = groups.find(key);
            if (g == groups.end()) {
                groups[key] = steps.size();
                steps.push_back({kind, nsteps, half, wf, {}});
                g = groups.find(key);
            }
            steps[g->second].jobs.push_back(j);
        };
        std::vector<std::pair<lfts_step_job, std::pair<int, int>>> first_steps;
        std::vector<lfts_step_job> half_jobs;
        for (const auto &job : slot) {
            const std::string &key = std::get<0>(job);
            const int n_from0 = std::get<1>(job);
            const int n_to = std::get<2>(job);
            const ComputationEdge &e = props.at(key);
            const std::string &type = e.monomer_type;
            for (int r = 0; r < R_; r++) {
                int n_from = n_from0;
                void *fac = (char *)types_.at(type).fac.get() + esz_ * Ml * r;
                if (continuous_) {
                    if (n_from == 0) {
                        lfts_junction_job j{slice(key, 0, r), nullptr, 0, 0, (int)deps.size(), 0};
                        if (e.deps.empty()) {
                            if (key[0] == '{') {
                                j.ndeps = 1;
                                deps.push_back((char *)q_init_.at(code::q_input_from_key(key)).get() + esz_ * Ml * r);
                                wts.push_back(1.0);
                            }
                        } else {
                            j.mode = key[0] == '[' ? 1 : 0;
                            j.ndeps = (int)e.deps.size();
                            for (const auto &d : e.deps) {
                                deps.push_back(slice(std::get<0>(d), std::get<1>(d), r));
                                wts.push_back((double)std::get<2>(d));
                            }
                        }
                        jj.push_back(j);
                    }
                    if (n_to > n_from)
                        add_step(1, n_to - n_from, 0, 1, step_job(slice(key, n_from, r), Ml, slice(key, n_from + 1, r), Ml, type, r));
                } else {
                    if (n_from == 0) {
                        if (e.deps.empty()) {
                            // leaf: q(1) = exp(-w ds) [* q_init]
                            lfts_junction_job j{slice(key, 1, r), fac, 0, 0, (int)deps.size(), 0};
                            if (key[0] == '{') {
                                j.ndeps = 1;
                                deps.push_back((char *)q_init_.at(code::q_input_from_key(key)).get() + esz_ * Ml * r);
                                wts.push_back(1.0);
                            }
                            jj.push_back(j);
                        } else if (key[0] == '[') {
                            lfts_junction_job j{slice(key, 1, r), nullptr, (int)e.deps.size(), 1, (int)deps.size(), 0};
                            for (const auto &d : e.deps) {
                                const int n = std::get<1>(d);
                                deps.push_back(n == 0 ? half_slice(std::get<0>(d), 0, r) : slice(std::get<0>(d), n, r));
                                wts.push_back((double)std::get<2>(d));
                            }
                            jj.push_back(j);
                            if (std::get<1>(e.deps[0]) == 0) {
                                Launch cp{};
                                cp.kind = 3;
                                cp.dst = half_slice(key, 0, r);
                                cp.src = slice(key, 1, r);
                                cp.bytes = esz_ * Ml;
                                copies.push_back(cp);
                                first_steps.push_back({step_job(slice(key, 1, r), 0, slice(key, 1, r), 0, type, r), {1, 1}});
                            } else {
                                first_steps.push_back({step_job(slice(key, 1, r), 0, slice(key, 1, r), 0, type, r), {0, 1}});
                            }
                        } else {
                            lfts_junction_job j{half_slice(key, 0, r), nullptr, (int)e.deps.size(), 0, (int)deps.size(), 0};
                            for (const auto &d : e.deps) {
                                deps.push_back(half_slice(std::get<0>(d), std::get<1>(d), r));
                                wts.push_back(1.0);
                            }
                            jj.push_back(j);
                            if (n_to > 0)
                                first_steps.push_back({step_job(half_slice(key, 0, r), 0, slice(key, 1, r), 0, type, r), {1, 1}});
                        }
                    }
                    if (n_to == 0) continue;
                    if (n_from == 0) {
                        if (keys_.at(key).half.count(1))
                            half_jobs.push_back(step_job(slice(key, 1, r), 0, half_slice(key, 1, r), 0, type, r));
                        n_from = 1;
                    }
                    if (n_to > n_from)
                        add_step(2, n_to - n_from, 0, 1, step_job(slice(key, n_from, r), Ml, slice(key, n_from + 1, r), Ml, type, r));
                    for (int n = n_from; n < n_to; n++)
                        if (e.junction_ends.count(n + 1) && n + 1 != 1)
                            half_jobs.push_back(step_job(slice(key, n + 1, r), 0, half_slice(key, n + 1, r), 0, type, r));
                }
            }
        }
        if (!jj.empty()) {
            Launch L{};
            L.kind = 0;
            L.jobs = arena_push(arena_host_, jj);
            L.njobs = (int)jj.size();
            L.deps = arena_push(arena_host_, deps);
            L.wts = arena_push(arena_host_, wts);
            plan_.push_back(L);
        }
        for (auto &cp : copies) plan_.push_back(cp);
        std::map<std::pair<int, int>, std::vector<lfts_step_job>> fs;
        for (auto &f : first_steps) fs[f.second].push_back(f.first);
        std::vector<PendingSteps> ordered;
        for (auto &g : fs) ordered.push_back({2, 1, g.first.first, g.first.second, g.second});
        for (auto &st : steps) ordered.push_back(st);
        if (!half_jobs.empty()) ordered.push_back({2, 1, 1, 0, half_jobs});
        for (auto &st : ordered) {
            for (size_t i = 0; i < st.jobs.size(); i++) st.jobs[i].spec = (void *)(intptr_t)i;
            max_jobs = std::max(max_jobs, (int)st.jobs.size());
            Launch L{};
            L.kind = st.kind;
            L.njobs = (int)st.jobs.size();
            L.nsteps = st.nsteps;
            L.half = st.half;
            L.with_fac = st.with_fac;
            L.jobs = arena_push(arena_host_, st.jobs);
            plan_.push_back(L);
        }
    }
    // per-job spectra scratch; patch spec indices into device addresses
    spec_.alloc(ctx_, (size_t)max_jobs * 2 * Mc_ * 2 * esz_);
    max_jobs_ = max_jobs;
    for (auto &L : plan_) {
        if (L.kind != 1 && L.kind != 2) continue;
        auto *jobs = (lfts_step_job *)(arena_host_.data() + L.jobs);
        for (int i = 0; i < L.njobs; i++)
            jobs[i].spec = (char *)spec_.get() + (size_t)(intptr_t)jobs[i].spec * 2 * Mc_ * 2 * esz_;
    }
}

// Single-chain partition functions: the first block of each polymer in block
// order (CpuComputationContinuous.cpp:62-91, CpuComputationDiscrete.cpp:92-122).
// Jobs are replica-major: Q of (replica r, polymer p) lands at r * P + p.
void GpuComputation::build_dot_jobs() {
    std::vector<lfts_dot_job> jobs;
    std::vector<std::pair<BlockKey, int>> chosen;
    int current_p = 0;
    for (const auto &bk : block_order_) {
        const int p = std::get<0>(bk);
        if (p != current_p) continue;
        const ComputationBlock &b = pa_->get_computation_block(bk);
        if (!continuous_ && b.n_segment_left == 0) continue;
        chosen.push_back({bk, p});
        current_p++;
    }
    const int P = mol_->get_n_polymer_types();
    if ((int)chosen.size() != P) LFTS_THROW("could not find a block for the partition function of every polymer");
    for (int r = 0; r < R_; r++) {
        for (const auto &c : chosen) {
            const BlockKey &bk = c.first;
            const ComputationBlock &b = pa_->get_computation_block(bk);
            const int NL = b.n_segment_left;
            if (continuous_)
                jobs.push_back({slice(std::get<1>(bk), NL, r), slice(std::get<2>(bk), 0, r), nullptr, 0.0});
            else
                jobs.push_back({slice(std::get<1>(bk), NL, r), slice(std::get<2>(bk), 1, r),
                                (const char *)types_.at(b.monomer_type).fac.get() + esz_ * M_ * r, 0.0});
        }
    }
    for (const auto &c : chosen) partition_polymer_.push_back(c.second);
    n_dot_jobs_ = (int)jobs.size();
    dot_jobs_ = arena_push(arena_host_, jobs);
}

// Concentration jobs with the normalisation ds phi_p / alpha_p * n_repeated
// divided on the device by Q_p of the same replica.
void GpuComputation::build_phi_jobs() {
    std::vector<lfts_phi_job> cont, disc;
    std::vector<double> coefs;
    const int P = mol_->get_n_polymer_types();
    for (int r = 0; r < R_; r++) {
        for (const auto &bk : block_order_) {
            const ComputationBlock &b = pa_->get_computation_block(bk);
            double *phi = phi_block_.at(bk).as<double>() + (size_t)r * M_;
            if (b.n_segment_right == 0) {
                if (r == 0) zero_blocks_.push_back({bk, 0});
                continue;
            }
            const int p = std::get<0>(bk);
            Polymer &pc = mol_->get_polymer(p);
            lfts_phi_job j;
            j.q_left = slice(std::get<1>(bk), 0, r);
            j.q_right = slice(std::get<2>(bk), 0, r);
            j.fac = (const char *)types_.at(b.monomer_type).fac.get() + esz_ * M_ * r;
            j.phi = phi;
            j.norm = mol_->get_ds() * pc.get_volume_fraction() / pc.get_alpha() * b.n_repeated;
            j.q_div = dev_scalars_.as<double>() + (size_t)r * P + p;
            j.n_left = b.n_segment_left;
            j.n_right = b.n_segment_right;
            j.coef_offset = 0;
            j.pad = 0;
            if (continuous_) {
                const auto c = simpson(b.n_segment_right);
                j.coef_offset = (int)coefs.size();
                coefs.insert(coefs.end(), c.begin(), c.end());
                cont.push_back(j);
            } else {
                disc.push_back(j);
            }
        }
    }
    n_phi_cont_ = (int)cont.size();
    n_phi_disc_ = (int)disc.size();
    phi_jobs_cont_ = arena_push(arena_host_, cont);
    phi_jobs_disc_ = arena_push(arena_host_, disc);
    coef_off_ = arena_push(arena_host_, coefs);
}

// (block, contour point) pairs of the stress sum with their weights, replica 0
// (CpuComputationContinuous.cpp:643-726, CpuComputationDiscrete.cpp:857-996).
void GpuComputation::build_stress_jobs() {
    std::vector<lfts_stress_job> jobs;
    auto &props = pa_->get_computation_propagators();
    for (size_t bi = 0; bi < block_order_.size(); bi++) {
        const BlockKey &bk = block_order_[bi];
        const ComputationBlock &b = pa_->get_computation_block(bk);
        const std::string &kl = std::get<1>(bk), &kr = std::get<2>(bk);
        const int NR = b.n_segment_right, NL = b.n_segment_left, rep = b.n_repeated;
        if (NR == 0) continue;
        const double bl = mol_->get_bond_lengths().at(b.monomer_type);
        const double b2 = bl * bl;
        const TypeStore &t = types_.at(b.monomer_type);
        if (continuous_) {
            const std::vector<double> c = simpson(NR);
            for (int n = 0; n <= NR; n++) {
                jobs.push_back({slice(kl, NL - n), slice(kr, n), nullptr, b2 * c[n] * rep});
                stress_block_.push_back((int)bi);
            }
        } else {
            for (int n = 0; n <= NR; n++) {
                if (n == NL) {
                    if (props.at(kl).deps.empty()) continue;
                    jobs.push_back({half_slice(kl, 0), slice(kr, NR), t.bond_half.get(), 0.5 * b2 * rep});
                } else if (n == 0 && NL == NR) {
                    if (props.at(kr).deps.empty()) continue;
                    jobs.push_back({slice(kl, NL), half_slice(kr, 0), t.bond_half.get(), 0.5 * b2 * rep});
                } else if (n == 0) {
                    continue;
                } else {
                    jobs.push_back({slice(kl, NL - n), slice(kr, n), t.bond.get(), b2 * rep});
                }
                stress_block_.push_back((int)bi);
            }
        }
    }
    n_stress_jobs_ = (int)jobs.size();
    if (n_stress_jobs_ == 0) return;
    stress_jobs_.alloc(ctx_, sizeof(lfts_stress_job) * jobs.size());
    check_rc(lfts_memcpy_h2d(ctx_, stress_jobs_.get(), jobs.data(), sizeof(lfts_stress_job) * jobs.size()));
    stress_out_.alloc(ctx_, sizeof(double) * 3 * jobs.size());
    const size_t per_job = 2 * (size_t)Mc_ * 2 * esz_;
    stress_chunk_ = (int)std::max<size_t>(1, std::min<size_t>(256, ((size_t)512 << 20) / per_job));
    stress_chunk_ = std::min(stress_chunk_, n_stress_jobs_);
}

void GpuComputation::update_laplacian_operator() {
    const std::vector<double> lx = cb_->get_lx();
    if (realspace_) {
        // Crank-Nicolson tables of every monomer type (CpuSolverReal.cpp:86-106)
        const std::vector<double> dx = cb_->get_dx();
        std::vector<double> tab((size_t)lfts_realspace_table_size(ctx_));
        for (const auto &kv : mol_->get_bond_lengths()) {
            check_rc(lfts_realspace_tables(ctx_, kv.second * kv.second, mol_->get_ds(), cb_->get_dim(), dx.data(),
                                           cb_->get_boundary_conditions().data(), tab.data()));
            check_rc(lfts_memcpy_h2d(ctx_, types_.at(kv.first).bond.get(), tab.data(), sizeof(double) * tab.size()));
        }
    } else {
        for (const auto &kv : mol_->get_bond_lengths()) {
            TypeStore &t = types_.at(kv.first);
            check_rc(lfts_bond_tables(ctx_, kv.second * kv.second, mol_->get_ds(), lx.data(), t.bond.get(), t.bond_half.get()));
        }
        check_rc(lfts_fourier_basis(ctx_, lx.data(), basis_.as<double>()));
    }
    // partition scale dv / (n_aggregated V): n_aggregated is structural, dv and V follow the box
    const auto *jobs = (const lfts_dot_job *)(arena_host_.data() + dot_jobs_);
    std::vector<lfts_dot_job> dj(jobs, jobs + n_dot_jobs_);
    const double dv = cb_->get_dv(0), V = cb_->get_volume();
    std::vector<double> scale;
    int current_p = 0;
    for (const auto &b : block_order_) {
        const int p = std::get<0>(b);
        if (p != current_p) continue;
        const ComputationBlock &cbk = pa_->get_computation_block(b);
        if (!continuous_ && cbk.n_segment_left == 0) continue;
        const int n_agg = (int)cbk.v_u.size() / cbk.n_repeated;
        scale.push_back(dv / n_agg / V);
        current_p++;
    }
    for (int j = 0; j < n_dot_jobs_; j++) dj[j].scale = scale[j % scale.size()];
    if (n_dot_jobs_ > 0)
        check_rc(lfts_memcpy_h2d(ctx_, (char *)arena_.get() + dot_jobs_, dj.data(), sizeof(lfts_dot_job) * n_dot_jobs_));
}

void GpuComputation::enqueue_propagation() {
    char *base = (char *)arena_.get();
    const double ds = mol_->get_ds();
    const size_t RM = (size_t)R_ * M_;
    (void)RM;
    for (auto &kv : types_)  // factor tables of all replicas in one pass over R*M points
        check_rc(lfts_field_factors_batch(ctx_, kv.second.w.as<double>(), continuous_ ? -ds / 4.0 : -ds, kv.second.fac.get(), R_));
    for (const auto &L : plan_) {
        switch (L.kind) {
            case 0:
                check_rc(lfts_junctions(ctx_, (const lfts_junction_job *)(base + L.jobs), L.njobs,
                                        (const void *const *)(base + L.deps), (const double *)(base + L.wts)));
                break;
            case 1:
                for (int s = 0; s < L.nsteps; s++) {
                    if (realspace_)
                        check_rc(lfts_step_realspace(ctx_, (const lfts_step_job *)(base + L.jobs), L.njobs, s, cb_->get_dim()));
                    else
                        check_rc(lfts_step_continuous(ctx_, (const lfts_step_job *)(base + L.jobs), L.njobs, s));
                }
                break;
            case 2:
                for (int s = 0; s < L.nsteps; s++)
                    check_rc(lfts_step_discrete(ctx_, (const lfts_step_job *)(base + L.jobs), L.njobs, s, L.half, L.with_fac));
                break;
            case 3:
                check_rc(lfts_memcpy_d2d_async(ctx_, L.dst, L.src, L.bytes));
                break;
        }
    }
    if (n_dot_jobs_ > 0)
        check_rc(lfts_dots(ctx_, (const lfts_dot_job *)(base + dot_jobs_), n_dot_jobs_, dev_scalars_.as<double>()));
}

void GpuComputation::enqueue_concentrations() {
    char *base = (char *)arena_.get();
    for (const auto &z : zero_blocks_)
        check_rc(lfts_memset_async(ctx_, phi_block_.at(z.first).get(), 0, sizeof(double) * M_ * R_));
    if (n_phi_cont_ > 0)
        check_rc(lfts_phi_blocks(ctx_, 0, (const lfts_phi_job *)(base + phi_jobs_cont_), n_phi_cont_, (const double *)(base + coef_off_)));
    if (n_phi_disc_ > 0)
        check_rc(lfts_phi_blocks(ctx_, 1, (const lfts_phi_job *)(base + phi_jobs_disc_), n_phi_disc_, (const double *)(base + coef_off_)));
    // per-type totals over all replicas at once (blocks are [R][M])
    for (auto &kv : phi_type_) {
        std::vector<const double *> srcs;
        for (const auto &bk : block_order_) {
            const ComputationBlock &b = pa_->get_computation_block(bk);
            if (code::monomer_type_from_key(std::get<1>(bk)) == kv.first && b.n_segment_right != 0)
                srcs.push_back(phi_block_.at(bk).as<double>());
        }
        check_rc(lfts_lincomb(ctx_, kv.second.as<double>(), (int)srcs.size(), srcs.data(), nullptr, (long long)M_ * R_));
    }
}

std::string GpuComputation::autotune(int reps) {
    if (stats_graph_ || graph_) LFTS_THROW("autotune must run before the first propagator computation (captured graphs keep their kernels)");
    char buf[512];
    check_rc(lfts_autotune(ctx_, max_jobs_, reps, buf, sizeof buf));
    return std::string(buf);
}

void GpuComputation::enqueue_statistics(bool use_graph) {
    if (mol_->get_n_solvent_types() > 0) LFTS_THROW("batched statistics do not support solvents");
    if (use_graph_ && use_graph) {
        if (!stats_graph_) {
            const long long before = lfts_ctx_launches(ctx_);
            check_rc(lfts_graph_begin(ctx_));
            enqueue_propagation();
            enqueue_concentrations();
            check_rc(lfts_graph_end(ctx_, &stats_graph_));
            stats_graph_kernels_ = lfts_ctx_launches(ctx_) - before;
        }
        check_rc(lfts_graph_launch(ctx_, stats_graph_));
        graph_kernels_replayed_ += stats_graph_kernels_;
    } else {
        enqueue_propagation();
        enqueue_concentrations();
    }
    have_propagators_ = true;
}

std::vector<double> GpuComputation::partitions_host() {
    std::vector<double> q((size_t)R_ * mol_->get_n_polymer_types());
    check_rc(lfts_memcpy_d2h(ctx_, q.data(), dev_scalars_.get(), sizeof(double) * q.size()));
    // a single system keeps them for get_total_partition / get_stress, as compute_concentrations does
    if (R_ == 1) q_poly_.assign(q.begin(), q.end());
    return q;
}

void GpuComputation::compute_propagators(const std::map<std::string, const double *> &w,
                                         const std::map<std::string, const double *> &q_init) {
    if (R_ != 1) LFTS_THROW("compute_propagators works on single systems; use the batched interface");
    for (const auto &it : pa_->get_computation_propagators())
        if (!w.count(it.second.monomer_type))
            LFTS_THROW("monomer_type \"" + it.second.monomer_type + "\" is not in w_input.");
    for (const auto &kv : w) {
        auto t = types_.find(kv.first);
        if (t == types_.end()) LFTS_THROW("monomer_type \"" + kv.first + "\" is not in exp_dw.");
        check_rc(lfts_memcpy_h2d(ctx_, t->second.w.get(), kv.second, sizeof(double) * M_));
    }
    for (auto &kv : q_init_) {
        auto it = q_init.find(kv.first);
        if (it == q_init.end()) LFTS_THROW("Could not find q_init[\"" + kv.first + "\"].");
        if (prec_ == 8) {
            check_rc(lfts_memcpy_h2d(ctx_, kv.second.get(), it->second, sizeof(double) * M_));
        } else {
            std::vector<float> f(it->second, it->second + M_);
            check_rc(lfts_memcpy_h2d(ctx_, kv.second.get(), f.data(), sizeof(float) * M_));
        }
    }
    if (use_graph_) {
        if (!graph_) {
            check_rc(lfts_graph_begin(ctx_));
            enqueue_propagation();
            check_rc(lfts_graph_end(ctx_, &graph_));
        }
        check_rc(lfts_graph_launch(ctx_, graph_));
    } else {
        enqueue_propagation();
    }
    sync_partitions();
    have_propagators_ = true;
}

void GpuComputation::sync_partitions() {
    std::vector<double> q(std::max(n_dot_jobs_, 1));
    check_rc(lfts_memcpy_d2h(ctx_, q.data(), dev_scalars_.get(), sizeof(double) * n_dot_jobs_));
    for (int j = 0; j < n_dot_jobs_; j++) q_poly_[j] = q[j];
}

void GpuComputation::compute_concentrations() {
    if (!have_propagators_) LFTS_THROW("compute_propagators must be called before compute_concentrations");
    enqueue_concentrations();
    // solvents (CpuComputationContinuous.cpp:425-436, CpuComputationDiscrete.cpp:441-452)
    const double dv_over_V = cb_->get_dv(0) / cb_->get_volume();
    double *qs = dev_scalars_.as<double>() + (size_t)R_ * mol_->get_n_polymer_types();
    for (int s = 0; s < mol_->get_n_solvent_types(); s++) {
        const auto sol = mol_->get_solvent(s);
        const TypeStore &t = types_.at(std::get<1>(sol));
        check_rc(lfts_solvent(ctx_, t.fac.get(), continuous_ ? 4 : 1, std::get<0>(sol), dv_over_V,
                              phi_solvent_[s].as<double>(), qs + s));
    }
    if (mol_->get_n_solvent_types() > 0)
        check_rc(lfts_memcpy_d2h(ctx_, q_solvent_.data(), qs, sizeof(double) * mol_->get_n_solvent_types()));
    check_rc(lfts_synchronize(ctx_));
}

void GpuComputation::compute_statistics(const std::map<std::string, const double *> &w,
                                        const std::map<std::string, const double *> &q_init) {
    compute_propagators(w, q_init);
    compute_concentrations();
}

double GpuComputation::get_total_partition(int p) {
    if (p < 0 || p >= mol_->get_n_polymer_types()) LFTS_THROW("Index (" + std::to_string(p) + ") is out of range.");
    return q_poly_[p];
}

void GpuComputation::get_chain_propagator(double *out, int p, int v, int u, int n) {
    Polymer &pc = mol_->get_polymer(p);
    const std::string key = pc.get_propagator_key(v, u);
    auto &props = pa_->get_computation_propagators();
    if (!props.count(key))
        LFTS_THROW("Could not find the propagator code '" + key + "'. Disable 'aggregation' option to obtain propagator_analyzer.");
    const int N = props.at(key).max_n_segment;
    const int lo = continuous_ ? 0 : 1;
    if (n < lo || n > N)
        LFTS_THROW("n (" + std::to_string(n) + ") must be in range [" + std::to_string(lo) + ", " + std::to_string(N) + "]");
    if (prec_ == 8) {
        check_rc(lfts_memcpy_d2h(ctx_, out, slice(key, n), sizeof(double) * M_));
    } else {
        std::vector<float> f(M_);
        check_rc(lfts_memcpy_d2h(ctx_, f.data(), slice(key, n), sizeof(float) * M_));
        for (long long i = 0; i < M_; i++) out[i] = f[i];
    }
}

void GpuComputation::get_total_concentration(const std::string &type, double *phi) {
    std::vector<const double *> srcs;
    for (const auto &bk : block_order_) {
        const ComputationBlock &b = pa_->get_computation_block(bk);
        if (code::monomer_type_from_key(std::get<1>(bk)) == type && b.n_segment_right != 0)
            srcs.push_back(phi_block_.at(bk).as<double>());
    }
    for (int s = 0; s < mol_->get_n_solvent_types(); s++)
        if (std::get<1>(mol_->get_solvent(s)) == type) srcs.push_back(phi_solvent_[s].as<double>());
    double *out = phi_tmp_.as<double>();
    check_rc(lfts_lincomb(ctx_, out, (int)srcs.size(), srcs.data(), nullptr, M_));
    check_rc(lfts_memcpy_d2h(ctx_, phi, out, sizeof(double) * M_));
}

void GpuComputation::get_total_concentration(int p, const std::string &type, double *phi) {
    const int P = mol_->get_n_polymer_types();
    if (p < 0 || p > P - 1) LFTS_THROW("Index (" + std::to_string(p) + ") must be in range [0, " + std::to_string(P - 1) + "]");
    std::vector<const double *> srcs;
    for (const auto &bk : block_order_) {
        const ComputationBlock &b = pa_->get_computation_block(bk);
        if (std::get<0>(bk) == p && code::monomer_type_from_key(std::get<1>(bk)) == type && b.n_segment_right != 0)
            srcs.push_back(phi_block_.at(bk).as<double>());
    }
    double *out = phi_tmp_.as<double>();
    check_rc(lfts_lincomb(ctx_, out, (int)srcs.size(), srcs.data(), nullptr, M_));
    check_rc(lfts_memcpy_d2h(ctx_, phi, out, sizeof(double) * M_));
}

void GpuComputation::get_total_concentration_gce(double fugacity, int p, const std::string &type, double *phi) {
    const int P = mol_->get_n_polymer_types();
    if (p < 0 || p > P - 1) LFTS_THROW("Index (" + std::to_string(p) + ") must be in range [0, " + std::to_string(P - 1) + "]");
    Polymer &pc = mol_->get_polymer(p);
    const double norm = fugacity / pc.get_volume_fraction() * pc.get_alpha() * q_poly_[p];
    std::vector<const double *> srcs;
    std::vector<double> coefs;
    for (const auto &bk : block_order_) {
        const ComputationBlock &b = pa_->get_computation_block(bk);
        if (std::get<0>(bk) == p && code::monomer_type_from_key(std::get<1>(bk)) == type && b.n_segment_right != 0) {
            srcs.push_back(phi_block_.at(bk).as<double>());
            coefs.push_back(norm);
        }
    }
    double *out = phi_tmp_.as<double>();
    check_rc(lfts_lincomb(ctx_, out, (int)srcs.size(), srcs.data(), coefs.data(), M_));
    check_rc(lfts_memcpy_d2h(ctx_, phi, out, sizeof(double) * M_));
}

void GpuComputation::get_block_concentration(int p, double *phi) {
    const int P = mol_->get_n_polymer_types();
    if (p < 0 || p > P - 1) LFTS_THROW("Index (" + std::to_string(p) + ") must be in range [0, " + std::to_string(P - 1) + "]");
    if (pa_->is_aggregated()) LFTS_THROW("Disable 'aggregation' option to invoke 'get_block_concentration'.");
    Polymer &pc = mol_->get_polymer(p);
    const auto &blocks = pc.get_blocks();
    for (size_t b = 0; b < blocks.size(); b++) {
        std::string kl = pc.get_propagator_key(blocks[b].v, blocks[b].u);
        std::string kr = pc.get_propagator_key(blocks[b].u, blocks[b].v);
        if (kl < kr) kl.swap(kr);
        check_rc(lfts_memcpy_d2h(ctx_, phi + b * M_, phi_block_.at(std::make_tuple(p, kl, kr)).get(), sizeof(double) * M_));
    }
}

double GpuComputation::get_solvent_partition(int s) {
    if (s < 0 || s >= (int)q_solvent_.size()) LFTS_THROW("Index (" + std::to_string(s) + ") is out of range.");
    return q_solvent_[s];
}

void GpuComputation::get_solvent_concentration(int s, double *phi) {
    const int S = mol_->get_n_solvent_types();
    if (s < 0 || s > S - 1) LFTS_THROW("Index (" + std::to_string(s) + ") must be in range [0, " + std::to_string(S - 1) + "]");
    check_rc(lfts_memcpy_d2h(ctx_, phi, phi_solvent_[s].get(), sizeof(double) * M_));
}

void GpuComputation::compute_stress() {
    if (realspace_) LFTS_THROW("Currently, the real-space method does not support stress computation.");  // CpuSolverReal.cpp:460-476
    if (!have_propagators_) LFTS_THROW("compute_propagators must be called before compute_stress");
    const int DIM = cb_->get_dim();
    const int P = mol_->get_n_polymer_types();
    std::vector<std::array<double, 3>> block_dq(block_order_.size(), {0.0, 0.0, 0.0});
    if (n_stress_jobs_ > 0) {
        if (!stress_spec_.get()) stress_spec_.alloc(ctx_, (size_t)stress_chunk_ * 2 * Mc_ * 2 * esz_);
        check_rc(lfts_stress(ctx_, stress_jobs_.as<lfts_stress_job>(), n_stress_jobs_, basis_.as<double>(),
                             stress_spec_.get(), stress_chunk_, stress_out_.as<double>()));
        std::vector<double> out(3 * (size_t)n_stress_jobs_);
        check_rc(lfts_memcpy_d2h(ctx_, out.data(), stress_out_.get(), sizeof(double) * out.size()));
        for (int j = 0; j < n_stress_jobs_; j++)
            for (int d = 0; d < DIM; d++) block_dq[stress_block_[j]][d] += out[3 * j + (3 - DIM) + d];
    }
    for (int p = 0; p < P; p++) dq_dl_[p] = {0.0, 0.0, 0.0};
    for (size_t bi = 0; bi < block_order_.size(); bi++)
        for (int d = 0; d < DIM; d++) dq_dl_[std::get<0>(block_order_[bi])][d] += block_dq[bi][d];
    const double M = (double)M_;
    for (int p = 0; p < P; p++)
        for (int d = 0; d < DIM; d++) dq_dl_[p][d] /= -3.0 * cb_->get_lx(d) * M * M / mol_->get_ds();
}

std::vector<double> GpuComputation::get_stress() {
    const int DIM = cb_->get_dim();
    std::vector<double> stress(DIM, 0.0);
    for (int p = 0; p < mol_->get_n_polymer_types(); p++) {
        Polymer &pc = mol_->get_polymer(p);
        for (int d = 0; d < DIM; d++) stress[d] += dq_dl_[p][d] * pc.get_volume_fraction() / pc.get_alpha() / q_poly_[p];
    }
    return stress;
}

std::vector<double> GpuComputation::get_stress_gce(const std::vector<double> &fug) {
    const int DIM = cb_->get_dim();
    std::vector<double> stress(DIM, 0.0);
    for (int p = 0; p < mol_->get_n_polymer_types(); p++)
        for (int d = 0; d < DIM; d++) stress[d] += fug.at(p) * dq_dl_[p][d];
    return stress;
}

// Q computed from every contour point of every block must agree
// (CpuComputationContinuous.cpp:755-816, CpuComputationDiscrete.cpp:1036-1089).
bool GpuComputation::check_total_partition() {
    std::vector<lfts_dot_job> jobs;
    std::vector<int> owner;
    const double dv = cb_->get_dv(0), V = cb_->get_volume();
    for (const auto &bk : block_order_) {
        const ComputationBlock &b = pa_->get_computation_block(bk);
        const int p = std::get<0>(bk);
        const int NR = b.n_segment_right, NL = b.n_segment_left;
        const double sc = dv * b.n_repeated / V / (double)b.v_u.size();
        if (continuous_) {
            for (int n = 0; n <= NR; n++) jobs.push_back({slice(std::get<1>(bk), NL - n), slice(std::get<2>(bk), n), nullptr, sc});
        } else {
            for (int n = 1; n <= NR; n++)
                jobs.push_back({slice(std::get<1>(bk), NL - n + 1), slice(std::get<2>(bk), n),
                                types_.at(b.monomer_type).fac.get(), sc});
        }
        owner.resize(jobs.size(), p);
    }
    if (jobs.empty()) return true;
    DevBuf dj(ctx_, sizeof(lfts_dot_job) * jobs.size()), dout(ctx_, sizeof(double) * jobs.size());
    check_rc(lfts_memcpy_h2d(ctx_, dj.get(), jobs.data(), dj.size()));
    check_rc(lfts_dots(ctx_, dj.as<lfts_dot_job>(), (int)jobs.size(), dout.as<double>()));
    std::vector<double> q(jobs.size());
    check_rc(lfts_memcpy_d2h(ctx_, q.data(), dout.get(), dout.size()));
    const int P = mol_->get_n_polymer_types();
    std::vector<double> mx(P, -1e20), mn(P, 1e20);
    for (size_t j = 0; j < q.size(); j++) {
        mx[owner[j]] = std::max(mx[owner[j]], q[j]);
        mn[owner[j]] = std::min(mn[owner[j]], q[j]);
    }
    std::cout << "Polymer id: maximum,  minimum, and difference of total partitions" << std::endl;
    for (int p = 0; p < P; p++) {
        const double diff = std::abs(mx[p] - mn[p]);
        std::cout << "\t" << p << ": " << mx[p] << ", " << mn[p] << ", " << diff << std::endl;
        if (diff > 1e-7) return false;
    }
    return true;
}

// ================================================================ Anderson mixing
static void find_an(std::vector<std::vector<double>> &u, std::vector<double> &v, std::vector<double> &a, int n) {
    // Gaussian elimination without pivoting, same operation order as
    // AndersonMixing::find_an (src/common/AndersonMixing.cpp:19-47)
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            const double f = u[j][i] / u[i][i];
            v[j] = v[j] - v[i] * f;
            for (int k = i + 1; k < n; k++) u[j][k] = u[j][k] - u[i][k] * f;
        }
    a[n - 1] = v[n - 1] / u[n - 1][n - 1];
    for (int i = n - 2; i >= 0; i--) {
        double s = 0.0;
        for (int j = i + 1; j < n; j++) s = s + u[i][j] * a[j];
        a[i] = (v[i] - s) / u[i][i];
    }
}

GpuAndersonMixing::GpuAndersonMixing(int n_var, int max_hist, double start_error, double mix_min, double mix_init, int device)
    : n_var_(n_var), max_hist_(max_hist), start_error_(start_error), mix_min_(mix_min), mix_(mix_init), mix_init_(mix_init) {
    if (n_var <= 0) LFTS_THROW("n_var must be positive");
    if (max_hist < 0) LFTS_THROW("max_hist must be non-negative");
    const int one = 1;
    check_rc(lfts_ctx_create(&ctx_, device, 1, &one, 8));
    ring_len_ = max_hist + 1;
    w_hist_.alloc(ctx_, sizeof(double) * (size_t)n_var * ring_len_);
    d_hist_.alloc(ctx_, sizeof(double) * (size_t)n_var * ring_len_);
    w_new_.alloc(ctx_, sizeof(double) * n_var);
    stage_w_.alloc(ctx_, sizeof(double) * n_var);
    stage_d_.alloc(ctx_, sizeof(double) * n_var);
    dots_.alloc(ctx_, sizeof(double) * ring_len_);
    a_.alloc(ctx_, sizeof(double) * (ring_len_ + 1));
    reset_count();
}

GpuAndersonMixing::~GpuAndersonMixing() {
    w_hist_.release(); d_hist_.release(); w_new_.release(); stage_w_.release(); stage_d_.release(); dots_.release(); a_.release();
    if (ctx_) lfts_ctx_destroy(ctx_);
}

void GpuAndersonMixing::reset_count() {
    mix_ = mix_init_;
    n_anderson_ = -1;
    head_ = -1;
    n_items_ = 0;
    dot_rows_.clear();
}

void GpuAndersonMixing::calculate_new_fields(double *w_new, const double *w_cur, const double *w_deriv, double old_err,
                                             double err) {
    step(w_new, w_cur, w_deriv, old_err, err, false);
}
void GpuAndersonMixing::calculate_new_fields_device(double *w_new, const double *w_cur, const double *w_deriv, double old_err,
                                                    double err) {
    step(w_new, w_cur, w_deriv, old_err, err, true);
}

void GpuAndersonMixing::step(double *w_new, const double *w_cur, const double *w_deriv, double old_err, double err,
                             bool device) {
    // host inputs are copied in synchronously; device inputs by this context's stream
    auto put = [&](void *dst, const void *src, size_t bytes) {
        if (device) check_rc(lfts_memcpy_d2d_async(ctx_, dst, src, bytes));
        else check_rc(lfts_memcpy_h2d(ctx_, dst, src, bytes));
    };
    if (err < start_error_ || n_anderson_ >= 0) n_anderson_ = n_anderson_ + 1;
    const size_t bytes = sizeof(double) * n_var_;
    const double *dw = nullptr, *dd = nullptr;
    if (n_anderson_ >= 0) {
        n_anderson_ = std::min(max_hist_, n_anderson_);
        head_ = (head_ + 1) % ring_len_;
        n_items_ = std::min(n_items_ + 1, ring_len_);
        double *wslot = w_hist_.as<double>() + (size_t)head_ * n_var_;
        double *dslot = d_hist_.as<double>() + (size_t)head_ * n_var_;
        put(wslot, w_cur, bytes);
        put(dslot, w_deriv, bytes);
        dw = wslot;
        dd = dslot;
        // d . d_i for the n_anderson+1 newest histories
        check_rc(lfts_am_dots(ctx_, dslot, d_hist_.as<double>(), n_var_, n_anderson_ + 1, n_var_, dots_.as<double>(), head_,
                              ring_len_));
        std::vector<double> row(n_anderson_ + 1);
        check_rc(lfts_memcpy_d2h(ctx_, row.data(), dots_.get(), sizeof(double) * row.size()));
        dot_rows_.insert(dot_rows_.begin(), row);
        if ((int)dot_rows_.size() > ring_len_) dot_rows_.resize(ring_len_);
    }
    if (n_anderson_ <= 0) {
        if (old_err < err) mix_ = std::max(mix_ * 0.7, mix_min_);
        else mix_ = mix_ * 1.01;
        if (!dw) {
            put(stage_w_.get(), w_cur, bytes);
            put(stage_d_.get(), w_deriv, bytes);
            dw = stage_w_.as<double>();
            dd = stage_d_.as<double>();
        }
        check_rc(lfts_am_simple(ctx_, w_new_.as<double>(), dw, dd, mix_, n_var_));
    } else {
        const int n = n_anderson_;
        std::vector<std::vector<double>> u(n, std::vector<double>(n));
        std::vector<double> v(n), a(n);
        const auto &d = dot_rows_;
        for (int i = 0; i < n; i++) {
            v[i] = d[0][0] - d[0][i + 1];
            for (int j = 0; j < n; j++)
                u[i][j] = d[0][0] - d[0][i + 1] - d[0][j + 1] + d[std::min(i + 1, j + 1)][std::abs(i - j)];
        }
        find_an(u, v, a, n);
        check_rc(lfts_memcpy_h2d(ctx_, a_.get(), a.data(), sizeof(double) * n));
        check_rc(lfts_am_update(ctx_, w_new_.as<double>(), w_hist_.as<double>(), d_hist_.as<double>(), n_var_, n,
                                a_.as<double>(), n_var_, head_, ring_len_));
    }
    if (device) {
        check_rc(lfts_memcpy_d2d_async(ctx_, w_new, w_new_.get(), bytes));
        check_rc(lfts_synchronize(ctx_));
    } else {
        check_rc(lfts_memcpy_d2h(ctx_, w_new, w_new_.get(), bytes));
    }
}

}  // namespace lfts
