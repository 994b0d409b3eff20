// Batched Langevin FTS driver loop (host side of lfts_langevin.cu).
// Per replica it follows the reference driver examples/fts/lfts.py:
//   Leimkuhler-Matthews step of the real fields         :697-706
//   saddle point of the imaginary fields by AM          :807-868
//   error = max over imaginary fields of std(dH/dw)     :833-834
//   restore the fields when the tolerance is missed     :713-730
// and the Anderson mixing control of CpuAndersonMixing.cpp:76-161.
#include "lfts_langevin.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace lfts {

namespace {
// Gaussian elimination without pivoting (src/common/AndersonMixing.cpp:19-47)
void solve_no_pivot(std::vector<std::vector<double>> &u, std::vector<double> &v, std::vector<double> &a, int n) {
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
}  // namespace

BatchedLangevin::BatchedLangevin(ComputationBox *cb, Molecules *mol, PropagatorAnalyzer *pa, int precision, int device,
                                 int n_replicas, const LangevinConfig &cfg)
    : cfg_(cfg), R_(n_replicas), mol_(mol) {
    S_ = (int)cfg.monomer_types.size();
    I_ = (int)cfg.imag_idx.size();
    Rr_ = (int)cfg.real_idx.size();
    if (S_ < 1 || S_ > LFTS_MAX_MONOMERS) LFTS_THROW("number of monomer types must be 1.." + std::to_string(LFTS_MAX_MONOMERS));
    if ((int)cfg.A.size() != S_ * S_) LFTS_THROW("matrix A must be S x S");
    if (I_ < 1 || Rr_ + I_ != S_) LFTS_THROW("real and imaginary field indices must partition the S fields");
    for (int c = 0; c < I_; c++)
        if (cfg.imag_idx[c] != S_ - I_ + c) LFTS_THROW("the imaginary fields must be the trailing auxiliary fields");
    if ((int)cfg.dt_scaling.size() != S_) LFTS_THROW("dt_scaling must have S entries");
    for (const auto &t : cfg.monomer_types)
        if (!mol->get_bond_lengths().count(t)) LFTS_THROW("monomer type " + t + " is not in the molecules");
    if (mol->get_bond_lengths().size() != (size_t)S_) LFTS_THROW("every monomer type of the molecules needs a field");
    comp_.reset(new GpuComputation(cb, mol, pa, precision, device, n_replicas));
    ctx_ = comp_->context();
    M_ = comp_->n_grid();
    const size_t RSM = (size_t)R_ * S_ * M_;
    w_aux_.alloc(ctx_, sizeof(double) * RSM);
    w_save_.alloc(ctx_, sizeof(double) * RSM);
    phi_save_.alloc(ctx_, sizeof(double) * RSM);
    d_cur_.alloc(ctx_, sizeof(double) * (size_t)R_ * I_ * M_);
    for (auto &x : xi_) {
        x.alloc(ctx_, sizeof(double) * (size_t)R_ * std::max(Rr_, 1) * M_);
        check_rc(lfts_memset_async(ctx_, x.get(), 0, x.size()));
    }
    L_ = cfg.am_max_hist + 1;
    partials_.alloc(ctx_, sizeof(double) * std::max<size_t>((size_t)128 * R_ * S_, (size_t)64 * R_ * L_));
    stats_.alloc(ctx_, sizeof(double) * 4 * (size_t)R_ * S_);
    ctl_.alloc(ctx_, sizeof(int) * 5 * (size_t)R_);
    am_w_.alloc(ctx_, sizeof(double) * (size_t)R_ * L_ * I_ * M_);
    am_d_.alloc(ctx_, sizeof(double) * (size_t)R_ * L_ * I_ * M_);
    am_dots_.alloc(ctx_, sizeof(double) * (size_t)R_ * L_);
    am_a_.alloc(ctx_, sizeof(double) * (size_t)R_ * (L_ + 1));
    sint_.alloc(ctx_, sizeof(int) * ((size_t)3 * R_ + 2));
    sdbl_.alloc(ctx_, sizeof(double) * (size_t)2 * R_);
    dot_ring_.alloc(ctx_, sizeof(double) * (size_t)R_ * L_ * L_);
    for (const auto &t : cfg.monomer_types) {
        phi_ptrs_.push_back(comp_->phi_type_device(t));
        w_mono_ptrs_.push_back(comp_->w_device(t));
    }
    check_rc(lfts_memset_async(ctx_, w_aux_.get(), 0, w_aux_.size()));
    for (auto p : phi_ptrs_) check_rc(lfts_memset_async(ctx_, p, 0, sizeof(double) * (size_t)R_ * M_));
    const int P = mol->get_n_polymer_types();
    for (int p = 0; p < P; p++) {
        Polymer &pc = mol->get_polymer(p);
        poly_coef_.push_back(pc.get_volume_fraction() / pc.get_alpha());
    }
    fin_stats_.alloc(ctx_, sizeof(double) * ((size_t)4 * R_ + (size_t)R_ * P + (size_t)2 * R_ * S_));
    fin_scratch_.alloc(ctx_, sizeof(double) * (size_t)R_);
    if (const char *e = std::getenv("LFTS_NO_GRAPH")) step_graph_on_ = std::string(e) != "1";
    check_rc(lfts_synchronize(ctx_));
    am_reset();
}

BatchedLangevin::~BatchedLangevin() {
    for (int k = 0; k < 2; k++) {
        if (g_update_[k]) lfts_graph_destroy(g_update_[k]);
        if (g_step_[k]) lfts_graph_destroy(g_step_[k]);
    }
    if (g_search_) lfts_graph_destroy(g_search_);
    fin_stats_.release(); fin_scratch_.release();
    w_aux_.release(); w_save_.release(); phi_save_.release(); d_cur_.release(); xi_[0].release(); xi_[1].release();
    partials_.release(); stats_.release(); ctl_.release(); am_w_.release(); am_d_.release(); am_dots_.release(); am_a_.release();
    sint_.release(); sdbl_.release(); dot_ring_.release(); pcg_.release(); noise_buf_.release();
    comp_.reset();
}

void BatchedLangevin::set_fields(const double *w) {
    check_rc(lfts_memcpy_h2d(ctx_, w_aux_.get(), w, w_aux_.size()));
}
void BatchedLangevin::get_fields(double *w) const { check_rc(lfts_memcpy_d2h(ctx_, w, w_aux_.get(), w_aux_.size())); }
void BatchedLangevin::get_concentrations(double *phi) const {
    for (int r = 0; r < R_; r++)
        for (int s = 0; s < S_; s++)
            check_rc(lfts_memcpy_d2h(ctx_, phi + ((size_t)r * S_ + s) * M_, phi_ptrs_[s] + (size_t)r * M_, sizeof(double) * M_));
}

void BatchedLangevin::am_reset() {
    n_anderson_.assign(R_, -1);
    head_.assign(R_, -1);
    mix_.assign(R_, cfg_.am_mix_init);
    dot_rows_.assign(R_, {});
}

double BatchedLangevin::hamiltonian(int r, const std::vector<double> &mean, const std::vector<double> &msq,
                                    const std::vector<double> &Q) const {
    // lfts.py:219-235
    double h = -mean[(size_t)r * S_ + S_ - 1];
    for (int i = 0; i < S_ - 1; i++) {
        h += cfg_.h_coef_mu2[i] * msq[(size_t)r * S_ + i];
        h += cfg_.h_coef_mu1[i] * mean[(size_t)r * S_ + i];
    }
    const int P = mol_->get_n_polymer_types();
    double hp = 0.0;
    for (int p = 0; p < P; p++) {
        Polymer &pc = mol_->get_polymer(p);
        hp -= pc.get_volume_fraction() / pc.get_alpha() * std::log(Q[(size_t)r * P + p]);
    }
    return hp + h + cfg_.h_const;
}

SaddleStats BatchedLangevin::find_saddle_point(bool restore_on_failure) {
    if (restore_on_failure && graph_mode()) {  // the search half of a step (after langevin_update_*)
        if (!g_search_) {
            check_rc(lfts_graph_begin(ctx_));
            enqueue_search(true);
            check_rc(lfts_graph_end(ctx_, &g_search_));
        }
        check_rc(lfts_graph_launch(ctx_, g_search_));
        return read_stats();
    }
    SaddleStats st;
    st.iterations.assign(R_, 0);
    st.error.assign(R_, 1e20);
    st.failed.assign(R_, 0);
    if (host_control_ || cfg_.am_max_hist > LFTS_AM_SOLVE_MAX_HIST) saddle_loop_host(st);
    else saddle_loop_device(st);
    double *d_mean = stats_.as<double>(), *d_var = d_mean + (size_t)R_ * S_;
    // Hamiltonian at the final fields (before the pressure shift, as the reference prints it)
    check_rc(lfts_lfts_row_moments(ctx_, w_aux_.as<double>(), R_, S_, M_, M_, (long long)S_ * M_, nullptr, partials_.as<double>(),
                                   d_mean, d_var));
    std::vector<double> mean((size_t)R_ * S_), msq((size_t)R_ * S_);
    check_rc(lfts_memcpy_d2h(ctx_, mean.data(), d_mean, sizeof(double) * mean.size()));
    check_rc(lfts_memcpy_d2h(ctx_, msq.data(), d_var, sizeof(double) * msq.size()));
    st.partitions = comp_->partitions_host();
    st.aux_mean = mean;
    st.aux_msq = msq;
    st.hamiltonian.resize(R_);
    for (int r = 0; r < R_; r++) st.hamiltonian[r] = hamiltonian(r, mean, msq, st.partitions);
    // zero-mean pressure field of every replica (lfts.py:866)
    std::vector<double> pmean(R_);
    for (int r = 0; r < R_; r++) pmean[r] = mean[(size_t)r * S_ + S_ - 1];
    check_rc(lfts_memcpy_h2d(ctx_, d_mean, pmean.data(), sizeof(double) * R_));
    check_rc(lfts_lfts_subtract_mean(ctx_, w_aux_.as<double>(), R_, S_, S_ - 1, M_, d_mean, nullptr));
    for (int r = 0; r < R_; r++) st.failed[r] = (std::isnan(st.error[r]) || st.error[r] >= cfg_.tolerance) ? 1 : 0;
    if (restore_on_failure) {
        const size_t SM = (size_t)S_ * M_;
        for (int r = 0; r < R_; r++) {
            if (!st.failed[r]) continue;
            check_rc(lfts_memcpy_d2d_async(ctx_, w_aux_.as<double>() + r * SM, w_save_.as<double>() + r * SM, sizeof(double) * SM));
            for (int s = 0; s < S_; s++)
                check_rc(lfts_memcpy_d2d_async(ctx_, phi_ptrs_[s] + (size_t)r * M_, phi_save_.as<double>() + r * SM + (size_t)s * M_,
                                               sizeof(double) * M_));
        }
    }
    check_rc(lfts_synchronize(ctx_));
    return st;
}

// The saddle-point iterations with the per-replica control on the host: one
// round trip per iteration for the errors and one for the Anderson dots.
void BatchedLangevin::saddle_loop_host(SaddleStats &st) {
    am_reset();
    const long long nI = (long long)I_ * M_;
    std::vector<int> active(R_, 1), head_flag(R_), ndots(R_), mode(R_), nh(R_);
    std::vector<double> err_old(R_, 1e20), err(R_, 1e20), a_host((size_t)R_ * L_, 0.0), var((size_t)R_ * I_);
    int *d_active = comp_->active_device();
    int *d_head = ctl_.as<int>(), *d_flag = d_head + R_, *d_ndots = d_flag + R_, *d_mode = d_ndots + R_, *d_nh = d_mode + R_;
    double *d_mix = am_a_.as<double>(), *d_a = d_mix + R_;
    double *d_mean = stats_.as<double>(), *d_var = d_mean + (size_t)R_ * S_;
    double *w_imag = w_aux_.as<double>() + (size_t)(S_ - I_) * M_;
    std::vector<double> scale(I_);
    for (int c = 0; c < I_; c++) scale[c] = cfg_.dt_scaling[cfg_.imag_idx[c]];

    for (int it = 1; it <= cfg_.max_iter; it++) {
        bool any = false;
        for (int r = 0; r < R_; r++) any = any || active[r];
        if (!any) break;
        check_rc(lfts_memcpy_h2d(ctx_, d_active, active.data(), sizeof(int) * R_));
        check_rc(lfts_lfts_monomer_fields(ctx_, R_, S_, M_, cfg_.A.data(), w_aux_.as<double>(), w_mono_ptrs_.data()));
        comp_->enqueue_statistics();
        // d = dt_scaling * dH/dw for the imaginary fields (the AM residual of lfts.py:858-863)
        check_rc(lfts_lfts_field_deriv(ctx_, R_, S_, M_, I_, cfg_.imag_idx.data(), scale.data(), cfg_.A.data(),
                                       cfg_.h_coef_mu1.data(), cfg_.h_coef_mu2.data(), w_aux_.as<double>(),
                                       (const double *const *)phi_ptrs_.data(), d_cur_.as<double>(), d_active));
        check_rc(lfts_lfts_row_moments(ctx_, d_cur_.as<double>(), R_, I_, M_, M_, nI, nullptr, partials_.as<double>(), d_mean,
                                       d_var));
        check_rc(lfts_lfts_row_moments(ctx_, d_cur_.as<double>(), R_, I_, M_, M_, nI, d_mean, partials_.as<double>(),
                                       stats_.as<double>() + 2 * (size_t)R_ * S_, d_var));
        check_rc(lfts_memcpy_d2h(ctx_, var.data(), d_var, sizeof(double) * R_ * I_));
        bool need_dots = false;
        for (int r = 0; r < R_; r++) {
            head_flag[r] = 0;
            ndots[r] = 0;
            mode[r] = 0;
            nh[r] = 0;
            if (!active[r]) continue;
            double e = 0.0;
            for (int c = 0; c < I_; c++) {
                const double sd = std::sqrt(std::max(var[(size_t)r * I_ + c], 0.0)) / scale[c];
                e = (c == 0 || sd > e || std::isnan(sd)) ? sd : e;
            }
            err_old[r] = err[r];
            err[r] = e;
            st.iterations[r] = it;
            st.error[r] = e;
            if (e < cfg_.tolerance) {
                active[r] = 0;  // converged: this replica's fields and statistics stay as they are
                continue;
            }
            // Anderson-mixing control (CpuAndersonMixing.cpp:86-121)
            if (e < cfg_.am_start_error || n_anderson_[r] >= 0) n_anderson_[r]++;
            if (n_anderson_[r] >= 0) {
                n_anderson_[r] = std::min(cfg_.am_max_hist, n_anderson_[r]);
                head_[r] = (head_[r] + 1) % L_;
                head_flag[r] = 1;
                ndots[r] = n_anderson_[r] + 1;
                need_dots = true;
            }
            if (n_anderson_[r] <= 0) {
                mix_[r] = (err_old[r] < e) ? std::max(mix_[r] * 0.7, cfg_.am_mix_min) : mix_[r] * 1.01;
                mode[r] = 1;
            } else {
                mode[r] = 2;
                nh[r] = n_anderson_[r];
            }
        }
        std::vector<int> hd(head_.begin(), head_.end());
        for (int r = 0; r < R_; r++) hd[r] = std::max(hd[r], 0);
        check_rc(lfts_memcpy_h2d(ctx_, d_head, hd.data(), sizeof(int) * R_));
        check_rc(lfts_memcpy_h2d(ctx_, d_flag, head_flag.data(), sizeof(int) * R_));
        check_rc(lfts_memcpy_h2d(ctx_, d_ndots, ndots.data(), sizeof(int) * R_));
        if (need_dots) {
            check_rc(lfts_am_batch_insert(ctx_, R_, nI, L_, d_head, d_flag, w_imag, (long long)S_ * M_, d_cur_.as<double>(), nI,
                                          am_w_.as<double>(), am_d_.as<double>()));
            check_rc(lfts_am_batch_dots(ctx_, R_, nI, L_, d_head, d_ndots, am_d_.as<double>(), partials_.as<double>(),
                                        am_dots_.as<double>()));
            std::vector<double> dots((size_t)R_ * L_);
            check_rc(lfts_memcpy_d2h(ctx_, dots.data(), am_dots_.get(), sizeof(double) * dots.size()));
            for (int r = 0; r < R_; r++) {
                if (!ndots[r]) continue;
                auto &rows = dot_rows_[r];
                rows.insert(rows.begin(), std::vector<double>(dots.begin() + (size_t)r * L_, dots.begin() + (size_t)r * L_ + ndots[r]));
                if ((int)rows.size() > L_) rows.resize(L_);
                if (mode[r] == 2) {
                    const int n = nh[r];
                    std::vector<std::vector<double>> u(n, std::vector<double>(n));
                    std::vector<double> v(n), a(n);
                    for (int i = 0; i < n; i++) {
                        v[i] = rows[0][0] - rows[0][i + 1];
                        for (int j = 0; j < n; j++)
                            u[i][j] = rows[0][0] - rows[0][i + 1] - rows[0][j + 1] + rows[std::min(i + 1, j + 1)][std::abs(i - j)];
                    }
                    solve_no_pivot(u, v, a, n);
                    for (int i = 0; i < n; i++) a_host[(size_t)r * L_ + i] = a[i];
                }
            }
        }
        check_rc(lfts_memcpy_h2d(ctx_, d_mode, mode.data(), sizeof(int) * R_));
        check_rc(lfts_memcpy_h2d(ctx_, d_nh, nh.data(), sizeof(int) * R_));
        check_rc(lfts_memcpy_h2d(ctx_, d_mix, mix_.data(), sizeof(double) * R_));
        check_rc(lfts_memcpy_h2d(ctx_, d_a, a_host.data(), sizeof(double) * a_host.size()));
        check_rc(lfts_am_batch_update(ctx_, R_, nI, L_, d_head, d_mode, d_nh, d_mix, d_a, w_imag, (long long)S_ * M_,
                                      d_cur_.as<double>(), nI, am_w_.as<double>(), am_d_.as<double>(), w_imag,
                                      (long long)S_ * M_));
    }
}

// The same iterations with the control on the device (lfts_saddle_control,
// lfts_am_batch_solve): no host round trip inside an iteration.  The host
// polls the "any replica active" word of iteration it - 1 while iteration it
// is queued; an iteration queued after the last replica converged changes
// nothing (every kernel skips inactive replicas or recomputes the same values).
lfts_saddle_state BatchedLangevin::saddle_state() {
    lfts_saddle_state ss;
    int *si = sint_.as<int>();
    int *d_head = ctl_.as<int>();
    ss.active = comp_->active_device();
    ss.n_anderson = si;
    ss.head_raw = si + R_;
    ss.iter = si + 2 * R_;
    ss.any_active = si + 3 * R_;
    ss.loop_iter = si + 3 * R_ + 1;
    ss.head = d_head;
    ss.flag = d_head + R_;
    ss.ndots = d_head + 2 * R_;
    ss.mode = d_head + 3 * R_;
    ss.nh = d_head + 4 * R_;
    ss.err = sdbl_.as<double>();
    ss.err_old = ss.err + R_;
    ss.mix = am_a_.as<double>();
    return ss;
}

void BatchedLangevin::saddle_loop_device(SaddleStats &st) {
    const long long nI = (long long)I_ * M_;
    int *d_active = comp_->active_device();
    int *d_head = ctl_.as<int>(), *d_flag = d_head + R_, *d_ndots = d_flag + R_, *d_mode = d_ndots + R_, *d_nh = d_mode + R_;
    double *d_mix = am_a_.as<double>(), *d_a = d_mix + R_;
    double *d_mean = stats_.as<double>(), *d_var = d_mean + (size_t)R_ * S_;
    double *w_imag = w_aux_.as<double>() + (size_t)(S_ - I_) * M_;
    std::vector<double> scale(I_);
    for (int c = 0; c < I_; c++) scale[c] = cfg_.dt_scaling[cfg_.imag_idx[c]];
    lfts_saddle_state ss = saddle_state();
    int *si = sint_.as<int>();
    // initial state of every replica: active, no Anderson history (am_reset)
    {
        std::vector<int> ints((size_t)3 * R_);
        std::fill(ints.begin(), ints.begin() + 2 * R_, -1);
        std::vector<int> ones(R_, 1);
        std::vector<double> err((size_t)2 * R_, 1e20), mix(R_, cfg_.am_mix_init);
        check_rc(lfts_memcpy_h2d(ctx_, si, ints.data(), sizeof(int) * ints.size()));
        check_rc(lfts_memcpy_h2d(ctx_, d_active, ones.data(), sizeof(int) * R_));
        check_rc(lfts_memcpy_h2d(ctx_, ss.err, err.data(), sizeof(double) * err.size()));
        check_rc(lfts_memcpy_h2d(ctx_, d_mix, mix.data(), sizeof(double) * R_));
    }
    for (int it = 1; it <= cfg_.max_iter; it++) {
        check_rc(lfts_lfts_monomer_fields(ctx_, R_, S_, M_, cfg_.A.data(), w_aux_.as<double>(), w_mono_ptrs_.data()));
        comp_->enqueue_statistics();
        check_rc(lfts_lfts_field_deriv(ctx_, R_, S_, M_, I_, cfg_.imag_idx.data(), scale.data(), cfg_.A.data(),
                                       cfg_.h_coef_mu1.data(), cfg_.h_coef_mu2.data(), w_aux_.as<double>(),
                                       (const double *const *)phi_ptrs_.data(), d_cur_.as<double>(), d_active));
        check_rc(lfts_lfts_row_moments(ctx_, d_cur_.as<double>(), R_, I_, M_, M_, nI, nullptr, partials_.as<double>(), d_mean,
                                       d_var));
        check_rc(lfts_lfts_row_moments(ctx_, d_cur_.as<double>(), R_, I_, M_, M_, nI, d_mean, partials_.as<double>(),
                                       stats_.as<double>() + 2 * (size_t)R_ * S_, d_var));
        check_rc(lfts_saddle_control(ctx_, R_, I_, it, d_var, scale.data(), cfg_.tolerance, cfg_.am_start_error,
                                     cfg_.am_max_hist, cfg_.am_mix_min, &ss));
        check_rc(lfts_am_batch_insert(ctx_, R_, nI, L_, d_head, d_flag, w_imag, (long long)S_ * M_, d_cur_.as<double>(), nI,
                                      am_w_.as<double>(), am_d_.as<double>()));
        check_rc(lfts_am_batch_dots(ctx_, R_, nI, L_, d_head, d_ndots, am_d_.as<double>(), partials_.as<double>(),
                                    am_dots_.as<double>()));
        check_rc(lfts_am_batch_solve(ctx_, R_, L_, d_head, d_ndots, d_mode, d_nh, am_dots_.as<double>(), dot_ring_.as<double>(),
                                     d_a));
        check_rc(lfts_am_batch_update(ctx_, R_, nI, L_, d_head, d_mode, d_nh, d_mix, d_a, w_imag, (long long)S_ * M_,
                                      d_cur_.as<double>(), nI, am_w_.as<double>(), am_d_.as<double>(), w_imag,
                                      (long long)S_ * M_));
        check_rc(lfts_status_post(ctx_, ss.any_active, it % LFTS_STATUS_SLOTS));
        if (it >= 2) {
            int any = 1;
            check_rc(lfts_status_wait(ctx_, (it - 1) % LFTS_STATUS_SLOTS, &any));
            if (!any) break;  // iteration it, already queued, finds no active replica
        }
    }
    std::vector<int> iter(R_);
    check_rc(lfts_memcpy_d2h(ctx_, iter.data(), ss.iter, sizeof(int) * R_));
    check_rc(lfts_memcpy_d2h(ctx_, st.error.data(), ss.err, sizeof(double) * R_));
    st.iterations.assign(iter.begin(), iter.end());
    // leave every replica active for propagator computations outside the loop
    const std::vector<int> ones(R_, 1);
    check_rc(lfts_memcpy_h2d(ctx_, d_active, ones.data(), sizeof(int) * R_));
}

bool BatchedLangevin::graph_mode() const {
    return step_graph_on_ && !host_control_ && cfg_.am_max_hist <= LFTS_AM_SOLVE_MAX_HIST && poly_coef_.size() <= 8;
}

// this step's noise into the buffer the update reads as "current"
void BatchedLangevin::put_noise(const double *noise_dev) {
    if (Rr_ > 0 && noise_dev)
        check_rc(lfts_memcpy_d2d_async(ctx_, xi_[1 - xi_cur_].get(), noise_dev, sizeof(double) * (size_t)R_ * Rr_ * M_));
}

// Leimkuhler-Matthews update of the real fields with xi_[parity] as the
// previous noise and xi_[1 - parity] as this step's; fields and concentrations
// are kept first for a restore
void BatchedLangevin::enqueue_update(int parity) {
    const size_t SM = (size_t)S_ * M_;
    check_rc(lfts_memcpy_d2d_async(ctx_, w_save_.get(), w_aux_.get(), w_aux_.size()));
    for (int r = 0; r < R_; r++)
        for (int s = 0; s < S_; s++)
            check_rc(lfts_memcpy_d2d_async(ctx_, phi_save_.as<double>() + r * SM + (size_t)s * M_, phi_ptrs_[s] + (size_t)r * M_,
                                           sizeof(double) * M_));
    if (Rr_ > 0) {
        std::vector<double> sc(Rr_);
        for (int c = 0; c < Rr_; c++) sc[c] = cfg_.dt_scaling[cfg_.real_idx[c]];
        check_rc(lfts_lfts_langevin(ctx_, R_, S_, M_, Rr_, cfg_.real_idx.data(), cfg_.A.data(), cfg_.h_coef_mu1.data(),
                                    cfg_.h_coef_mu2.data(), (const double *const *)phi_ptrs_.data(), cfg_.dt, sc.data(),
                                    w_aux_.as<double>(), xi_[parity].as<double>(), xi_[1 - parity].as<double>(), nullptr));
    }
}

// one saddle-point iteration of every active replica, control on the device
void BatchedLangevin::enqueue_search_body(const lfts_saddle_state &ss) {
    const long long nI = (long long)I_ * M_;
    double *d_a = am_a_.as<double>() + R_;
    double *d_mean = stats_.as<double>(), *d_var = d_mean + (size_t)R_ * S_;
    double *w_imag = w_aux_.as<double>() + (size_t)(S_ - I_) * M_;
    std::vector<double> scale(I_);
    for (int c = 0; c < I_; c++) scale[c] = cfg_.dt_scaling[cfg_.imag_idx[c]];
    check_rc(lfts_lfts_monomer_fields(ctx_, R_, S_, M_, cfg_.A.data(), w_aux_.as<double>(), w_mono_ptrs_.data()));
    comp_->enqueue_statistics(false);
    check_rc(lfts_lfts_field_deriv(ctx_, R_, S_, M_, I_, cfg_.imag_idx.data(), scale.data(), cfg_.A.data(),
                                   cfg_.h_coef_mu1.data(), cfg_.h_coef_mu2.data(), w_aux_.as<double>(),
                                   (const double *const *)phi_ptrs_.data(), d_cur_.as<double>(), ss.active));
    check_rc(lfts_lfts_row_moments(ctx_, d_cur_.as<double>(), R_, I_, M_, M_, nI, nullptr, partials_.as<double>(), d_mean, d_var));
    check_rc(lfts_lfts_row_moments(ctx_, d_cur_.as<double>(), R_, I_, M_, M_, nI, d_mean, partials_.as<double>(),
                                   stats_.as<double>() + 2 * (size_t)R_ * S_, d_var));
    check_rc(lfts_saddle_control(ctx_, R_, I_, 0, d_var, scale.data(), cfg_.tolerance, cfg_.am_start_error, cfg_.am_max_hist,
                                 cfg_.am_mix_min, &ss));
    check_rc(lfts_am_batch_insert(ctx_, R_, nI, L_, ss.head, ss.flag, w_imag, (long long)S_ * M_, d_cur_.as<double>(), nI,
                                  am_w_.as<double>(), am_d_.as<double>()));
    check_rc(lfts_am_batch_dots(ctx_, R_, nI, L_, ss.head, ss.ndots, am_d_.as<double>(), partials_.as<double>(),
                                am_dots_.as<double>()));
    check_rc(lfts_am_batch_solve(ctx_, R_, L_, ss.head, ss.ndots, ss.mode, ss.nh, am_dots_.as<double>(), dot_ring_.as<double>(),
                                 d_a));
    check_rc(lfts_am_batch_update(ctx_, R_, nI, L_, ss.head, ss.mode, ss.nh, ss.mix, d_a, w_imag, (long long)S_ * M_,
                                  d_cur_.as<double>(), nI, am_w_.as<double>(), am_d_.as<double>(), w_imag, (long long)S_ * M_));
}

// the saddle-point search of a step as device work: reset, WHILE loop of
// iterations, moments, Hamiltonian, pressure shift, restore of failed replicas
void BatchedLangevin::enqueue_search(bool restore) {
    const lfts_saddle_state ss = saddle_state();
    const long long k0 = lfts_ctx_launches(ctx_);
    check_rc(lfts_saddle_begin(ctx_, R_, cfg_.am_mix_init, &ss));
    unsigned long long handle = 0;
    check_rc(lfts_graph_while_begin(ctx_, &handle));
    const long long k1 = lfts_ctx_launches(ctx_);
    enqueue_search_body(ss);
    check_rc(lfts_saddle_next(ctx_, handle, &ss, cfg_.max_iter));
    const long long k2 = lfts_ctx_launches(ctx_);
    check_rc(lfts_graph_while_end(ctx_));
    double *d_mean = stats_.as<double>(), *d_var = d_mean + (size_t)R_ * S_;
    check_rc(lfts_lfts_row_moments(ctx_, w_aux_.as<double>(), R_, S_, M_, M_, (long long)S_ * M_, nullptr, partials_.as<double>(),
                                   d_mean, d_var));
    check_rc(lfts_lfts_step_finish(ctx_, R_, S_, (int)poly_coef_.size(), M_, &ss, cfg_.tolerance, d_mean, d_var,
                                   comp_->partition_device(), cfg_.h_coef_mu1.data(), cfg_.h_coef_mu2.data(), cfg_.h_const,
                                   poly_coef_.data(), restore ? 1 : 0, w_aux_.as<double>(), w_save_.as<double>(),
                                   phi_ptrs_.data(), phi_save_.as<double>(), fin_scratch_.as<double>(), fin_stats_.as<double>()));
    k_body_ = k2 - k1;
    k_search_fixed_ = (lfts_ctx_launches(ctx_) - k0) - k_body_;
}

// the packed statistics of lfts_lfts_step_finish (one copy, which also waits for the step)
SaddleStats BatchedLangevin::read_stats() {
    const int P = (int)poly_coef_.size();
    std::vector<double> h((size_t)4 * R_ + (size_t)R_ * P + (size_t)2 * R_ * S_);
    check_rc(lfts_memcpy_d2h(ctx_, h.data(), fin_stats_.get(), sizeof(double) * h.size()));
    SaddleStats st;
    st.iterations.resize(R_);
    st.error.resize(R_);
    st.hamiltonian.resize(R_);
    st.failed.resize(R_);
    int it_max = 0;
    for (int r = 0; r < R_; r++) {
        st.iterations[r] = (int)h[r];
        st.error[r] = h[R_ + r];
        st.hamiltonian[r] = h[2 * R_ + r];
        st.failed[r] = h[3 * R_ + r] != 0.0 ? 1 : 0;
        it_max = std::max(it_max, st.iterations[r]);
    }
    const double *o = h.data() + 4 * (size_t)R_;
    st.partitions.assign(o, o + (size_t)R_ * P);
    o += (size_t)R_ * P;
    st.aux_mean.assign(o, o + (size_t)R_ * S_);
    st.aux_msq.assign(o + (size_t)R_ * S_, o + (size_t)2 * R_ * S_);
    comp_->count_replayed(k_search_fixed_ + k_body_ * (long long)std::max(it_max, 1));
    return st;
}

SaddleStats BatchedLangevin::step(const double *noise) {
    if (Rr_ > 0) {
        DevBuf &cur = xi_[1 - xi_cur_];
        check_rc(lfts_memcpy_h2d(ctx_, cur.get(), noise, sizeof(double) * (size_t)R_ * Rr_ * M_));
    }
    return step_device(nullptr);
}

SaddleStats BatchedLangevin::step_device(const double *noise_dev) {
    if (!graph_mode()) {
        langevin_update_device(noise_dev);
        return find_saddle_point(true);
    }
    put_noise(noise_dev);
    const int par = xi_cur_;
    if (!g_step_[par]) {
        const long long k0 = lfts_ctx_launches(ctx_);
        check_rc(lfts_graph_begin(ctx_));
        enqueue_update(par);
        k_update_ = lfts_ctx_launches(ctx_) - k0;
        enqueue_search(true);
        check_rc(lfts_graph_end(ctx_, &g_step_[par]));
    }
    check_rc(lfts_graph_launch(ctx_, g_step_[par]));
    if (Rr_ > 0) xi_cur_ = 1 - xi_cur_;  // this step's draw is the next step's "previous" noise (lfts.py:708-709)
    comp_->count_replayed(k_update_);
    return read_stats();
}

void BatchedLangevin::langevin_update_device(const double *noise_dev) {
    if (graph_mode()) {
        put_noise(noise_dev);
        const int par = xi_cur_;
        if (!g_update_[par]) {
            const long long k0 = lfts_ctx_launches(ctx_);
            check_rc(lfts_graph_begin(ctx_));
            enqueue_update(par);
            check_rc(lfts_graph_end(ctx_, &g_update_[par]));
            k_update_ = lfts_ctx_launches(ctx_) - k0;
        }
        check_rc(lfts_graph_launch(ctx_, g_update_[par]));
        comp_->count_replayed(k_update_);
        if (Rr_ > 0) xi_cur_ = 1 - xi_cur_;
        return;
    }
    const size_t SM = (size_t)S_ * M_;
    // keep the fields and concentrations to restore replicas whose saddle point fails
    check_rc(lfts_memcpy_d2d_async(ctx_, w_save_.get(), w_aux_.get(), w_aux_.size()));
    for (int r = 0; r < R_; r++)
        for (int s = 0; s < S_; s++)
            check_rc(lfts_memcpy_d2d_async(ctx_, phi_save_.as<double>() + r * SM + (size_t)s * M_, phi_ptrs_[s] + (size_t)r * M_,
                                           sizeof(double) * M_));
    if (Rr_ > 0) {
        DevBuf &cur = xi_[1 - xi_cur_];
        if (noise_dev)
            check_rc(lfts_memcpy_d2d_async(ctx_, cur.get(), noise_dev, sizeof(double) * (size_t)R_ * Rr_ * M_));
        std::vector<double> s(Rr_);
        for (int c = 0; c < Rr_; c++) s[c] = cfg_.dt_scaling[cfg_.real_idx[c]];
        check_rc(lfts_lfts_langevin(ctx_, R_, S_, M_, Rr_, cfg_.real_idx.data(), cfg_.A.data(), cfg_.h_coef_mu1.data(),
                                    cfg_.h_coef_mu2.data(), (const double *const *)phi_ptrs_.data(), cfg_.dt, s.data(),
                                    w_aux_.as<double>(), xi_[xi_cur_].as<double>(), cur.as<double>(), nullptr));
        xi_cur_ = 1 - xi_cur_;  // this step's draw is the next step's "previous" noise (lfts.py:708-709)
    }
}

void BatchedLangevin::langevin_update_rng(double sigma) {
    if (!pcg_.get()) LFTS_THROW("no device noise streams (set_noise_streams first)");
    check_rc(lfts_pcg64_normal(ctx_, pcg_.as<unsigned long long>(), R_, (long long)Rr_ * M_, sigma, noise_buf_.as<double>()));
    langevin_update_device(noise_buf_.as<double>());
}

void BatchedLangevin::set_noise_streams(const unsigned long long *states) {
    if (Rr_ < 1) LFTS_THROW("no real auxiliary field draws noise");
    if (!pcg_.get()) {
        pcg_.alloc(ctx_, sizeof(unsigned long long) * 4 * (size_t)R_);
        noise_buf_.alloc(ctx_, sizeof(double) * (size_t)R_ * Rr_ * M_);
    }
    check_rc(lfts_memcpy_h2d(ctx_, pcg_.get(), states, pcg_.size()));
}
void BatchedLangevin::get_noise_streams(unsigned long long *states) const {
    if (!pcg_.get()) LFTS_THROW("no device noise streams (set_noise_streams first)");
    check_rc(lfts_memcpy_d2h(ctx_, states, pcg_.get(), pcg_.size()));
}
SaddleStats BatchedLangevin::step_device_rng(double sigma) {
    if (!pcg_.get()) LFTS_THROW("no device noise streams (set_noise_streams first)");
    check_rc(lfts_pcg64_normal(ctx_, pcg_.as<unsigned long long>(), R_, (long long)Rr_ * M_, sigma, noise_buf_.as<double>()));
    return step_device(noise_buf_.as<double>());
}

void BatchedLangevin::get_noise_prev(double *out) const {
    if (Rr_ > 0) check_rc(lfts_memcpy_d2h(ctx_, out, xi_[xi_cur_].get(), sizeof(double) * (size_t)R_ * Rr_ * M_));
}
void BatchedLangevin::set_noise_prev(const double *in) {
    if (Rr_ > 0) check_rc(lfts_memcpy_h2d(ctx_, xi_[xi_cur_].get(), in, sizeof(double) * (size_t)R_ * Rr_ * M_));
}

long long BatchedLangevin::n_complex_grid() const {
    long long M = 0, Mc = 0;
    check_rc(lfts_ctx_info(ctx_, &M, &Mc, nullptr));
    return Mc;
}

void BatchedLangevin::sf_accumulate(const double *coef, const std::vector<int> &pairs) {
    const int np = (int)pairs.size() / 2;
    if (np < 1 || (int)pairs.size() != 2 * np) LFTS_THROW("pairs must hold (a, b) monomer type indices");
    for (int v : pairs)
        if (v < 0 || v >= S_) LFTS_THROW("monomer type index out of range in pairs");
    const long long Mc = n_complex_grid();
    const int W = S_ - 1;    // auxiliary fields 0..S-2 enter mu (lfts.py:760-762)
    const int F = S_ + W;    // transformed fields per replica: phi_0..phi_{S-1}, w_aux_0..w_aux_{S-2}
    if (!sf_spec_.get()) {
        sf_spec_.alloc(ctx_, 2 * sizeof(double) * (size_t)R_ * F * Mc);
        std::vector<lfts_step_job> jobs((size_t)R_ * F);
        for (int r = 0; r < R_; r++)
            for (int f = 0; f < F; f++) {
                lfts_step_job jb;
                std::memset(&jb, 0, sizeof jb);
                jb.in = f < S_ ? (const void *)(phi_ptrs_[f] + (size_t)r * M_)
                               : (const void *)(w_aux_.as<double>() + ((size_t)r * S_ + (f - S_)) * M_);
                jb.spec = sf_spec_.as<double>() + 2 * ((size_t)r * F + f) * Mc;
                jobs[(size_t)r * F + f] = jb;
            }
        sf_jobs_.alloc(ctx_, sizeof(lfts_step_job) * jobs.size());
        check_rc(lfts_memcpy_h2d(ctx_, sf_jobs_.get(), jobs.data(), sf_jobs_.size()));
        sf_coef_.alloc(ctx_, sizeof(double) * (size_t)std::max(W, 1) * S_);
    }
    if (np != sf_np_ || pairs != sf_pairs_host_) {
        sf_acc_.alloc(ctx_, 2 * sizeof(double) * (size_t)R_ * np * Mc);
        check_rc(lfts_memset_async(ctx_, sf_acc_.get(), 0, sf_acc_.size()));
        sf_pairs_.alloc(ctx_, sizeof(int) * pairs.size());
        check_rc(lfts_memcpy_h2d(ctx_, sf_pairs_.get(), pairs.data(), sf_pairs_.size()));
        sf_np_ = np;
        sf_pairs_host_ = pairs;
    }
    if (W > 0) check_rc(lfts_memcpy_h2d(ctx_, sf_coef_.get(), coef, sizeof(double) * (size_t)W * S_));
    check_rc(lfts_fft_forward(ctx_, sf_jobs_.as<lfts_step_job>(), R_ * F));
    check_rc(lfts_sf_accumulate(ctx_, R_, S_, W, sf_spec_.get(), sf_coef_.as<double>(), 1.0 / (double)M_, np,
                                sf_pairs_.as<int>(), sf_acc_.get()));
}

void BatchedLangevin::sf_get(double *out, bool reset) {
    if (!sf_np_) LFTS_THROW("no structure function has been accumulated");
    check_rc(lfts_memcpy_d2h(ctx_, out, sf_acc_.get(), sf_acc_.size()));
    if (reset) check_rc(lfts_memset_async(ctx_, sf_acc_.get(), 0, sf_acc_.size()));
}

}  // namespace lfts
