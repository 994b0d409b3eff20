// Device-resident SCFT iteration (examples/scft/scft.py:617-736).
#include "lfts_scft.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace lfts {

DeviceScft::DeviceScft(ComputationBox *cb, Molecules *mol, PropagatorAnalyzer *pa, int precision, int device,
                       const ScftConfig &cfg)
    : cfg_(cfg), cb_(cb), mol_(mol) {
    S_ = (int)cfg.monomer_types.size();
    if (S_ < 1 || S_ > LFTS_MAX_MONOMERS) LFTS_THROW("number of monomer types must be 1.." + std::to_string(LFTS_MAX_MONOMERS));
    if ((int)cfg.chi.size() != S_ * S_ || (int)cfg.P.size() != S_ * S_ || (int)cfg.A_inv.size() != S_ * S_)
        LFTS_THROW("chi, P and A_inv must be S x S");
    if (cfg.optimizer != "am" && cfg.optimizer != "adam") LFTS_THROW("optimizer must be \"am\" or \"adam\"");
    if (mol->get_n_solvent_types() > 0) LFTS_THROW("the device SCFT loop does not support solvents");
    for (const auto &t : cfg.monomer_types)
        if (!mol->get_bond_lengths().count(t)) LFTS_THROW("monomer type " + t + " is not in the molecules");
    comp_.reset(new GpuComputation(cb, mol, pa, precision, device, 1));
    ctx_ = comp_->context();
    M_ = comp_->n_grid();
    dim_ = cb->get_dim();
    n_var_ = (long long)S_ * M_ + (cfg.box_altering ? dim_ : 0);
    cur_.alloc(ctx_, sizeof(double) * n_var_);
    diff_.alloc(ctx_, sizeof(double) * n_var_);
    new_.alloc(ctx_, sizeof(double) * n_var_);
    waux_.alloc(ctx_, sizeof(double) * (size_t)S_ * M_);
    ones_.alloc(ctx_, sizeof(double) * M_);
    scal_.alloc(ctx_, sizeof(double) * 8 * S_);
    std::vector<double> ones((size_t)M_, 1.0);
    check_rc(lfts_memcpy_h2d(ctx_, ones_.get(), ones.data(), ones_.size()));
    check_rc(lfts_memset_async(ctx_, cur_.get(), 0, cur_.size()));
    check_rc(lfts_memset_async(ctx_, diff_.get(), 0, diff_.size()));
    for (const auto &t : cfg.monomer_types) {
        phi_.push_back(comp_->phi_type_device(t));
        wdev_.push_back(comp_->w_device(t));
    }
    // reduction jobs, fixed pointers: [0,S) means of residual rows; [S,6S) per
    // iteration sums (|w_diff|^2 dv, |w|^2 dv, mean phi, mean w_aux, mean w_aux^2);
    // [6S,7S) means of field rows
    const double inv_m = 1.0 / (double)M_, dv = cb->get_volume() / (double)M_;
    const double *cur = cur_.as<double>(), *dif = diff_.as<double>(), *aux = waux_.as<double>(), *one = ones_.as<double>();
    std::vector<lfts_dot_job> jobs((size_t)7 * S_);
    for (int i = 0; i < S_; i++) {
        const size_t o = (size_t)i * M_;
        jobs[i] = {dif + o, one, nullptr, inv_m};
        jobs[S_ + i] = {dif + o, dif + o, nullptr, dv};
        jobs[2 * S_ + i] = {cur + o, cur + o, nullptr, dv};
        jobs[3 * S_ + i] = {phi_[i], one, nullptr, inv_m};
        jobs[4 * S_ + i] = {aux + o, one, nullptr, inv_m};
        jobs[5 * S_ + i] = {aux + o, aux + o, nullptr, inv_m};
        jobs[6 * S_ + i] = {cur + o, one, nullptr, inv_m};
    }
    jobs_.alloc(ctx_, sizeof(lfts_dot_job) * jobs.size());
    check_rc(lfts_memcpy_h2d(ctx_, jobs_.get(), jobs.data(), jobs_.size()));
    if (cfg.optimizer == "am") {
        am_.reset(new GpuAndersonMixing((int)n_var_, cfg.am_max_hist, cfg.am_start_error, cfg.am_mix_min, cfg.am_mix_init,
                                        device));
    } else {
        m_.alloc(ctx_, sizeof(double) * n_var_);
        v_.alloc(ctx_, sizeof(double) * n_var_);
    }
    reset();
}

DeviceScft::~DeviceScft() = default;

void DeviceScft::reset() {
    if (am_) am_->reset_count();
    if (m_.get()) {
        check_rc(lfts_memset_async(ctx_, m_.get(), 0, m_.size()));
        check_rc(lfts_memset_async(ctx_, v_.get(), 0, v_.size()));
    }
    adam_count_ = 1;
    err_ = err_old_ = 1e20;
    evaluated_ = false;
}

// means of S rows (stride M) starting at rows, by the matching prebuilt jobs
void DeviceScft::row_means(const double *rows, double *d_out) {
    const lfts_dot_job *j = jobs_.as<lfts_dot_job>() + (rows == diff_.as<double>() ? 0 : 6 * S_);
    check_rc(lfts_dots_static(8, M_, j, S_, d_out, lfts_ctx_stream(ctx_)));
    for (int i = 0; i < S_; i++)
        check_rc(lfts_lfts_subtract_mean(ctx_, const_cast<double *>(rows), 1, S_, i, M_, d_out + i, nullptr));
}

void DeviceScft::set_fields(const double *w) {
    check_rc(lfts_memcpy_h2d(ctx_, cur_.get(), w, sizeof(double) * (size_t)S_ * M_));
    row_means(cur_.as<double>(), scal_.as<double>() + 6 * S_);
    evaluated_ = false;
}

void DeviceScft::get_fields(double *w) const {
    check_rc(lfts_memcpy_d2h(ctx_, w, cur_.get(), sizeof(double) * (size_t)S_ * M_));
}

void DeviceScft::get_concentrations(double *phi) const {
    for (int i = 0; i < S_; i++) check_rc(lfts_memcpy_d2h(ctx_, phi + (size_t)i * M_, phi_[i], sizeof(double) * M_));
}

ScftStats DeviceScft::evaluate() {
    const double *cur = cur_.as<double>();
    double *dif = diff_.as<double>(), *sc = scal_.as<double>();
    for (int i = 0; i < S_; i++)
        check_rc(lfts_memcpy_d2d_async(ctx_, wdev_[i], cur + (size_t)i * M_, sizeof(double) * M_));
    comp_->enqueue_statistics();
    // w_diff_i = sum_j chi_ij phi_j - P_ij w_j, then zero mean (scft.py:661-672)
    std::vector<const double *> src;
    std::vector<double> coef;
    for (int i = 0; i < S_; i++) {
        src.clear();
        coef.clear();
        for (int j = 0; j < S_; j++) {
            src.push_back(phi_[j]);
            coef.push_back(cfg_.chi[(size_t)i * S_ + j]);
            src.push_back(cur + (size_t)j * M_);
            coef.push_back(-cfg_.P[(size_t)i * S_ + j]);
        }
        check_rc(lfts_lincomb(ctx_, dif + (size_t)i * M_, (int)src.size(), src.data(), coef.data(), M_));
    }
    row_means(dif, sc);
    // w_aux = A_inv w for the Hamiltonian's field averages
    std::vector<const double *> rows;
    for (int j = 0; j < S_; j++) rows.push_back(cur + (size_t)j * M_);
    for (int k = 0; k < S_; k++)
        check_rc(lfts_lincomb(ctx_, waux_.as<double>() + (size_t)k * M_, S_, rows.data(), cfg_.A_inv.data() + (size_t)k * S_, M_));
    check_rc(lfts_dots_static(8, M_, jobs_.as<lfts_dot_job>() + S_, 5 * S_, sc + S_, lfts_ctx_stream(ctx_)));
    std::vector<double> h((size_t)5 * S_);
    check_rc(lfts_memcpy_d2h(ctx_, h.data(), sc + S_, sizeof(double) * h.size()));
    ScftStats st;
    st.partitions = comp_->partitions_host();
    double dd = 0.0, ww = 1.0, phit = 0.0;  // 1.0 prevents dividing by zero (scft.py:682)
    for (int i = 0; i < S_; i++) {
        dd += h[i];
        ww += h[S_ + i];
        phit += h[2 * S_ + i];
        st.aux_mean.push_back(h[3 * S_ + i]);
        st.aux_msq.push_back(h[4 * S_ + i]);
    }
    st.error_level = std::sqrt(dd / ww);
    st.mass_error = phit - 1.0;
    st.lx = cb_->get_lx();
    if (cfg_.box_altering) {
        comp_->compute_stress();
        st.stress = comp_->get_stress();
        double s2 = 0.0;
        for (double v : st.stress) s2 += v * v;
        st.error_level += std::sqrt(s2);
    }
    stress_ = st.stress;
    err_old_ = err_;
    err_ = st.error_level;
    evaluated_ = true;
    return st;
}

void DeviceScft::update() {
    if (!evaluated_) LFTS_THROW("update() needs an evaluate() at the current fields");
    const size_t SM = (size_t)S_ * M_;
    if (cfg_.box_altering) {
        // am_current = [w, lx], am_diff = [w_diff, -scale_stress * stress] (scft.py:698-701)
        std::vector<double> lx = cb_->get_lx(), dl(dim_);
        for (int d = 0; d < dim_; d++) dl[d] = cfg_.scale_stress * (-stress_[d]);
        check_rc(lfts_memcpy_h2d(ctx_, cur_.as<double>() + SM, lx.data(), sizeof(double) * dim_));
        check_rc(lfts_memcpy_h2d(ctx_, diff_.as<double>() + SM, dl.data(), sizeof(double) * dim_));
    }
    if (am_) {
        check_rc(lfts_synchronize(ctx_));
        am_->calculate_new_fields_device(new_.as<double>(), cur_.as<double>(), diff_.as<double>(), err_old_, err_);
    } else {
        const double lr = cfg_.adam_lr * std::pow(cfg_.adam_gamma, (double)(adam_count_ - 1));
        check_rc(lfts_adam_update(ctx_, new_.as<double>(), cur_.as<double>(), diff_.as<double>(), m_.as<double>(),
                                  v_.as<double>(), n_var_, lr, 0.9, 0.999, 1e-8, adam_count_));
        adam_count_++;
    }
    if (cfg_.box_altering) {
        // new box, each |dL/L| clipped to 10 % (scft.py:706-713)
        std::vector<double> got(dim_), old = cb_->get_lx(), lx(dim_);
        check_rc(lfts_memcpy_d2h(ctx_, got.data(), new_.as<double>() + SM, sizeof(double) * dim_));
        for (int d = 0; d < dim_; d++) {
            const double r = std::min(std::max((got[d] - old[d]) / old[d], -0.1), 0.1);
            lx[d] = (1.0 + r) * old[d];
        }
        cb_->set_lx(lx);
        comp_->update_laplacian_operator();
    }
    check_rc(lfts_memcpy_d2d_async(ctx_, cur_.get(), new_.get(), sizeof(double) * SM));
    row_means(cur_.as<double>(), scal_.as<double>() + 6 * S_);
    evaluated_ = false;
}

}  // namespace lfts
