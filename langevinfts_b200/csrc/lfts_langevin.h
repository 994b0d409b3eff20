// Batched Langevin field-theoretic simulation: many independent replicas of
// one system advance together; the propagators of every replica run in the
// same launches and each replica's saddle-point search stops on its own
// (examples/fts/lfts.py:631-868 of the reference, per replica).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "lfts_computation.h"

namespace lfts {

struct LangevinConfig {
    std::vector<std::string> monomer_types;  // sorted; order of the auxiliary/monomer field rows
    std::vector<double> A;                   // S*S, w = A w_aux
    std::vector<double> h_coef_mu1, h_coef_mu2;  // S-1
    double h_const = 0.0;
    std::vector<int> real_idx, imag_idx;     // imaginary fields must be the trailing block
    std::vector<double> dt_scaling;          // S
    double dt = 0.0;
    double tolerance = 1e-4;
    int max_iter = 100;
    int am_max_hist = 20;
    double am_start_error = 0.5, am_mix_min = 0.01, am_mix_init = 0.01;
};

struct SaddleStats {
    std::vector<int> iterations;      // per replica
    std::vector<double> error;        // per replica
    std::vector<double> hamiltonian;  // per replica
    std::vector<int> failed;          // per replica: tolerance not met (fields restored)
    std::vector<double> partitions;   // R x P
    std::vector<double> aux_mean;     // R x S: <w_aux[i]> at the returned fields (dH/dchiN, lfts.py:265-274)
    std::vector<double> aux_msq;      // R x S: <w_aux[i]^2>
};

class BatchedLangevin {
   public:
    BatchedLangevin(ComputationBox *cb, Molecules *mol, PropagatorAnalyzer *pa, int precision, int device, int n_replicas,
                    const LangevinConfig &cfg);
    ~BatchedLangevin();
    int n_replicas() const { return R_; }
    int n_grid() const { return (int)M_; }
    int n_real() const { return (int)cfg_.real_idx.size(); }
    void set_fields(const double *w_aux);  // host [R][S][M]
    void get_fields(double *w_aux) const;
    void get_concentrations(double *phi) const;  // host [R][S][M], monomer_types order
    SaddleStats find_saddle_point(bool restore_on_failure = false);
    // Saddle-point control on the host (one round trip per iteration for the
    // errors and one for the Anderson dots) instead of on the device; the two
    // give the same iterates.  The host form also serves am_max_hist > 32.
    void set_host_control(bool on) { host_control_ = on; }
    bool host_control() const { return host_control_; }
    // One Langevin step of every replica; noise host [R][n_real][M] (the draw of this step)
    SaddleStats step(const double *noise);
    // Same, with this step's noise already on the device ([R][n_real][M] doubles)
    SaddleStats step_device(const double *noise_dev);
    void *stream() const { return lfts_ctx_stream(ctx_); }
    // The previous step's noise of every replica ([R][n_real][M] host doubles),
    // the state the Leimkuhler-Matthews update carries between steps
    // (normal_noise_prev of lfts.py:569-629): read for a checkpoint, written on
    // resume.
    void get_noise_prev(double *out) const;
    void set_noise_prev(const double *in);
    // Noise drawn on the device from one PCG64 stream per replica
    // (lfts_pcg64_normal): states host [R][4] uint64 (state hi, lo, inc hi,
    // lo), the state of numpy's PCG64 of the replica.  step_device_rng draws
    // this step's noise (sigma * N(0, 1), [R][n_real][M]) and steps.
    void set_noise_streams(const unsigned long long *states);
    void get_noise_streams(unsigned long long *states) const;
    bool has_noise_streams() const { return pcg_.get() != nullptr; }
    SaddleStats step_device_rng(double sigma);
    // The two halves of a step, for a caller that changes the imaginary fields
    // in between (a learned saddle-point start): the Langevin update of the
    // real fields (saving fields and concentrations for a restore), then
    // find_saddle_point(true).  w_aux_device: the [R][S][M] fields, written on
    // stream() only.
    void langevin_update_device(const double *noise_dev);
    void langevin_update_rng(double sigma);
    double *w_aux_device() { return w_aux_.as<double>(); }
    // Structure function of every replica (examples/fts/lfts.py:753-767):
    //   sf[r][p] += mu_a conj(phi_b / M),  mu_a = sum_{q < S-1} F[w_aux_q] coef[q][a],
    // for the type pairs p = (pairs[2p], pairs[2p+1]); coef (host, (S-1) x S) =
    // A_inv[q][a] / eigenvalue[q] / M.  A new pair set starts new (zeroed) sums.
    // Double-precision engines only.
    void sf_accumulate(const double *coef, const std::vector<int> &pairs);
    // the sums as host complex doubles [R][npairs][nx][ny][nz/2+1]; reset zeroes them
    void sf_get(double *out, bool reset);
    int sf_npairs() const { return sf_np_; }
    long long n_complex_grid() const;
    GpuComputation &computation() { return *comp_; }

    // One CUDA graph per Langevin step (default; set_step_graph(false) or the
    // host control or more than LFTS_AM_SOLVE_MAX_HIST histories fall back to
    // the loop driven from the host): the update of the real fields, then the
    // saddle loop as a conditional WHILE node controlled on the device, then
    // the Hamiltonian, pressure shift and restore-on-failure on the device.
    void set_step_graph(bool on) { step_graph_on_ = on; }
    bool step_graph() const { return graph_mode(); }

   private:
    void am_reset();
    void saddle_loop_host(SaddleStats &st);
    void saddle_loop_device(SaddleStats &st);
    lfts_saddle_state saddle_state();
    bool graph_mode() const;
    void enqueue_update(int parity);
    void enqueue_search_body(const lfts_saddle_state &ss);
    void enqueue_search(bool restore);
    SaddleStats read_stats();
    void put_noise(const double *noise_dev);
    double hamiltonian(int r, const std::vector<double> &mean, const std::vector<double> &msq, const std::vector<double> &Q) const;

    LangevinConfig cfg_;
    int R_, S_, I_, Rr_;
    long long M_;
    std::unique_ptr<GpuComputation> comp_;
    lfts_ctx ctx_;
    Molecules *mol_;
    DevBuf w_aux_, w_save_, phi_save_, d_cur_, xi_[2], partials_, stats_, ctl_, am_w_, am_d_, am_dots_, am_a_;
    // device saddle control: n_anderson, head_raw, iter (R ints each) + the
    // any-active word; err, err_old (R doubles each); dot ring R*L*L
    DevBuf sint_, sdbl_, dot_ring_;
    DevBuf pcg_, noise_buf_;  // device noise: PCG64 states [R][4], this step's draw [R][n_real][M]
    bool host_control_ = false;
    int xi_cur_ = 0;
    std::vector<double *> phi_ptrs_, w_mono_ptrs_;
    // per replica Anderson-mixing control (CpuAndersonMixing.cpp:76-161)
    int L_;
    std::vector<int> n_anderson_, head_;
    std::vector<double> mix_;
    std::vector<std::vector<std::vector<double>>> dot_rows_;
    // structure-function state: spectra of phi and the real auxiliary fields, sums
    DevBuf sf_spec_, sf_jobs_, sf_acc_, sf_coef_, sf_pairs_;
    int sf_np_ = 0;
    std::vector<int> sf_pairs_host_;
    // per-step graphs: update[parity of the noise buffers], search (loop + finish), and both in one
    bool step_graph_on_ = true;
    lfts_graph g_update_[2] = {nullptr, nullptr}, g_step_[2] = {nullptr, nullptr}, g_search_ = nullptr;
    long long k_update_ = 0, k_search_fixed_ = 0, k_body_ = 0;
    DevBuf fin_stats_, fin_scratch_;
    std::vector<double> poly_coef_;
};

}  // namespace lfts
