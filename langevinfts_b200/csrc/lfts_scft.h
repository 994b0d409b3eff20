// Device-resident SCFT iteration: the fields, residuals and optimizer state of
// examples/scft/scft.py:617-736 stay in HBM; per iteration only scalars cross
// to the host (partition functions, error sums, stress, the box).
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "lfts_computation.h"

namespace lfts {

struct ScftConfig {
    std::vector<std::string> monomer_types;  // sorted; order of the field rows
    std::vector<double> chi;                 // S x S, matrix_chi (scft.py:71-81)
    std::vector<double> P;                   // S x S, matrix_p (projection, scft.py:65)
    std::vector<double> A_inv;               // S x S, w_aux = A_inv w (energy moments)
    bool box_altering = false;
    double scale_stress = 1.0;
    std::string optimizer = "am";            // "am" or "adam"
    int am_max_hist = 20;
    double am_start_error = 1e-1, am_mix_min = 1e-1, am_mix_init = 1e-1;
    double adam_lr = 1e-2, adam_gamma = 1.0;
};

struct ScftStats {
    double error_level = 0.0;             // scft.py:680-691 (+ |stress| when the box moves)
    double mass_error = 0.0;              // integral(phi_total - 1) / V
    std::vector<double> partitions;       // Q_p
    std::vector<double> stress;           // dim values (box_altering)
    std::vector<double> lx;               // box at this iteration
    std::vector<double> aux_mean, aux_msq;  // <w_aux_i>, <w_aux_i^2> (the Hamiltonian, scft.py:206-222)
};

class DeviceScft {
   public:
    DeviceScft(ComputationBox *cb, Molecules *mol, PropagatorAnalyzer *pa, int precision, int device,
               const ScftConfig &cfg);
    ~DeviceScft();
    int n_grid() const { return (int)M_; }
    int n_types() const { return S_; }
    // host [S][M] monomer fields; each row's mean is removed (scft.py:643-645)
    void set_fields(const double *w);
    void get_fields(double *w) const;
    void get_concentrations(double *phi) const;  // host [S][M]
    // statistics, residual and error level at the current fields
    ScftStats evaluate();
    // one optimizer step from the last evaluate(): new fields (and box), then
    // the mean shift of every field row (scft.py:697-733)
    void update();
    void reset();  // optimizer state back to its start (reset_count)

   private:
    void row_means(const double *rows, double *d_out);  // S means of rows at stride M

    ScftConfig cfg_;
    ComputationBox *cb_;
    Molecules *mol_;
    int S_, dim_;
    long long M_, n_var_;
    std::unique_ptr<GpuComputation> comp_;
    lfts_ctx ctx_;
    std::unique_ptr<GpuAndersonMixing> am_;
    DevBuf cur_, diff_, new_, waux_, ones_, scal_, jobs_, m_, v_;
    std::vector<double *> phi_, wdev_;
    int adam_count_ = 1;
    double err_ = 1e20, err_old_ = 1e20;
    std::vector<double> stress_;
    bool evaluated_ = false;
};

}  // namespace lfts
