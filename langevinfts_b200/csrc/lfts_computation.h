// GPU propagator computation and Anderson mixing behind the langevinfts API.
//
// Same surface as the reference's PropagatorComputation / AndersonMixing
// (src/common/PropagatorComputation.h:21-75, AndersonMixing.h:13-29); all
// arithmetic runs in liblfts_b200 through the C ABI (include/lfts_b200.h).
// Host code here only plans launches (which slices feed which kernel) and
// moves numpy inputs/outputs across the host<->device boundary.
#pragma once

#include <array>
#include <map>
#include <string>
#include <vector>

#include "lfts_b200.h"
#include "lfts_host.h"

namespace lfts {

void check_rc(int rc);

// One device allocation owned by a context.
class DevBuf {
   public:
    DevBuf() = default;
    DevBuf(lfts_ctx c, size_t bytes) { alloc(c, bytes); }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : ctx_(o.ctx_), p_(o.p_), n_(o.n_), host_(o.host_) { o.p_ = nullptr; }
    void alloc(lfts_ctx c, size_t bytes);
    // pinned host memory mapped into the device (lfts_malloc_host)
    void alloc_host(lfts_ctx c, size_t bytes);
    void release();
    void *get() const { return p_; }
    size_t size() const { return n_; }
    template <typename T> T *as() const { return (T *)p_; }

   private:
    lfts_ctx ctx_ = nullptr;
    void *p_ = nullptr;
    size_t n_ = 0;
    bool host_ = false;
};

class GpuComputation {
   public:
    // n_replicas independent systems of the same molecules and box advance in
    // the same launches (replica r of every device array at offset r * size).
    // method: "pseudospectral" (periodic boxes) or "realspace" (the
    // Crank-Nicolson step of lfts_step_realspace, continuous chains, FP64;
    // any boundary conditions, no stress).  reduce_memory: every propagator
    // slice in pinned host memory mapped into the device, read and written in
    // place by the same kernels (the reference's memory-saving mode keeps its
    // slices in pinned host memory too); device memory then holds the fields,
    // tables, concentrations and step scratch only.
    GpuComputation(ComputationBox *cb, Molecules *molecules, PropagatorAnalyzer *analyzer, int precision, int device,
                   int n_replicas = 1, const std::string &method = "pseudospectral", bool reduce_memory = false);
    ~GpuComputation();

    int get_n_grid() const { return cb_->get_n_grid(); }
    int get_n_blocks(int p) { return mol_->get_polymer(p).get_n_blocks(); }
    int get_precision() const { return prec_; }
    void update_laplacian_operator();
    void compute_propagators(const std::map<std::string, const double *> &w,
                             const std::map<std::string, const double *> &q_init = {});
    void compute_concentrations();
    void compute_statistics(const std::map<std::string, const double *> &w,
                            const std::map<std::string, const double *> &q_init = {});
    void compute_stress();
    double get_total_partition(int p);
    void get_chain_propagator(double *out, int p, int v, int u, int n);
    void get_total_concentration(const std::string &monomer_type, double *phi);
    void get_total_concentration(int p, const std::string &monomer_type, double *phi);
    void get_total_concentration_gce(double fugacity, int p, const std::string &monomer_type, double *phi);
    void get_block_concentration(int p, double *phi);
    double get_solvent_partition(int s);
    void get_solvent_concentration(int s, double *phi);
    std::vector<double> get_stress();
    std::vector<double> get_stress_gce(const std::vector<double> &fugacities);
    bool check_total_partition();

    lfts_ctx context() const { return ctx_; }
    const Scheduler &scheduler() const { return *sched_; }

    // ---- batched (device-resident) interface, all replicas at once
    int n_replicas() const { return R_; }
    long long n_grid() const { return M_; }
    // fields w of a monomer type, R x M doubles on the device (filled by the caller)
    double *w_device(const std::string &type);
    // total concentration of a monomer type, R x M doubles on the device
    double *phi_type_device(const std::string &type);
    // single-chain partition functions, R x P doubles on the device
    double *partition_device();
    // per-replica flags: replicas with 0 are skipped by the step kernels
    int *active_device() { return active_.as<int>(); }
    // Enqueue field factors, propagators, partition functions, block and
    // per-type concentrations for every active replica (graph-capturable).
    void enqueue_statistics(bool use_graph = true);
    // kernels run by an outside graph replay, for kernel_launches()
    void count_replayed(long long n) { graph_kernels_replayed_ += n; }
    // Copy the partition functions of every replica to the host.
    std::vector<double> partitions_host();
    // kernels launched so far: direct launches + kernels replayed in graphs
    long long kernel_launches() const { return lfts_ctx_launches(ctx_) + graph_kernels_replayed_; }
    // largest step launch of the schedule (jobs), the batch lfts_autotune times
    int max_jobs_per_launch() const { return max_jobs_; }
    // time the step implementations at that batch and keep the fastest (before
    // the first captured graph); returns lfts_autotune's report
    std::string autotune(int reps = 5);

   private:
    struct KeyStore {
        DevBuf q;                      // slices 0..max_n_segment
        std::map<int, DevBuf> half;    // discrete: q(n + 1/2) at junction ends, q_junction at 0
    };
    struct TypeStore {
        DevBuf w, fac, bond, bond_half;
    };
    struct Launch {
        int kind;     // 0 junctions, 1 continuous steps, 2 discrete steps, 3 d2d copy
        size_t jobs;  // byte offset into the job arena
        int njobs;
        int nsteps;
        int half, with_fac;
        size_t deps, wts;  // junction dependency arrays (byte offsets)
        void *dst;
        const void *src;
        size_t bytes;
    };

    void *slice(const std::string &key, int n, int r = 0) const;
    void *half_slice(const std::string &key, int n, int r = 0) const;
    void build_plan();
    void build_stress_jobs();
    void build_dot_jobs();
    void build_phi_jobs();
    void enqueue_propagation();
    void enqueue_concentrations();
    void sync_partitions();

    bool realspace_ = false;
    ComputationBox *cb_;
    Molecules *mol_;
    PropagatorAnalyzer *pa_;
    int prec_ = 8;
    int R_ = 1;
    size_t esz_ = 8;
    bool continuous_ = true;
    lfts_ctx ctx_ = nullptr;
    long long M_ = 0, Mc_ = 0;
    Scheduler *sched_ = nullptr;

    std::map<std::string, KeyStore> keys_;
    std::map<std::string, TypeStore> types_;
    std::map<std::string, DevBuf> q_init_;
    std::map<BlockKey, DevBuf> phi_block_;
    std::map<std::string, DevBuf> phi_type_;
    std::vector<DevBuf> phi_solvent_;
    int max_jobs_ = 1;
    DevBuf active_, phi_tmp_, spec_, arena_, dev_scalars_, basis_, phi_jobs_, coefs_, stress_jobs_, stress_out_, stress_spec_;
    std::vector<Launch> plan_;
    size_t phi_jobs_cont_ = 0, phi_jobs_disc_ = 0, coef_off_ = 0;
    int n_phi_cont_ = 0, n_phi_disc_ = 0;
    std::vector<std::pair<BlockKey, int>> zero_blocks_;
    std::vector<unsigned char> arena_host_;
    lfts_graph graph_ = nullptr, stats_graph_ = nullptr;
    bool use_graph_ = true;
    long long stats_graph_kernels_ = 0, graph_kernels_replayed_ = 0;

    // single-chain partition: (polymer, dot job index)
    std::vector<int> partition_polymer_;
    size_t dot_jobs_ = 0;
    int n_dot_jobs_ = 0;
    std::vector<double> q_poly_, q_solvent_;
    std::vector<std::array<double, 3>> dq_dl_;
    // stress job bookkeeping: job -> block index (map order)
    std::vector<int> stress_block_;
    std::vector<BlockKey> block_order_;
    int n_stress_jobs_ = 0, stress_chunk_ = 1;
    bool have_propagators_ = false;
};

class GpuAndersonMixing {
   public:
    GpuAndersonMixing(int n_var, int max_hist, double start_error, double mix_min, double mix_init, int device);
    ~GpuAndersonMixing();
    void reset_count();
    int get_n_var() const { return n_var_; }
    void calculate_new_fields(double *w_new, const double *w_current, const double *w_deriv, double old_error_level,
                              double error_level);
    // Same with device arrays of n_var doubles (work on other streams that
    // produced w_current / w_deriv must be complete); returns with w_new written.
    void calculate_new_fields_device(double *w_new, const double *w_current, const double *w_deriv,
                                     double old_error_level, double error_level);

   private:
    int n_var_, max_hist_, n_anderson_ = -1;
    double start_error_, mix_min_, mix_, mix_init_;
    lfts_ctx ctx_ = nullptr;
    DevBuf w_hist_, d_hist_, w_new_, stage_w_, stage_d_, dots_, a_;
    int ring_len_, head_ = -1, n_items_ = 0;
    // dots ring: row i (0 = newest) holds d_i . d_{i+j} for j <= n_anderson at insertion
    std::vector<std::vector<double>> dot_rows_;
    void step(double *w_new, const double *w_cur, const double *w_deriv, double old_err, double err, bool device);
};

}  // namespace lfts
