/*
 * lfts_b200.h -- C ABI of the B200 chain-propagator engine (liblfts_b200.so).
 *
 * Plain pointers and sizes only; every call returns 0 on success or a negative
 * status, with the message available from lfts_last_error().  Device buffers
 * are allocated by the caller (lfts_malloc or any CUDA allocator) and passed
 * in; no entry point below allocates except lfts_ctx_create / lfts_malloc.
 * All work is enqueued on the context's stream; nothing synchronises with the
 * host except lfts_synchronize and the blocking copies.
 *
 * Real-valued device arrays of a context use its precision (8 = double,
 * 4 = float): propagator slices, exp(-w ds) factor tables, Boltzmann bond
 * tables and spectra (complex = two reals).  Fields w, concentrations,
 * partition functions, stress and every reduction are always double.
 *
 * Grid layout: a 1D/2D/3D periodic box is handled as n0 x n1 x n2 (z fastest)
 * with leading extents of 1, M = n0*n1*n2 reals, Mc = n0*n1*(n2/2+1) complex,
 * exactly the real / conjugate-even layouts of the reference
 * (src/platforms/cpu/MklFFT3D.cpp:14-19, src/common/Pseudo.cpp:5-15).
 */
#ifndef LFTS_B200_H_
#define LFTS_B200_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lfts_ctx_s *lfts_ctx;

/* ---- context, memory, errors ------------------------------------------ */

/* Replaces CudaSolverPseudo's constructor (cuFFT plans, device tables;
 * src/platforms/cuda/CudaSolverPseudo.cu:6-147).  dim = 1..3, nx[0..dim-1];
 * precision = 8 (FP64) or 4 (FP32).  Prime factors of each extent must be
 * <= 64 and the x-plane must fit in shared memory (checked, error otherwise). */
int lfts_ctx_create(lfts_ctx *out, int device, int dim, const int *nx, int precision);
int lfts_ctx_destroy(lfts_ctx ctx);
/* Use an external CUDA stream (cudaStream_t as void*); NULL = the context's own. */
int lfts_ctx_set_stream(lfts_ctx ctx, void *stream);
void *lfts_ctx_stream(lfts_ctx ctx);
int lfts_ctx_info(lfts_ctx ctx, long long *M, long long *Mc, int *precision);
/* Number of kernels enqueued through this context so far (kernels replayed by
 * lfts_graph_launch are not counted; count them at capture). */
long long lfts_ctx_launches(lfts_ctx ctx);
/* Message of the last failing call on this thread. */
const char *lfts_last_error(void);

int lfts_malloc(lfts_ctx ctx, void **ptr, size_t bytes);
int lfts_free(lfts_ctx ctx, void *ptr);
/* Pinned host memory mapped into the device's address space (the same
 * address on both sides): kernels read and write it in place over the host
 * link.  The propagator slices of the reduce-memory mode live there.  Free
 * with lfts_free_host. */
int lfts_malloc_host(lfts_ctx ctx, void **ptr, size_t bytes);
int lfts_free_host(lfts_ctx ctx, void *ptr);
int lfts_memset_async(lfts_ctx ctx, void *ptr, int value, size_t bytes);
/* Blocking copies (used by the host wrapper for numpy inputs/outputs). */
int lfts_memcpy_h2d(lfts_ctx ctx, void *dst, const void *src, size_t bytes);
int lfts_memcpy_d2h(lfts_ctx ctx, void *dst, const void *src, size_t bytes);
int lfts_memcpy_d2d_async(lfts_ctx ctx, void *dst, const void *src, size_t bytes);
int lfts_synchronize(lfts_ctx ctx);
/* Status words read one step behind the GPU: lfts_status_post enqueues a copy
 * of one device int into pinned host slot `slot` (< LFTS_STATUS_SLOTS) and
 * records an event after it; lfts_status_wait waits for that event only and
 * returns the copied value (then checks the device error word).  The device
 * saddle loop polls its "any replica still active" word this way while the
 * next iteration is already queued.  No counterpart in the reference, whose
 * driver synchronises on every scalar it reads. */
#define LFTS_STATUS_SLOTS 4
int lfts_status_post(lfts_ctx ctx, const int *d_word, int slot);
int lfts_status_wait(lfts_ctx ctx, int slot, int *value);

/* CUDA graph capture of everything enqueued on the context stream between
 * begin and end (replaces the reference's per-step launches driven by OpenMP
 * host threads, CudaComputationContinuous.cu:273-505). */
typedef struct lfts_graph_s *lfts_graph;
int lfts_graph_begin(lfts_ctx ctx);
int lfts_graph_end(lfts_ctx ctx, lfts_graph *out);
int lfts_graph_launch(lfts_ctx ctx, lfts_graph g);
int lfts_graph_destroy(lfts_graph g);
/* A device-controlled loop inside a capture (no counterpart in the reference,
 * whose saddle loop runs on the host): between lfts_graph_begin and
 * lfts_graph_end, lfts_graph_while_begin appends a conditional WHILE node after
 * the work captured so far and sends the context stream's work into the node's
 * body until lfts_graph_while_end; work captured afterwards follows the loop.
 * The body repeats while the condition *handle is non-zero.  The condition is 1
 * when each graph launch reaches the node (the body runs at least once), and
 * device code in the body sets it (lfts_saddle_next).  Loops do not nest. */
int lfts_graph_while_begin(lfts_ctx ctx, unsigned long long *handle);
int lfts_graph_while_end(lfts_ctx ctx);

/* ---- tables ------------------------------------------------------------ */

/* Boltzmann bond factors exp(-b^2 |k|^2 ds / 6) and exp(-b^2 |k|^2 ds / 12),
 * each pre-divided by M (the inverse-FFT normalisation), precision of ctx.
 * Replaces Pseudo::get_boltz_bond (src/common/Pseudo.cpp:17-82) +
 * CudaSolverPseudo::update_laplacian_operator (CudaSolverPseudo.cu:211-253). */
int lfts_bond_tables(lfts_ctx ctx, double bond_length_sq, double ds, const double *lx,
                     void *bond_out, void *bond_half_out);
/* Weighted Fourier basis k_d^2 (x2 for 0 < kz < n2/2), 3 x Mc doubles.
 * Replaces Pseudo::get_weighted_fourier_basis (src/common/Pseudo.cpp:84-153). */
int lfts_fourier_basis(lfts_ctx ctx, const double *lx, double *basis_out);
/* fac[i] = exp(coef * w[i]) with w double (device), fac in ctx precision.
 * coef = -ds/4 (continuous: exp(-w ds/4), its square is exp(-w ds/2)) or
 * -ds (discrete).  Replaces update_dw (CudaSolverPseudo.cu:254-343). */
int lfts_field_factors(lfts_ctx ctx, const double *w, double coef, void *fac_out);
/* The same for `count` consecutive fields (count*M points, e.g. all replicas). */
int lfts_field_factors_batch(lfts_ctx ctx, const double *w, double coef, void *fac_out, int count);

/* ---- contour steps ------------------------------------------------------ */

/* One propagation job.  For step index s of a launch, the input slice is
 * in + s*in_stride and the output slice out + s*out_stride (elements of the
 * ctx precision), so one job array covers a whole schedule slot.
 * spec: scratch for two complex half spectra (2*Mc complex elements).
 * active/replica: when active != NULL the job is skipped unless
 * active[replica] != 0 (converged replicas of a batch stop without changing
 * the launch, so a captured graph stays valid). */
typedef struct {
    const void *in;
    long long in_stride;
    void *out;
    long long out_stride;
    const void *fac;        /* exp(-w ds/4) (continuous) or exp(-w ds) (discrete) */
    const void *bond;       /* bond table (lfts_bond_tables: bond_out) */
    const void *bond_half;  /* half-bond table */
    void *spec;
    const int *active;
    int replica;
    int pad;
} lfts_step_job;

/* 4th-order Richardson continuous step, q' = (4 q_{ds/2,ds/2} - q_ds)/3, for
 * njobs jobs (array in DEVICE memory) at step index s.  Replaces
 * CudaSolverPseudo::advance_propagator_continuous (CudaSolverPseudo.cu:345-412)
 * and CpuSolverPseudo::advance_propagator_continuous (CpuSolverPseudo.cpp:120-188). */
int lfts_step_continuous(lfts_ctx ctx, const lfts_step_job *jobs, int njobs, int s);
/* ---- real-space solver (continuous chains) ------------------------------- */

/* Tables of the real-space Crank-Nicolson step for one monomer type, on the
 * host, in DOUBLES: for each padded axis a = 0, 1, 2 (extent n_a; 1D and 2D
 * boxes pad to 3D with leading extents of 1, the box's axis d being padded
 * axis 3 - dim + d) seven rows of n_a values: the tridiagonal coefficients
 * l, d, h of src/common/FiniteDifference.cpp:6-101 (off-diagonals -b^2 ds /
 * (12 dx^2), diagonal 1 + b^2 ds / (6 dx^2); at a reflecting side the outer
 * off-diagonal folds into the diagonal, at an absorbing side it is dropped),
 * then the Thomas pivots p, the ratios c = h / p and, for a periodic axis,
 * the Sherman-Morrison vector v of CpuSolverReal.cpp:480-549, and 1 / p: seven rows
 * (tridiagonal_periodic, :509-549), in the reference's operation order; after the
 * three axes, the periodic denominators 1 + v[0] + l[0] v[n-1] (3 values) and
 * the periodic flags (3 values, 1.0 or 0.0).  bc: 2 * dim codes (0 periodic,
 * 1 reflecting, 2 absorbing), lower side first; dx: dim spacings.  Size in
 * doubles: lfts_realspace_table_size.  No counterpart in the reference (its
 * solver recomputes the pivots on every line). */
long long lfts_realspace_table_size(lfts_ctx ctx);
int lfts_realspace_tables(lfts_ctx ctx, double b2, double ds, int dim, const double *dx, const int *bc, double *tables_host);
/* One real-space Crank-Nicolson step of each job (CpuSolverReal.cpp:135-478,
 * CudaSolverReal.cu:371-407, continuous chains, FP64 contexts):
 * q_out = e ADI(e q_in), e = fac^2 = exp(-w ds/2) (fac holds exp(-w ds/4) as
 * for the pseudo-spectral step), ADI = the alternating-direction sweeps of
 * the reference (the first implicit in the box's first axis with the full
 * explicit operator on the right, then one implicit sweep per further axis).
 * jobs[j].bond: the job's device copy of its type's tables; jobs[j].spec:
 * 2 * M doubles of scratch; in/out/in_stride/out_stride/active as for
 * lfts_step_continuous (step index s).  dim: the box's dimension (1..3). */
int lfts_step_realspace(lfts_ctx ctx, const lfts_step_job *jobs, int njobs, int s, int dim);

/* Step autotuner (no counterpart in the reference, whose cuFFT plans are fixed):
 * times lfts_step_continuous for every implementation this grid supports
 * (register-resident line transforms at 64^3 / 96^3 with their x-pass CTA
 * residencies, the compile-time cubic kernels, the generic mixed-radix
 * kernels) on njobs synthetic jobs, reps timed calls each, and makes the
 * fastest the context's step implementation (continuous and discrete).  The
 * most specialised one stays unless another is more than 5 % faster.  It
 * allocates and frees its own buffers, synchronises, and must not run inside a
 * graph capture.  report (may be NULL) receives the timings and the choice. */
int lfts_autotune(lfts_ctx ctx, int njobs, int reps, char *report, size_t report_cap);
/* Name of the context's current step implementation ("register-64",
 * "register-64 xcap2", "register-96", "cubic", "generic"): the default chosen
 * at creation, or lfts_autotune's choice.  No counterpart in the reference. */
int lfts_step_impl(lfts_ctx ctx, char *name, size_t cap);
/* Make name the context's step implementation ("register-64", "register-96",
 * "cubic", "generic"); an error when the context has no such implementation.
 * Not during a graph capture.  No counterpart in the reference. */
int lfts_set_step_impl(lfts_ctx ctx, const char *name);
/* Discrete chain: out = [fac *] F^-1[ b * F[in] ] with b = bond (half=0) or
 * bond_half (half=1), multiplied by fac when with_fac=1.  (half=0, with_fac=1)
 * replaces advance_propagator_discrete (CudaSolverPseudo.cu:413-450);
 * (half=1, with_fac=0) replaces advance_propagator_discrete_half_bond_step
 * (CudaSolverPseudo.cu:451-476); (half=1, with_fac=1) is the junction start of
 * CpuComputationDiscrete.cpp:402-445 fused into one pass. */
int lfts_step_discrete(lfts_ctx ctx, const lfts_step_job *jobs, int njobs, int s, int half, int with_fac);

/* ---- junctions and initial slices --------------------------------------- */

/* out[i] = prod_d dep_d[i] (mode 0) or sum_d weight_d * dep_d[i] (mode 1),
 * optionally times fac[i] (continuous: fac^2 = exp(-w ds/2) is NOT applied;
 * the factor is used by discrete leaves).  dep pointers/weights in device
 * arrays.  Replaces the junction code of CudaComputationContinuous.cu:326-392
 * and CpuComputationDiscrete.cpp:298-445. */
typedef struct {
    void *out;
    const void *fac;      /* NULL or a factor table multiplied into out */
    int ndeps;            /* 0: out = 1 (times fac) */
    int mode;             /* 0 product, 1 weighted sum */
    int dep_offset;       /* first entry in dep_ptrs/dep_weights */
    int pad;
} lfts_junction_job;
int lfts_junctions(lfts_ctx ctx, const lfts_junction_job *jobs, int njobs, const void *const *dep_ptrs,
                   const double *dep_weights);

/* ---- reductions (FP64 accumulation) ------------------------------------- */

/* out[j] = scale_j * sum_i a_j[i] b_j[i] (/ w_j[i] if w_j != NULL).
 * Replaces ComputationBox::inner_product / inner_product_inverse_weight
 * (src/common/ComputationBox.cpp:273-286, CudaComputationBox.cu:56-117).
 * a, b, w in ctx precision; out (device) double. */
typedef struct {
    const void *a;
    const void *b;
    const void *w;
    double scale;
} lfts_dot_job;
int lfts_dots(lfts_ctx ctx, const lfts_dot_job *jobs, int njobs, double *out);

/* Block concentrations.  Continuous (model 0):
 *   phi[i] = norm * sum_{n=0}^{NR} c[coef_offset+n] q_left[(NL-n)*M+i] q_right[n*M+i]
 * Discrete (model 1):
 *   phi[i] = norm * sum_{n=1}^{NR} q_left[(NL-n+1)*M+i] q_right[n*M+i] / fac[i]
 * (norm divided by *q_div when q_div != NULL); phi (double).
 * Replaces calculate_phi_one_block + normalisation
 * (CpuComputationContinuous.cpp:371-465, CpuComputationDiscrete.cpp:584-679,
 * CudaComputationContinuous.cu:527-620). */
typedef struct {
    const void *q_left;
    const void *q_right;
    const void *fac;
    double *phi;
    double norm;
    const double *q_div;  /* NULL, or a device scalar the norm is divided by (Q_p) */
    int n_left;
    int n_right;
    int coef_offset;
    int pad;
} lfts_phi_job;
int lfts_phi_blocks(lfts_ctx ctx, int model, const lfts_phi_job *jobs, int njobs, const double *coefs);

/* Stress contributions: out[3*j+d] = weight_j * sum_k Re(F[q1_j](k) conj F[q2_j](k))
 * * basis_d(k) (* bond_j(k) if bond_j != NULL).  spec: scratch of 2*Mc complex
 * per job (jobs are processed in chunks of at most max_chunk).  Replaces
 * compute_single_segment_stress_{continuous,discrete}
 * (CudaSolverPseudo.cu:477-608, CpuSolverPseudo.cpp:250-356). */
typedef struct {
    const void *q1;
    const void *q2;
    const void *bond;   /* NULL (continuous) or bond / half-bond table already / M */
    double weight;
} lfts_stress_job;
int lfts_stress(lfts_ctx ctx, const lfts_stress_job *jobs, int njobs, const double *basis, void *spec,
                int max_chunk, double *out);

/* ---- Anderson mixing (FP64) --------------------------------------------- */

/* History vectors live in a ring of ring_len slots of `stride` doubles; the
 * i-th newest (i = 0 newest) is slot (head - i) mod ring_len.
 * dots[i] = sum_k d[k] * hist_i[k] for i < nhist.  Replaces the per-history
 * dot loop of CudaAndersonMixing.cu:245-250 (CpuAndersonMixing.cpp:100-108). */
int lfts_am_dots(lfts_ctx ctx, const double *d, const double *hist, long long stride, int nhist, long long n,
                 double *dots, int head, int ring_len);
/* w_new = w_0 + d_0 + sum_{i<nh} a[i] (w_{i+1} + d_{i+1} - w_0 - d_0), ring
 * indexing as above; a in DEVICE memory.  Replaces CudaAndersonMixing.cu:292-304
 * (CpuAndersonMixing.cpp:143-158). */
int lfts_am_update(lfts_ctx ctx, double *w_new, const double *w_hist, const double *d_hist, long long stride,
                   int nh, const double *a, long long n, int head, int ring_len);
/* w_new = w + mix * d (simple mixing, CpuAndersonMixing.cpp:110-121). */
int lfts_am_simple(lfts_ctx ctx, double *w_new, const double *w, const double *d, double mix, long long n);

/* ---- small helpers ------------------------------------------------------ */

/* out[i] = sum_k coefs[k] * srcs[k][i] (doubles; srcs/coefs are HOST arrays of
 * device pointers / values, any count).  Sums block concentrations into the
 * per-monomer totals (get_total_concentration, CpuComputationContinuous.cpp:466-520). */
int lfts_lincomb(lfts_ctx ctx, double *out, int nsrc, const double *const *srcs, const double *coefs, long long n);
/* Solvent: Q = dv_over_V * sum_i fac[i]^power (written to Q_out, device), then
 * phi[i] = vf * fac[i]^power / Q.  power 4 with fac = exp(-w ds/4) gives the
 * continuous solvent exp(-w ds)^... of CpuComputationContinuous.cpp:425-436;
 * power 1 with fac = exp(-w ds) the discrete one (CpuComputationDiscrete.cpp:441-452). */
int lfts_solvent(lfts_ctx ctx, const void *fac, int power, double vf, double dv_over_V, double *phi_out, double *Q_out);

/* ---- batched Langevin FTS (FP64; replicas r < R, fields w_aux[r][S][M]) --- */

#define LFTS_MAX_MONOMERS 8

/* w_mono[i][r][m] = sum_j A[i*S+j] w_aux[r][j][m]: auxiliary -> monomer fields
 * (SymmetricPolymerTheory.to_monomer_fields, examples/fts/lfts.py:181-182).
 * A: host S*S; w_mono: host array of S device pointers (each R x M). */
int lfts_lfts_monomer_fields(lfts_ctx ctx, int R, int S, long long M, const double *A, const double *w_aux,
                             double *const *w_mono);
/* out[r][c][m] = scale[c] * dH/dw_aux[idx[c]] (lfts.py:238-262): for i < S-1
 * 2 h2[i] w_i + h1[i] + sum_j A[j*S+i] phi_j, for i = S-1 sum_j phi_j - 1.
 * phi: host array of S device pointers (R x M each).  Replicas with
 * active[r] == 0 are skipped (active may be NULL). */
int lfts_lfts_field_deriv(lfts_ctx ctx, int R, int S, long long M, int nf, const int *idx, const double *scale,
                          const double *A, const double *h1, const double *h2, const double *w_aux,
                          const double *const *phi, double *out, const int *active);
/* Leimkuhler-Matthews update of the real fields idx[0..nreal-1]
 * (lfts.py:697-706): w += -dH/dw dt s + (xi_prev + xi_cur)/2 sqrt(s),
 * s = dt_scaling[c]; xi_* are [R][nreal][M]. */
int lfts_lfts_langevin(lfts_ctx ctx, int R, int S, long long M, int nreal, const int *idx, const double *A,
                       const double *h1, const double *h2, const double *const *phi, double dt,
                       const double *dt_scaling, double *w_aux, const double *xi_prev, const double *xi_cur,
                       const int *active);
/* Row moments: for row = r*rows_per_rep + c, x_row = x + r*rep_stride +
 * c*row_stride (M doubles): mean[row] = <x - center[row]>, msq[row] =
 * <(x - center[row])^2> (center may be NULL).  partials: >= 128*R*rows_per_rep
 * doubles of device scratch.  Gives the saddle-point error max_c std (lfts.py:833)
 * and the field averages of the Hamiltonian (lfts.py:219-235). */
int lfts_lfts_row_moments(lfts_ctx ctx, const double *x, int R, int rows_per_rep, long long M, long long row_stride,
                          long long rep_stride, const double *center, double *partials, double *mean, double *msq);
/* w_aux[r][field] -= mean[r] (zero-mean pressure field, lfts.py:866). */
int lfts_lfts_subtract_mean(lfts_ctx ctx, double *w_aux, int R, int S, int field, long long M, const double *mean,
                            const int *active);

/* Batched Anderson mixing: per replica a ring of L slots of n doubles
 * (hist + (r*L + slot)*n); i-th newest slot = (head[r] - i) mod L.
 * insert: where flag[r], copy w_cur/d_cur (replica stride *_stride) into slot head[r].
 * dots:   dots[r*L + i] = d_0 . d_i for i < ndots[r] (partials: >= 64*R*L doubles).
 * update: mode[r] 0 skip, 1 simple mixing w_cur + mix[r] d_cur, 2 Anderson
 *         w_0 + d_0 + sum_{h<nh[r]} a[r*L+h] (w_{h+1} + d_{h+1} - w_0 - d_0).
 * All control arrays are device arrays.  Replaces CpuAndersonMixing.cpp:76-161
 * for a batch of independent mixers. */
int lfts_am_batch_insert(lfts_ctx ctx, int R, long long n, int L, const int *head, const int *flag, const double *w_cur,
                         long long w_stride, const double *d_cur, long long d_stride, double *w_hist, double *d_hist);
int lfts_am_batch_dots(lfts_ctx ctx, int R, long long n, int L, const int *head, const int *ndots, const double *d_hist,
                       double *partials, double *dots);
int lfts_am_batch_update(lfts_ctx ctx, int R, long long n, int L, const int *head, const int *mode, const int *nh,
                         const double *mix, const double *a, const double *w_cur, long long w_stride, const double *d_cur,
                         long long d_stride, const double *w_hist, const double *d_hist, double *w_out, long long out_stride);

/* Device control of one saddle-point iteration of every replica: the host
 * loop of examples/fts/lfts.py:807-868 with the Anderson-mixing bookkeeping of
 * src/platforms/cpu/CpuAndersonMixing.cpp:86-121, per replica, without a host
 * round trip.  For each replica r with active[r]:
 *   e = max_c sqrt(max(var[r*I+c], 0)) / scale[c] (a NaN wins), err_old = err,
 *   err = e, iter = it; e < tolerance ends the replica (active = 0); otherwise
 *   n_anderson advances (once e < am_start_error or already >= 0, capped at
 *   am_max_hist), head_raw advances in the ring of L = am_max_hist + 1 slots
 *   with flag = 1, ndots = n_anderson + 1, and mode = 1 (simple mixing, mix
 *   x0.7 floored at am_mix_min when the error grew, else x1.01) while
 *   n_anderson <= 0, else mode = 2 with nh = n_anderson.
 * Every replica gets head = max(head_raw, 0), and flag/ndots/mode/nh = 0 unless
 * set above; *any_active (reset here) becomes 1 if a replica stays active.
 * All pointers in st are device pointers; scale is host (I values). */
typedef struct {
    int *active, *n_anderson, *head_raw, *iter, *head, *flag, *ndots, *mode, *nh, *any_active;
    double *err, *err_old, *mix;
    int *loop_iter;  /* device iteration counter of a graph loop; read when it <= 0 (may be NULL otherwise) */
} lfts_saddle_state;
int lfts_saddle_control(lfts_ctx ctx, int R, int I, int it, const double *var, const double *scale, double tolerance,
                        double am_start_error, int am_max_hist, double am_mix_min, const lfts_saddle_state *st);
/* The saddle-point loop of one Langevin step as device work (for one graph per
 * step; no counterpart in the reference, whose loop runs on the host):
 * lfts_saddle_begin resets every replica to the start of a search (active,
 * no Anderson history, err = err_old = 1e20, iter = 0, mix = mix_init) and
 * sets *st->loop_iter = 1.  lfts_saddle_next, the last work of the loop body,
 * sets the WHILE condition handle to (*any_active && *loop_iter < max_iter)
 * and advances *loop_iter, so a loop runs at most max_iter times. */
int lfts_saddle_begin(lfts_ctx ctx, int R, double mix_init, const lfts_saddle_state *st);
int lfts_saddle_next(lfts_ctx ctx, unsigned long long handle, const lfts_saddle_state *st, int max_iter);
/* After the saddle-point loop of a step, per replica r (examples/fts/lfts.py:
 * 219-235, 711-730, 866): failed = isnan(err) || err >= tolerance; the
 * Hamiltonian from the field moments mean/msq ([R][S], of the fields before the
 * pressure shift) and Q ([R][P]):
 *   H = (sum_p -poly[p] ln Q[r][p]) + (-mean[S-1] + sum_{i<S-1} h2[i] msq[i]
 *       + h1[i] mean[i]) + h_const,   poly[p] = volume fraction / alpha;
 * the pressure field w_aux[r][S-1] loses its mean; when restore != 0 a failed
 * replica gets w_save and phi_save ([R][S][M]) back into w_aux and phi[s][r];
 * active[r] = 1.  stats (device doubles) receives, for a host read in one copy:
 *   [iter (R) | err (R) | H (R) | failed (R) | Q (R*P) | mean (R*S) | msq (R*S)].
 * S <= LFTS_MAX_MONOMERS, P <= 8. */
int lfts_lfts_step_finish(lfts_ctx ctx, int R, int S, int P, long long M, const lfts_saddle_state *st, double tolerance,
                          const double *mean, const double *msq, const double *Q, const double *h1, const double *h2,
                          double h_const, const double *poly, int restore, double *w_aux, const double *w_save,
                          double *const *phi, const double *phi_save, double *scratch, double *stats);
/* Anderson-mixing coefficients of every replica on the device
 * (src/common/AndersonMixing.cpp:19-47 and CpuAndersonMixing.cpp:122-146):
 * where ndots[r] > 0 the new dot row dots[r*L + i] (i < ndots[r]) enters the
 * ring dot_ring[r][head[r]][0..L); where mode[r] == 2, with rows k = (head - k)
 * mod L, U_ij = r0[0] - r0[i+1] - r0[j+1] + r_{min(i,j)+1}[|i-j|] and
 * V_i = r0[0] - r0[i+1] are solved by Gaussian elimination without pivoting, in
 * the reference's operation order with every product and sum rounded on its
 * own, into a[r*L + i], i < nh[r].  dot_ring: R*L*L device doubles.
 * Holds at most LFTS_AM_SOLVE_MAX_HIST history vectors (L <= 33). */
#define LFTS_AM_SOLVE_MAX_HIST 32
int lfts_am_batch_solve(lfts_ctx ctx, int R, int L, const int *head, const int *ndots, const int *mode, const int *nh,
                        const double *dots, double *dot_ring, double *a);

/* PCG64 streams on the device: the generator of numpy's PCG64 (128-bit LCG
 * state = state * 0x2360ED051FC65DA44385DF649FCCF645 + inc, then the XSL-RR
 * output of the new state), one per stream, states[4*s..4*s+3] = state hi,
 * state lo, inc hi, inc lo (device uint64; take them from
 * numpy's bit_generator.state).  Replaces the host draws of lfts.py:700
 * (numpy Generator.normal) for the batched driver.
 * raw:    out[s][i], i < n = the next n raw outputs of stream s (numpy's
 *         PCG64.random_raw(n), bit for bit).
 * normal: out[s][i] = sigma * N(0, 1) by Box-Muller on pairs of 53-bit
 *         uniforms from consecutive raw outputs (2*ceil(n/2) raw outputs used).
 *         The normal transform is this library's, not numpy's ziggurat: the
 *         normals are N(0, 1) but not numpy's sequence.
 * Both advance every state by the raw outputs used, so calls continue the
 * streams. */
int lfts_pcg64_raw(lfts_ctx ctx, unsigned long long *states, int nstreams, long long n, unsigned long long *out);
int lfts_pcg64_normal(lfts_ctx ctx, unsigned long long *states, int nstreams, long long n, double sigma, double *out);

/* ---- learned saddle-point start: U-Net convolution ---------------------- */

/* Periodic 3D convolution of channels-last BF16 activations on the tensor
 * cores (tcgen05 implicit GEMM, FP32 accumulation in tensor memory):
 *   out[p][co] = act(bias[co] + sum_{tap, ci} w[tap][co][ci] in[(p + tap) mod box][ci])
 * in: [B][D][H][W][cin], out: [B][D][H][W][cout] (BF16, 16-byte aligned),
 * wpk: packed weights [taps][cin/8][cout][8] BF16 (tap = 9 kz + 3 ky + kx,
 * offset (kz-1, ky-1, kx-1); taps = 27 for 3x3x3, 1 for 1x1x1), bias: cout
 * FP32 (device).  cin, cout: multiples of 16, cin <= LFTS_CONV_MAX_CIN,
 * cout <= LFTS_CONV_MAX_COUT, and the two shared stages, 32 cin (128 + cout)
 * bytes, within 200 KB; act = ReLU when relu != 0.  stream: cudaStream_t.
 * Kernel choice: 3x3x3 with H % 16 == 0 and W % 8 == 0 stages each tile's halo
 * in shared memory (from 48 input channels by slices of 16 channels with all
 * taps' weights, else once with a ring of per-tap weights); other grids and
 * 1x1x1 gather the shifted rows per tap.  The results agree to FP32
 * accumulation order.  LFTS_CONV_KSLICE, LFTS_CONV_KSLICE_TZ,
 * LFTS_CONV_KSLICE_NS and LFTS_CONV_TZ (environment) override the choice, for
 * tests and measurement.
 * No counterpart in the reference (it has no learned component). */
#define LFTS_CONV_MAX_CIN 160
#define LFTS_CONV_MAX_COUT 256
int lfts_conv3d_bf16(void *stream, const void *in, const void *wpk, const float *bias, void *out, int B, int D, int H, int W,
                     int cin, int cout, int taps, int relu);
/* Its weight gradient, also on the tensor cores:
 *   dw[tap][co][ci] += sum_p gy[p][co] x[(p + tap) mod box][ci]
 * x: [B][D][H][W][cin], gy: [B][D][H][W][cout] BF16 channels-last; dw: FP32
 * [taps][cout][ci], accumulated (zero it first); cout <= 128, at most 65535
 * chunks of 32-256 stages of 64 positions.  The input gradient is
 * lfts_conv3d_bf16 of gy with the weights transposed and the taps mirrored.
 * LFTS_CONV_WGRAD_RING, LFTS_CONV_WGRAD_STAGES and LFTS_CONV_WGRAD_GATHER
 * (environment) override the ring depth, the stages per CTA and the x staging,
 * for tests and measurement. */
int lfts_conv3d_wgrad_bf16(void *stream, const void *x, const void *gy, float *dw, int B, int D, int H, int W, int cin,
                           int cout, int taps);

/* AdamW step of the U-Net's training on n FP32 parameters (device p, g, m,
 * v on the given cudaStream_t), in torch.optim.AdamW's order: p *= 1 - lr wd;
 * m += (1 - b1)(g - m); v = b2 v + (1 - b2) g^2; p -= (lr / (1 - b1^step)) m /
 * (sqrt(v) / sqrt(1 - b2^step) + eps).  step >= 1 counts the calls.  No
 * counterpart in the reference (it has no learned component). */
int lfts_adamw_f32(void *stream, float *p, const float *g, float *m, float *v, long long n, double lr, double b1, double b2,
                   double eps, double weight_decay, int step);

/* Backward of the ReLU after a U-Net convolution (training): g = gy where
 * y > 0, else 0, for every one of the cpad channels of npos positions (BF16,
 * channels last, 16-byte aligned), and db[c] += sum over positions of g[p][c]
 * for c < co (FP32, on the device; the caller zeroes it).  cpad a multiple of
 * 8 up to 256.  The reference has no learned start; this replaces torch's
 * autograd of the ReLU and of the bias sum in the U-Net's training. */
int lfts_relu_grad_bf16(void *stream, const void *gy, const void *y, void *g, float *db, long long npos, int cpad, int co);

/* Adam field update of the SCFT driver (examples/scft/scft.py:42-54), on n
 * doubles: m = b1 m + (1-b1) d; v = b2 v + (1-b2) d^2;
 * w_new = w + lr (m / (1 - b1^count)) / (sqrt(v / (1 - b2^count)) + eps).
 * m and v (device) carry the moments between calls; count >= 1. */
int lfts_adam_update(lfts_ctx ctx, double *w_new, const double *w, const double *d, double *m, double *v, long long n,
                     double lr, double b1, double b2, double eps, int count);

/* ---- structure function (recording of the L-FTS driver) ------------------ */

/* Forward real-to-complex 3D FFT of double fields, unnormalised, in the
 * numpy.fft.rfftn layout [nx][ny][nz/2+1]: jobs[j].in (M doubles) ->
 * jobs[j].spec (Mc complex doubles); in_stride, out, fac and the bond tables
 * are ignored, active/replica mask jobs as in the step calls.  Double-precision
 * contexts only.  Replaces the host np.fft.rfftn of the structure-function
 * recording (examples/fts/lfts.py:757-762). */
int lfts_fft_forward(lfts_ctx ctx, const lfts_step_job *jobs, int njobs);

/* Structure-function accumulation (examples/fts/lfts.py:754-767), for each
 * replica r and monomer pair p = (a, b) = (pairs[2p], pairs[2p+1]):
 *   sf[r][p][k] += mu_a(k) * conj(phi_b(k) * inv_m),
 *   mu_a(k) = sum_{q < I} spec[r][S + q][k] * coef[q*S + a],
 * where spec[r][s] (s < S) is the transform of phi_s and spec[r][S + q] that of
 * the q-th real auxiliary field (Mc complex doubles each, replica stride
 * (S + I)*Mc).  coef (device, I x S) = A_inv[q][a] / eigenvalue[q] / M;
 * pairs: device ints; sf: device complex doubles [R][npairs][Mc]. */
int lfts_sf_accumulate(lfts_ctx ctx, int R, int S, int I, const void *spec, const double *coef, double inv_m, int npairs,
                       const int *pairs, void *sf);

/* ---- allocation-free inner products (no reference counterpart) ----------
 * lfts_dots_static computes what lfts_dots computes,
 *   out[j] = scale_j * sum_{i<M} a_j[i] b_j[i] (/ w_j[i] if w_j != NULL),
 * without a context and without allocating any device memory.  The reference
 * has no such entry point: its inner products run through a computation box
 * that owns allocated scratch.  It serves hosts that hold no lfts context and
 * may not let a library allocate, e.g. a runtime that hands out all device
 * memory from its own fixed pool.
 * precision: 8 (a, b, w double) or 4 (float).  M > 0.  jobs: device array of
 * njobs entries; out: device array of njobs doubles; stream: a cudaStream_t
 * (NULL = the default stream).  Everything is enqueued on that stream.
 * Scratch: one file-scope device array of LFTS_DOTS_STATIC_MAX_JOBS x 128
 * doubles (256 KiB) per device.  njobs above LFTS_DOTS_STATIC_MAX_JOBS is
 * rejected with an error.  Every call on a device shares that array, so calls
 * that overlap in time (two streams, or two host threads, on one device) race
 * and must be serialised by the caller.  Each call writes every scratch entry
 * it reads, so nothing needs clearing between calls.
 * The first call in each device context looks up the array's address
 * (cudaGetSymbolAddress) with that device current and caches it with the
 * context's id; make that first call before any stream capture.  A new
 * context on the device (after cudaDeviceReset) gets a fresh lookup on its
 * first call, which must likewise precede any capture. */
#define LFTS_DOTS_STATIC_MAX_JOBS 256
int lfts_dots_static(int precision, long long M, const lfts_dot_job *jobs, int njobs, double *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif
