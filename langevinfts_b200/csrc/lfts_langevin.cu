// Batched Langevin field-theoretic simulation kernels (FP64), all replicas of
// a batch per launch.  Field layout: w_aux[r][S][M] (auxiliary fields),
// per-monomer arrays [r][M].  Restates the driver arithmetic of the reference's
// examples/fts/lfts.py (func derivatives :238-262, Leimkuhler-Matthews update
// :697-706, saddle error :833-834, zero-mean pressure :866, Hamiltonian
// :219-235) and the Anderson mixing of src/platforms/cpu/CpuAndersonMixing.cpp.
#include <cuda_runtime.h>

#include <string>

#include "../../include/lfts_b200.h"

namespace {

constexpr int NT = 256;
constexpr int NW = NT / 32;

}  // namespace
// error channel shared with the engine (lfts_last_error)
int lfts_internal_fail(const std::string &msg);
void lfts_internal_count(lfts_ctx c, int n);
namespace {
int lfail(const std::string &m) { return lfts_internal_fail(m); }
#define LCK(call)                                                                                     \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return lfail(std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

__device__ __forceinline__ double bsum(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    v = 0;
    if (w == 0) {
        v = lane < NW ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

struct DerivArgs {
    int S, nf;
    int idx[LFTS_MAX_MONOMERS];
    double scale[LFTS_MAX_MONOMERS];
    double A[LFTS_MAX_MONOMERS * LFTS_MAX_MONOMERS];
    double h1[LFTS_MAX_MONOMERS], h2[LFTS_MAX_MONOMERS];
    const double *phi[LFTS_MAX_MONOMERS];
};

// g_i = 2 h2_i w_i + h1_i + sum_j A[j][i] phi_j  (i < S-1);  sum_j phi_j - 1 (i = S-1)
__device__ __forceinline__ double deriv(const DerivArgs &a, int i, const double *w_r, long long M, long long m,
                                        long long off) {
    double g;
    if (i != a.S - 1) {
        g = 2.0 * a.h2[i] * w_r[(long long)i * M + m] + a.h1[i];
        for (int j = 0; j < a.S; j++) g += a.A[j * a.S + i] * a.phi[j][off];
    } else {
        g = -1.0;
        for (int j = 0; j < a.S; j++) g += a.phi[j][off];
    }
    return g;
}

__global__ void k_deriv(DerivArgs a, const double *__restrict__ w_aux, long long M, int R, double *__restrict__ out,
                        const int *__restrict__ active) {
    const int r = blockIdx.y;
    if (active && !active[r]) return;
    const double *w_r = w_aux + (long long)r * a.S * M;
    for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < M; m += (long long)gridDim.x * NT) {
        const long long off = (long long)r * M + m;
        for (int c = 0; c < a.nf; c++) out[((long long)r * a.nf + c) * M + m] = a.scale[c] * deriv(a, a.idx[c], w_r, M, m, off);
    }
}

// Leimkuhler-Matthews: w_i += -g_i dt s_i + (xi_prev + xi_cur)/2 sqrt(s_i) for the real fields
struct LangevinArgs {
    DerivArgs d;
    double dt;
    double s[LFTS_MAX_MONOMERS];
    double sqrt_s[LFTS_MAX_MONOMERS];
};
__global__ void k_langevin(LangevinArgs a, double *__restrict__ w_aux, long long M, const double *__restrict__ xi_prev,
                           const double *__restrict__ xi_cur, const int *__restrict__ active) {
    const int r = blockIdx.y;
    if (active && !active[r]) return;
    double *w_r = w_aux + (long long)r * a.d.S * M;
    for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < M; m += (long long)gridDim.x * NT) {
        const long long off = (long long)r * M + m;
        double g[LFTS_MAX_MONOMERS];
        for (int c = 0; c < a.d.nf; c++) g[c] = deriv(a.d, a.d.idx[c], w_r, M, m, off);
        for (int c = 0; c < a.d.nf; c++) {
            const long long n = ((long long)r * a.d.nf + c) * M + m;
            w_r[(long long)a.d.idx[c] * M + m] += -g[c] * a.dt * a.s[c] + 0.5 * (xi_prev[n] + xi_cur[n]) * a.sqrt_s[c];
        }
    }
}

struct MonoArgs {
    int S;
    double A[LFTS_MAX_MONOMERS * LFTS_MAX_MONOMERS];
    double *w[LFTS_MAX_MONOMERS];
};
__global__ void k_monomer_fields(MonoArgs a, const double *__restrict__ w_aux, long long M, int R) {
    const long long n = (long long)R * M;
    for (long long t = blockIdx.x * (long long)NT + threadIdx.x; t < n; t += (long long)gridDim.x * NT) {
        const long long r = t / M, m = t - r * M;
        const double *w_r = w_aux + r * a.S * M;
        for (int i = 0; i < a.S; i++) {
            double v = 0.0;
            for (int j = 0; j < a.S; j++) v += a.A[i * a.S + j] * w_r[(long long)j * M + m];
            a.w[i][t] = v;
        }
    }
}

// per (row) sums of x and x^2 -> partials; rows of length M
__global__ void k_row_sums(const double *__restrict__ x, long long M, long long row_stride, int rows_per_rep,
                           long long rep_stride, const double *__restrict__ center, double *partials) {
    __shared__ double sh[NW];
    const int row = blockIdx.y;
    const int r = row / rows_per_rep, c = row % rows_per_rep;
    const double *p = x + (long long)r * rep_stride + (long long)c * row_stride;
    const double mu = center ? center[row] : 0.0;
    double s1 = 0.0, s2 = 0.0;
    for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < M; m += (long long)gridDim.x * NT) {
        const double v = p[m] - mu;
        s1 += v;
        s2 += v * v;
    }
    s1 = bsum(s1, sh);
    s2 = bsum(s2, sh);
    if (threadIdx.x == 0) {
        partials[((long long)row * gridDim.x + blockIdx.x) * 2] = s1;
        partials[((long long)row * gridDim.x + blockIdx.x) * 2 + 1] = s2;
    }
}
__global__ void k_row_finish(const double *__restrict__ partials, int nparts, long long M, double *mean, double *msq) {
    __shared__ double sh[NW];
    const int row = blockIdx.x;
    double s1 = 0.0, s2 = 0.0;
    for (int p = threadIdx.x; p < nparts; p += NT) {
        s1 += partials[((long long)row * nparts + p) * 2];
        s2 += partials[((long long)row * nparts + p) * 2 + 1];
    }
    s1 = bsum(s1, sh);
    s2 = bsum(s2, sh);
    if (threadIdx.x == 0) {
        mean[row] = s1 / (double)M;
        msq[row] = s2 / (double)M;
    }
}

__global__ void k_subtract_mean(double *__restrict__ w_aux, int S, int field, long long M, const double *__restrict__ mean,
                                const int *__restrict__ active) {
    const int r = blockIdx.y;
    if (active && !active[r]) return;
    double *p = w_aux + ((long long)r * S + field) * M;
    const double mu = mean[r];
    for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < M; m += (long long)gridDim.x * NT) p[m] -= mu;
}

// ---- batched Anderson mixing: per replica ring of L slots, vectors of n doubles
__device__ __forceinline__ long long ring(int i, int head, int L) { return (long long)(((head - i) % L + L) % L); }

__global__ void k_am_insert(int R, long long n, int L, const int *__restrict__ head, const int *__restrict__ flag,
                            const double *__restrict__ w_cur, long long w_stride, const double *__restrict__ d_cur,
                            long long d_stride, double *__restrict__ w_hist, double *__restrict__ d_hist) {
    const int r = blockIdx.y;
    if (!flag[r]) return;
    const long long slot = ((long long)r * L + head[r]) * n;
    for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < n; m += (long long)gridDim.x * NT) {
        w_hist[slot + m] = w_cur[(long long)r * w_stride + m];
        d_hist[slot + m] = d_cur[(long long)r * d_stride + m];
    }
}

__global__ void k_am_batch_dots(int R, long long n, int L, const int *__restrict__ head, const int *__restrict__ ndots,
                                const double *__restrict__ d_hist, double *partials) {
    __shared__ double sh[NW];
    const int r = blockIdx.y, i = blockIdx.z;
    if (i >= ndots[r]) return;
    const double *d0 = d_hist + ((long long)r * L + ring(0, head[r], L)) * n;
    const double *di = d_hist + ((long long)r * L + ring(i, head[r], L)) * n;
    double acc = 0.0;
    for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < n; m += (long long)gridDim.x * NT) acc += d0[m] * di[m];
    acc = bsum(acc, sh);
    if (threadIdx.x == 0) partials[(((long long)r * L + i) * gridDim.x) + blockIdx.x] = acc;
}
__global__ void k_am_batch_dots_finish(int L, int nparts, const int *__restrict__ ndots, const double *__restrict__ partials,
                                       double *dots) {
    __shared__ double sh[NW];
    const int r = blockIdx.y, i = blockIdx.x;
    if (i >= ndots[r]) return;
    double acc = 0.0;
    for (int p = threadIdx.x; p < nparts; p += NT) acc += partials[(((long long)r * L + i) * nparts) + p];
    acc = bsum(acc, sh);
    if (threadIdx.x == 0) dots[(long long)r * L + i] = acc;
}

// mode 0: skip; 1: simple mixing w = w_cur + mix d_cur; 2: Anderson update from the ring
__global__ void k_am_batch_update(int R, long long n, int L, const int *__restrict__ head, const int *__restrict__ mode,
                                  const int *__restrict__ nh, const double *__restrict__ mix, const double *__restrict__ a,
                                  const double *__restrict__ w_cur, long long w_stride, const double *__restrict__ d_cur,
                                  long long d_stride, const double *__restrict__ w_hist, const double *__restrict__ d_hist,
                                  double *__restrict__ w_out, long long out_stride) {
    const int r = blockIdx.y;
    const int md = mode[r];
    if (md == 0) return;
    double *o = w_out + (long long)r * out_stride;
    if (md == 1) {
        const double mx = mix[r];
        const double *w = w_cur + (long long)r * w_stride, *d = d_cur + (long long)r * d_stride;
        for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < n; m += (long long)gridDim.x * NT) o[m] = w[m] + mx * d[m];
        return;
    }
    const int hd = head[r], k = nh[r];
    const double *w1 = w_hist + ((long long)r * L + ring(0, hd, L)) * n;
    const double *d1 = d_hist + ((long long)r * L + ring(0, hd, L)) * n;
    for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < n; m += (long long)gridDim.x * NT) {
        const double b = w1[m] + d1[m];
        double acc = b;
        for (int h = 0; h < k; h++) {
            const long long s = ((long long)r * L + ring(h + 1, hd, L)) * n;
            acc += a[(long long)r * L + h] * (w_hist[s + m] + d_hist[s + m] - w1[m] - d1[m]);
        }
        o[m] = acc;
    }
}

// ---- device control of the saddle-point loop (one thread per replica)
struct SaddleArgs {
    lfts_saddle_state st;
    double scale[LFTS_MAX_MONOMERS];
    double tol, start, mix_min;
    int R, I, it, maxh, L;
};

__global__ void k_saddle_control(SaddleArgs a, const double *__restrict__ var) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.R) return;
    const lfts_saddle_state &s = a.st;
    const int it = a.it > 0 ? a.it : *s.loop_iter;  // a graph loop keeps its iteration number on the device
    s.flag[r] = 0;
    s.ndots[r] = 0;
    s.mode[r] = 0;
    s.nh[r] = 0;
    if (s.active[r]) {
        double e = 0.0;
        for (int c = 0; c < a.I; c++) {
            const double v = var[(long long)r * a.I + c];
            const double sd = sqrt(v < 0.0 ? 0.0 : v) / a.scale[c];  // a NaN variance stays NaN
            e = (c == 0 || sd > e || isnan(sd)) ? sd : e;
        }
        const double eo = s.err[r];
        s.err_old[r] = eo;
        s.err[r] = e;
        s.iter[r] = it;
        if (e < a.tol) {
            s.active[r] = 0;  // converged: fields and statistics stay as they are
        } else {
            int na = s.n_anderson[r];
            if (e < a.start || na >= 0) na++;
            if (na >= 0) {
                na = na < a.maxh ? na : a.maxh;
                s.head_raw[r] = (s.head_raw[r] + 1) % a.L;
                s.flag[r] = 1;
                s.ndots[r] = na + 1;
            }
            if (na <= 0) {
                const double m = s.mix[r], m7 = m * 0.7;
                s.mix[r] = (eo < e) ? (m7 < a.mix_min ? a.mix_min : m7) : m * 1.01;
                s.mode[r] = 1;
            } else {
                s.mode[r] = 2;
                s.nh[r] = na;
            }
            s.n_anderson[r] = na;
            atomicOr(s.any_active, 1);
        }
    }
    s.head[r] = s.head_raw[r] > 0 ? s.head_raw[r] : 0;
}

// start of a saddle-point search of every replica (the state am_reset and the
// host loop start from); thread 0 also starts the graph loop's counter
__global__ void k_saddle_begin(lfts_saddle_state s, int R, double mix_init) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r == 0) {
        *s.loop_iter = 1;
        *s.any_active = 1;
    }
    if (r >= R) return;
    s.active[r] = 1;
    s.n_anderson[r] = -1;
    s.head_raw[r] = -1;
    s.iter[r] = 0;
    s.err[r] = 1e20;
    s.err_old[r] = 1e20;
    s.mix[r] = mix_init;
}
// last work of a loop body: continue while a replica is active and fewer than
// max_iter iterations have run; the counter bounds the loop by itself
__global__ void k_saddle_next(lfts_saddle_state s, cudaGraphConditionalHandle h, int max_iter) {
    const int it = *s.loop_iter;
    const unsigned go = (*s.any_active != 0 && it < max_iter && it < 1000000) ? 1u : 0u;
    *s.loop_iter = it + 1;
    cudaGraphSetConditional(h, go);
}

constexpr int FINISH_MAX_POLY = 8;
struct FinishArgs {
    lfts_saddle_state st;
    int R, S, P;
    double tol, h_const;
    double h1[LFTS_MAX_MONOMERS], h2[LFTS_MAX_MONOMERS], poly[FINISH_MAX_POLY];
};
// per replica: failure flag, Hamiltonian, the pressure mean, the packed statistics
__global__ void k_step_finish(FinishArgs a, const double *__restrict__ mean, const double *__restrict__ msq,
                              const double *__restrict__ Q, double *__restrict__ pm, double *__restrict__ stats) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.R) return;
    const int R = a.R, S = a.S, P = a.P;
    const double e = a.st.err[r];
    const double *mr = mean + (long long)r * S, *qr = msq + (long long)r * S;
    double h = -mr[S - 1];
    for (int i = 0; i < S - 1; i++) {
        h += a.h2[i] * qr[i];
        h += a.h1[i] * mr[i];
    }
    double hp = 0.0;
    for (int p = 0; p < P; p++) hp -= a.poly[p] * log(Q[(long long)r * P + p]);
    stats[r] = (double)a.st.iter[r];
    stats[R + r] = e;
    stats[2 * R + r] = hp + h + a.h_const;
    stats[3 * R + r] = (isnan(e) || e >= a.tol) ? 1.0 : 0.0;
    double *o = stats + 4 * (long long)R;
    for (int p = 0; p < P; p++) o[(long long)r * P + p] = Q[(long long)r * P + p];
    o += (long long)R * P;
    for (int i = 0; i < S; i++) {
        o[(long long)r * S + i] = mr[i];
        o[(long long)R * S + (long long)r * S + i] = qr[i];
    }
    pm[r] = mr[S - 1];
    a.st.active[r] = 1;
}
struct PhiPtrs {
    double *phi[LFTS_MAX_MONOMERS];
};
// a replica whose saddle point failed gets its fields and concentrations back
__global__ void k_restore_failed(int R, int S, long long M, const double *__restrict__ failed, double *__restrict__ w_aux,
                                 const double *__restrict__ w_save, PhiPtrs phi, const double *__restrict__ phi_save) {
    const int r = blockIdx.y;
    if (failed[r] == 0.0) return;
    const long long n = (long long)S * M, base = (long long)r * n;
    for (long long t = blockIdx.x * (long long)NT + threadIdx.x; t < n; t += (long long)gridDim.x * NT) {
        w_aux[base + t] = w_save[base + t];
        const int sidx = (int)(t / M);
        phi.phi[sidx][(long long)r * M + (t - (long long)sidx * M)] = phi_save[base + t];
    }
}

// Largest Anderson history the device solve holds (shared memory of one block).
constexpr int AM_SOLVE_MAX = LFTS_AM_SOLVE_MAX_HIST;

// One block of 32 threads per replica; U and V in shared memory.  The threads
// split the rows j of each elimination step i, which leaves every element's
// sequence of operations that of the serial loop.
__global__ void k_am_solve(int R, int L, const int *__restrict__ head, const int *__restrict__ ndots,
                           const int *__restrict__ mode, const int *__restrict__ nh, const double *__restrict__ dots,
                           double *__restrict__ dot_ring, double *__restrict__ a) {
    __shared__ double u[AM_SOLVE_MAX][AM_SOLVE_MAX + 1], v[AM_SOLVE_MAX], x[AM_SOLVE_MAX];
    const int r = blockIdx.x, t = threadIdx.x;
    const int nd = ndots[r];
    if (nd == 0) return;
    const int hd = head[r];
    double *row0 = dot_ring + ((long long)r * L + hd) * L;
    for (int i = t; i < nd; i += 32) row0[i] = dots[(long long)r * L + i];
    __syncthreads();
    if (mode[r] != 2) return;
    const int n = nh[r];
    for (int e = t; e < n * n; e += 32) {
        const int i = e / n, j = e - i * n;
        const int k = (i < j ? i : j) + 1, d = i > j ? i - j : j - i;
        const double *rk = dot_ring + ((long long)r * L + ((hd - k) % L + L) % L) * L;
        u[i][j] = row0[0] - row0[i + 1] - row0[j + 1] + rk[d];
    }
    for (int i = t; i < n; i += 32) v[i] = row0[0] - row0[i + 1];
    __syncthreads();
    // elimination without pivoting; products and sums rounded separately (no
    // fused multiply-add), as the host computes them
    for (int i = 0; i < n; i++) {
        for (int j = i + 1 + t; j < n; j += 32) {
            const double f = u[j][i] / u[i][i];
            v[j] = __dsub_rn(v[j], __dmul_rn(v[i], f));
            for (int k = i + 1; k < n; k++) u[j][k] = __dsub_rn(u[j][k], __dmul_rn(u[i][k], f));
        }
        __syncthreads();
    }
    if (t == 0) {
        x[n - 1] = v[n - 1] / u[n - 1][n - 1];
        for (int i = n - 2; i >= 0; i--) {
            double sum = 0.0;
            for (int j = i + 1; j < n; j++) sum = __dadd_rn(sum, __dmul_rn(u[i][j], x[j]));
            x[i] = (v[i] - sum) / u[i][i];
        }
        for (int i = 0; i < n; i++) a[(long long)r * L + i] = x[i];
    }
}

// ---- PCG64 streams on the device (O'Neill's PCG, 128-bit LCG with the XSL-RR
// 64-bit output; the generator numpy's PCG64 implements): per stream four
// uint64 (state hi, lo, increment hi, lo).  Each thread jumps to its offset by
// Brown's O(log k) LCG jump-ahead and draws RAW_PER_THREAD consecutive outputs.
typedef unsigned __int128 u128;
constexpr unsigned long long PCG_MULT_HI = 0x2360ED051FC65DA4ULL, PCG_MULT_LO = 0x4385DF649FCCF645ULL;
constexpr int RAW_PER_THREAD = 16;

__device__ __forceinline__ u128 u128_of(unsigned long long hi, unsigned long long lo) { return ((u128)hi << 64) | lo; }
__device__ __forceinline__ unsigned long long pcg_output(u128 s) {
    const unsigned long long hi = (unsigned long long)(s >> 64), lo = (unsigned long long)s;
    const unsigned long long x = hi ^ lo;
    const unsigned r = (unsigned)(hi >> 58);
    return (x >> r) | (x << ((64 - r) & 63));
}
// state after k steps of s -> s * MULT + inc
__device__ u128 pcg_jump(u128 s, u128 inc, unsigned long long k) {
    u128 acc_mult = 1, acc_plus = 0, cur_mult = u128_of(PCG_MULT_HI, PCG_MULT_LO), cur_plus = inc;
    while (k) {
        if (k & 1) {
            acc_mult *= cur_mult;
            acc_plus = acc_plus * cur_mult + cur_plus;
        }
        cur_plus = (cur_mult + 1) * cur_plus;
        cur_mult *= cur_mult;
        k >>= 1;
    }
    return acc_mult * s + acc_plus;
}

// MODE 0: raw outputs to out_raw; MODE 1: sigma * N(0,1) by Box-Muller on
// pairs (u1, u2) = 53-bit uniforms of raw outputs 2p, 2p + 1:
// z = sqrt(-2 ln(1 - u1)) (cos, sin)(2 pi u2)
template <int MODE>
__global__ void k_pcg64(const unsigned long long *__restrict__ states, long long n, double sigma,
                        unsigned long long *__restrict__ out_raw, double *__restrict__ out) {
    const int st = blockIdx.y;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long first = t * RAW_PER_THREAD;
    const long long nraw = MODE == 0 ? n : 2 * ((n + 1) / 2);
    if (first >= nraw) return;
    const unsigned long long *sp = states + 4 * (long long)st;
    const u128 inc = u128_of(sp[2], sp[3]);
    u128 s = pcg_jump(u128_of(sp[0], sp[1]), inc, (unsigned long long)first);
    const u128 mult = u128_of(PCG_MULT_HI, PCG_MULT_LO);
    unsigned long long raw[RAW_PER_THREAD];
#pragma unroll
    for (int i = 0; i < RAW_PER_THREAD; i++) {
        s = s * mult + inc;
        raw[i] = pcg_output(s);
    }
    if (MODE == 0) {
        unsigned long long *o = out_raw + (long long)st * n + first;
#pragma unroll
        for (int i = 0; i < RAW_PER_THREAD; i++)
            if (first + i < n) o[i] = raw[i];
    } else {
        double *o = out + (long long)st * n + first;
#pragma unroll
        for (int i = 0; i < RAW_PER_THREAD; i += 2) {
            const double u1 = (double)(raw[i] >> 11) * 0x1.0p-53, u2 = (double)(raw[i + 1] >> 11) * 0x1.0p-53;
            const double r = sqrt(-2.0 * log1p(-u1));
            double sn, cs;
            sincospi(2.0 * u2, &sn, &cs);
            if (first + i < n) o[i] = sigma * r * cs;
            if (first + i + 1 < n) o[i + 1] = sigma * r * sn;
        }
    }
}

__global__ void k_pcg64_advance(unsigned long long *__restrict__ states, int nstreams, unsigned long long k) {
    const int st = blockIdx.x * blockDim.x + threadIdx.x;
    if (st >= nstreams) return;
    unsigned long long *sp = states + 4 * (long long)st;
    const u128 s = pcg_jump(u128_of(sp[0], sp[1]), u128_of(sp[2], sp[3]), k);
    sp[0] = (unsigned long long)(s >> 64);
    sp[1] = (unsigned long long)s;
}

int grid1(long long n, int cap) {
    long long b = (n + NT - 1) / NT;
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

bool fill_deriv(DerivArgs &d, int S, int nf, const int *idx, const double *scale, const double *A, const double *h1,
                const double *h2, const double *const *phi) {
    if (S < 1 || S > LFTS_MAX_MONOMERS || nf < 0 || nf > S) return false;
    d.S = S;
    d.nf = nf;
    for (int c = 0; c < nf; c++) {
        d.idx[c] = idx[c];
        d.scale[c] = scale ? scale[c] : 1.0;
        if (idx[c] < 0 || idx[c] >= S) return false;
    }
    for (int i = 0; i < S * S; i++) d.A[i] = A[i];
    for (int i = 0; i < S; i++) {
        d.h1[i] = (h1 && i < S - 1) ? h1[i] : 0.0;
        d.h2[i] = (h2 && i < S - 1) ? h2[i] : 0.0;
        d.phi[i] = phi[i];
    }
    return true;
}

}  // namespace

extern "C" int lfts_lfts_monomer_fields(lfts_ctx ctx, int R, int S, long long M, const double *A, const double *w_aux,
                                        double *const *w_mono) {
    if (S < 1 || S > LFTS_MAX_MONOMERS) return lfail("monomer count out of range");
    MonoArgs a;
    a.S = S;
    for (int i = 0; i < S * S; i++) a.A[i] = A[i];
    for (int i = 0; i < S; i++) a.w[i] = w_mono[i];
    k_monomer_fields<<<grid1((long long)R * M, 148 * 16), NT, 0, (cudaStream_t)lfts_ctx_stream(ctx)>>>(a, w_aux, M, R);
    lfts_internal_count(ctx, 1);
    LCK(cudaPeekAtLastError());
    return 0;
}

extern "C" int lfts_lfts_field_deriv(lfts_ctx ctx, int R, int S, long long M, int nf, const int *idx, const double *scale,
                                     const double *A, const double *h1, const double *h2, const double *w_aux,
                                     const double *const *phi, double *out, const int *active) {
    DerivArgs d;
    if (!fill_deriv(d, S, nf, idx, scale, A, h1, h2, phi)) return lfail("invalid field-derivative arguments");
    k_deriv<<<dim3(grid1(M, 1024), R), NT, 0, (cudaStream_t)lfts_ctx_stream(ctx)>>>(d, w_aux, M, R, out, active);
    lfts_internal_count(ctx, 1);
    LCK(cudaPeekAtLastError());
    return 0;
}

extern "C" int lfts_lfts_langevin(lfts_ctx ctx, int R, int S, long long M, int nreal, const int *idx, const double *A,
                                  const double *h1, const double *h2, const double *const *phi, double dt,
                                  const double *dt_scaling, double *w_aux, const double *xi_prev, const double *xi_cur,
                                  const int *active) {
    LangevinArgs a;
    if (!fill_deriv(a.d, S, nreal, idx, nullptr, A, h1, h2, phi)) return lfail("invalid Langevin arguments");
    a.dt = dt;
    for (int c = 0; c < nreal; c++) {
        a.s[c] = dt_scaling[c];
        a.sqrt_s[c] = sqrt(dt_scaling[c]);
    }
    k_langevin<<<dim3(grid1(M, 1024), R), NT, 0, (cudaStream_t)lfts_ctx_stream(ctx)>>>(a, w_aux, M, xi_prev, xi_cur, active);
    lfts_internal_count(ctx, 1);
    LCK(cudaPeekAtLastError());
    return 0;
}

extern "C" int lfts_lfts_row_moments(lfts_ctx ctx, const double *x, int R, int rows_per_rep, long long M, long long row_stride,
                                     long long rep_stride, const double *center, double *partials, double *mean, double *msq) {
    const int rows = R * rows_per_rep;
    const int chunks = 64;
    cudaStream_t st = (cudaStream_t)lfts_ctx_stream(ctx);
    k_row_sums<<<dim3(chunks, rows), NT, 0, st>>>(x, M, row_stride, rows_per_rep, rep_stride, center, partials);
    k_row_finish<<<rows, NT, 0, st>>>(partials, chunks, M, mean, msq);
    lfts_internal_count(ctx, 2);
    LCK(cudaPeekAtLastError());
    return 0;
}

extern "C" int lfts_lfts_subtract_mean(lfts_ctx ctx, double *w_aux, int R, int S, int field, long long M, const double *mean,
                                       const int *active) {
    k_subtract_mean<<<dim3(grid1(M, 1024), R), NT, 0, (cudaStream_t)lfts_ctx_stream(ctx)>>>(w_aux, S, field, M, mean, active);
    lfts_internal_count(ctx, 1);
    LCK(cudaPeekAtLastError());
    return 0;
}

extern "C" int lfts_am_batch_insert(lfts_ctx ctx, int R, long long n, int L, const int *head, const int *flag,
                                    const double *w_cur, long long w_stride, const double *d_cur, long long d_stride,
                                    double *w_hist, double *d_hist) {
    k_am_insert<<<dim3(grid1(n, 1024), R), NT, 0, (cudaStream_t)lfts_ctx_stream(ctx)>>>(R, n, L, head, flag, w_cur, w_stride,
                                                                                       d_cur, d_stride, w_hist, d_hist);
    lfts_internal_count(ctx, 1);
    LCK(cudaPeekAtLastError());
    return 0;
}

extern "C" int lfts_am_batch_dots(lfts_ctx ctx, int R, long long n, int L, const int *head, const int *ndots,
                                  const double *d_hist, double *partials, double *dots) {
    const int chunks = 64;
    cudaStream_t st = (cudaStream_t)lfts_ctx_stream(ctx);
    k_am_batch_dots<<<dim3(chunks, R, L), NT, 0, st>>>(R, n, L, head, ndots, d_hist, partials);
    k_am_batch_dots_finish<<<dim3(L, R), NT, 0, st>>>(L, chunks, ndots, partials, dots);
    lfts_internal_count(ctx, 2);
    LCK(cudaPeekAtLastError());
    return 0;
}

extern "C" int lfts_am_batch_update(lfts_ctx ctx, int R, long long n, int L, const int *head, const int *mode,
                                    const int *nh, const double *mix, const double *a, const double *w_cur, long long w_stride,
                                    const double *d_cur, long long d_stride, const double *w_hist, const double *d_hist,
                                    double *w_out, long long out_stride) {
    k_am_batch_update<<<dim3(grid1(n, 1024), R), NT, 0, (cudaStream_t)lfts_ctx_stream(ctx)>>>(
        R, n, L, head, mode, nh, mix, a, w_cur, w_stride, d_cur, d_stride, w_hist, d_hist, w_out, out_stride);
    lfts_internal_count(ctx, 1);
    LCK(cudaPeekAtLastError());
    return 0;
}

extern "C" int lfts_saddle_control(lfts_ctx ctx, int R, int I, int it, const double *var, const double *scale, double tolerance,
                                   double am_start_error, int am_max_hist, double am_mix_min, const lfts_saddle_state *st) {
    if (!ctx || !var || !scale || !st) return lfts_internal_fail("null argument");
    if (R < 1 || I < 1 || I > LFTS_MAX_MONOMERS) return lfts_internal_fail("saddle control: bad replica or field count");
    if (am_max_hist < 0) return lfts_internal_fail("saddle control: am_max_hist must be >= 0");
    SaddleArgs a;
    a.st = *st;
    for (int c = 0; c < I; c++) a.scale[c] = scale[c];
    a.tol = tolerance;
    a.start = am_start_error;
    a.mix_min = am_mix_min;
    a.R = R;
    a.I = I;
    a.it = it;
    a.maxh = am_max_hist;
    a.L = am_max_hist + 1;
    cudaStream_t s = (cudaStream_t)lfts_ctx_stream(ctx);
    LCK(cudaMemsetAsync(st->any_active, 0, sizeof(int), s));
    k_saddle_control<<<(R + 63) / 64, 64, 0, s>>>(a, var);
    lfts_internal_count(ctx, 1);
    LCK(cudaPeekAtLastError());
    return 0;
}

extern "C" int lfts_saddle_begin(lfts_ctx ctx, int R, double mix_init, const lfts_saddle_state *st) {
    if (!ctx || !st || !st->loop_iter || !st->any_active) return lfts_internal_fail("null argument");
    if (R < 1) return lfts_internal_fail("saddle begin: R must be positive");
    k_saddle_begin<<<(R + 63) / 64, 64, 0, (cudaStream_t)lfts_ctx_stream(ctx)>>>(*st, R, mix_init);
    lfts_internal_count(ctx, 1);
    LCK(cudaPeekAtLastError());
    return 0;
}

extern "C" int lfts_saddle_next(lfts_ctx ctx, unsigned long long handle, const lfts_saddle_state *st, int max_iter) {
    if (!ctx || !st || !st->loop_iter || !st->any_active) return lfts_internal_fail("null argument");
    if (max_iter < 1) return lfts_internal_fail("saddle next: max_iter must be positive");
    k_saddle_next<<<1, 1, 0, (cudaStream_t)lfts_ctx_stream(ctx)>>>(*st, (cudaGraphConditionalHandle)handle, max_iter);
    lfts_internal_count(ctx, 1);
    LCK(cudaPeekAtLastError());
    return 0;
}

extern "C" int lfts_lfts_step_finish(lfts_ctx ctx, int R, int S, int P, long long M, const lfts_saddle_state *st,
                                     double tolerance, const double *mean, const double *msq, const double *Q, const double *h1,
                                     const double *h2, double h_const, const double *poly, int restore, double *w_aux,
                                     const double *w_save, double *const *phi, const double *phi_save, double *scratch,
                                     double *stats) {
    if (!ctx || !st || !mean || !msq || !Q || !poly || !w_aux || !scratch || !stats) return lfts_internal_fail("null argument");
    if (R < 1 || S < 1 || S > LFTS_MAX_MONOMERS || P < 1 || P > FINISH_MAX_POLY)
        return lfts_internal_fail("step finish: R, S (<= " + std::to_string(LFTS_MAX_MONOMERS) + ") or P (<= 8) out of range");
    if (restore && (!w_save || !phi || !phi_save)) return lfts_internal_fail("step finish: restore needs the saved state");
    FinishArgs a;
    a.st = *st;
    a.R = R;
    a.S = S;
    a.P = P;
    a.tol = tolerance;
    a.h_const = h_const;
    for (int i = 0; i < LFTS_MAX_MONOMERS; i++) {
        a.h1[i] = (h1 && i < S - 1) ? h1[i] : 0.0;
        a.h2[i] = (h2 && i < S - 1) ? h2[i] : 0.0;
    }
    for (int p = 0; p < FINISH_MAX_POLY; p++) a.poly[p] = p < P ? poly[p] : 0.0;
    cudaStream_t s = (cudaStream_t)lfts_ctx_stream(ctx);
    k_step_finish<<<(R + 63) / 64, 64, 0, s>>>(a, mean, msq, Q, scratch, stats);
    k_subtract_mean<<<dim3(grid1(M, 1024), R), NT, 0, s>>>(w_aux, S, S - 1, M, scratch, nullptr);
    int n = 2;
    if (restore) {
        PhiPtrs pp;
        for (int i = 0; i < LFTS_MAX_MONOMERS; i++) pp.phi[i] = i < S ? phi[i] : nullptr;
        k_restore_failed<<<dim3(grid1((long long)S * M, 1024), R), NT, 0, s>>>(R, S, M, stats + 3 * (long long)R, w_aux, w_save,
                                                                               pp, phi_save);
        n++;
    }
    lfts_internal_count(ctx, n);
    LCK(cudaPeekAtLastError());
    return 0;
}

extern "C" int lfts_am_batch_solve(lfts_ctx ctx, int R, int L, const int *head, const int *ndots, const int *mode, const int *nh,
                                   const double *dots, double *dot_ring, double *a) {
    if (!ctx || !head || !ndots || !mode || !nh || !dots || !dot_ring || !a) return lfts_internal_fail("null argument");
    if (L < 1 || L - 1 > AM_SOLVE_MAX) return lfts_internal_fail("device Anderson solve holds at most 32 history vectors");
    k_am_solve<<<R, 32, 0, (cudaStream_t)lfts_ctx_stream(ctx)>>>(R, L, head, ndots, mode, nh, dots, dot_ring, a);
    lfts_internal_count(ctx, 1);
    LCK(cudaPeekAtLastError());
    return 0;
}

static int pcg64_launch(lfts_ctx ctx, unsigned long long *states, int nstreams, long long n, double sigma,
                        unsigned long long *out_raw, double *out) {
    if (!ctx || !states || (!out_raw && !out)) return lfts_internal_fail("null argument");
    if (nstreams < 1 || nstreams > 65535 || n < 0) return lfts_internal_fail("pcg64: nstreams must be 1..65535 and n >= 0");
    if (n == 0) return 0;
    const long long nraw = out_raw ? n : 2 * ((n + 1) / 2);
    const long long threads = (nraw + RAW_PER_THREAD - 1) / RAW_PER_THREAD;
    const long long blocks = (threads + NT - 1) / NT;
    if (blocks > 0x7fffffffLL) return lfts_internal_fail("pcg64: too many draws in one call");
    cudaStream_t s = (cudaStream_t)lfts_ctx_stream(ctx);
    if (out_raw) k_pcg64<0><<<dim3((unsigned)blocks, nstreams), NT, 0, s>>>(states, n, sigma, out_raw, nullptr);
    else k_pcg64<1><<<dim3((unsigned)blocks, nstreams), NT, 0, s>>>(states, n, sigma, nullptr, out);
    k_pcg64_advance<<<(nstreams + 63) / 64, 64, 0, s>>>(states, nstreams, (unsigned long long)nraw);
    lfts_internal_count(ctx, 2);
    LCK(cudaPeekAtLastError());
    return 0;
}

extern "C" int lfts_pcg64_normal(lfts_ctx ctx, unsigned long long *states, int nstreams, long long n, double sigma,
                                 double *out) {
    return pcg64_launch(ctx, states, nstreams, n, sigma, nullptr, out);
}

extern "C" int lfts_pcg64_raw(lfts_ctx ctx, unsigned long long *states, int nstreams, long long n, unsigned long long *out) {
    return pcg64_launch(ctx, states, nstreams, n, 0.0, out, nullptr);
}
