// Real-space Crank-Nicolson step for continuous chains (the reference's
// "realspace" method, src/platforms/cpu/CpuSolverReal.cpp:135-549 and
// src/platforms/cuda/CudaSolverReal.cu:371-956): for boxes with reflecting or
// absorbing walls, where the pseudo-spectral step does not apply.
//
//   q_out = e * ADI(e * q_in),  e = exp(-w ds / 2)
//
// ADI (alternating direction implicit, the reference's scheme): a first sweep
// implicit along the box's first axis whose right-hand side applies the full
// explicit half of the operator, then one sweep per further axis implicit
// along it, each a batch of independent tridiagonal solves (periodic axes by
// Sherman-Morrison).  The pivots of every axis depend only on its matrix, so
// the host computes them once (lfts_realspace_tables) and a line solve is the
// reference's forward and backward substitution with those pivots.
//
// Launch shape: one thread per line, lines of all jobs of a launch in one
// grid (blockIdx.y = job).  Lines along the first padded axes are coalesced
// across the threads of a warp; lines along the last axis (contiguous in
// memory) are read through L1, each thread walking its own line.
#pragma once
#include "lfts_step_kernels.cuh"

namespace lfts {
namespace rs {

constexpr int ROWS = 7;  // l, d, h, pivot, ratio, periodic vector, 1 / pivot

// view of one type's tables (device doubles, layout of lfts_realspace_tables)
struct Axis {
    const double *l, *d, *h, *c, *v, *rp;
    double denom;
    bool periodic;
    int n;
};
__device__ __forceinline__ Axis axis(const double *tab, const GridPlan &g, int a) {
    const int n[3] = {g.n0, g.n1, g.n2};
    long long off = 0;
    for (int b = 0; b < a; b++) off += (long long)ROWS * n[b];
    const double *t = tab + off;
    const long long tail = (long long)ROWS * (n[0] + n[1] + n[2]);
    Axis ax;
    ax.n = n[a];
    ax.l = t;
    ax.d = t + n[a];
    ax.h = t + 2 * n[a];
    ax.c = t + 4 * n[a];
    ax.v = t + 5 * n[a];
    ax.rp = t + 6 * n[a];
    ax.denom = tab[tail + a];
    ax.periodic = tab[tail + 3 + a] != 0.0;
    return ax;
}
__device__ __forceinline__ int nb_lo(const Axis &ax, int i) { return ax.periodic ? (i + ax.n - 1) % ax.n : (i > 0 ? i - 1 : 0); }
__device__ __forceinline__ int nb_hi(const Axis &ax, int i) { return ax.periodic ? (i + 1) % ax.n : (i < ax.n - 1 ? i + 1 : ax.n - 1); }

// The tridiagonal solve of one line x[0..n) (stride st), right-hand side
// already in x: forward substitution with the pivots, backward with the
// ratios, and for a periodic axis the Sherman-Morrison correction.
// (The forward substitution multiplies by the reciprocal pivots: one rounding
// away from the reference's division.)
__device__ __forceinline__ void solve_line(const Axis &ax, double *x, long long st) {
    const int n = ax.n;
    double prev = x[0] * ax.rp[0];
    x[0] = prev;
    for (int i = 1; i < n; i++) {
        prev = (x[i * st] - ax.l[i] * prev) * ax.rp[i];
        x[i * st] = prev;
    }
    double next = prev;
    for (int i = n - 2; i >= 0; i--) {
        next = x[i * st] - ax.c[i] * next;
        x[i * st] = next;
    }
    if (ax.periodic) {
        const double value = (x[0] + ax.l[0] * x[(n - 1) * st]) / ax.denom;
        for (int i = 0; i < n; i++) x[i * st] = x[i * st] - ax.v[i] * value;
    }
}

// line `line` along padded axis A: base offset and element stride
__device__ __forceinline__ void line_of(const GridPlan &g, int A, long long line, long long &base, long long &st) {
    if (A == 0) {
        base = line;  // (j, k) -> j n2 + k
        st = (long long)g.n1 * g.n2;
    } else if (A == 1) {
        const long long i = line / g.n2, k = line - i * g.n2;
        base = i * g.n1 * g.n2 + k;
        st = g.n2;
    } else {
        base = line * g.n2;  // (i, j) -> (i n1 + j) n2
        st = 1;
    }
}

// e * q at flat index m (e = fac^2)
__device__ __forceinline__ double eq(const double *q, const double *fac, long long m) {
    const double f = fac[m];
    return q[m] * (f * f);
}

// First sweep: implicit along the box's first axis (padded A0 = 3 - dim),
// right-hand side the explicit operator of all axes
// (CpuSolverReal.cpp:223-242, 2D :355-373, 1D :437-449); the solution goes to
// dst (the scratch, or q_out when dim = 1, then times e).
template <int DIM>
__global__ void __launch_bounds__(NTHR) k_rs_first(GridPlan g, const lfts_step_job *__restrict__ jobs, int s) {
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    constexpr int A0 = 3 - DIM;
    const long long nlines = g.M / (A0 == 0 ? g.n0 : A0 == 1 ? g.n1 : g.n2);
    const long long line = blockIdx.x * (long long)NTHR + threadIdx.x;
    if (line >= nlines) return;
    const double *q = (const double *)jb.in + s * jb.in_stride;
    const double *fac = (const double *)jb.fac;
    const double *tab = (const double *)jb.bond;
    double *dst = DIM == 1 ? (double *)jb.out + s * jb.out_stride : (double *)jb.spec;
    long long base, st;
    line_of(g, A0, line, base, st);
    const Axis X = axis(tab, g, A0);
    if (DIM == 3) {
        const Axis Y = axis(tab, g, 1), Z = axis(tab, g, 2);
        const int j = (int)(line / g.n2), k = (int)(line - (long long)j * g.n2);
        const int jm = nb_lo(Y, j), jp = nb_hi(Y, j), km = nb_lo(Z, k), kp = nb_hi(Z, k);
        const long long pj = (long long)g.n2, dj_m = (jm - j) * pj, dj_p = (jp - j) * pj, dk_m = km - k, dk_p = kp - k;
        for (int i = 0; i < X.n; i++) {
            const int im = nb_lo(X, i), ip = nb_hi(X, i);
            const long long m = base + i * st;
            dst[m] = 2.0 * ((3.0 - 0.5 * X.d[i] - Y.d[j] - Z.d[k]) * eq(q, fac, m) - Z.l[k] * eq(q, fac, m + dk_m) -
                            Z.h[k] * eq(q, fac, m + dk_p) - Y.l[j] * eq(q, fac, m + dj_m) - Y.h[j] * eq(q, fac, m + dj_p)) -
                     X.l[i] * eq(q, fac, base + im * st) - X.h[i] * eq(q, fac, base + ip * st);
        }
    } else if (DIM == 2) {
        const Axis Y = axis(tab, g, 2);
        const int j = (int)line;  // padded axes (1, 2): a line along axis 1 is column j of axis 2
        const int jm = nb_lo(Y, j), jp = nb_hi(Y, j);
        for (int i = 0; i < X.n; i++) {
            const int im = nb_lo(X, i), ip = nb_hi(X, i);
            const long long m = base + i * st;
            dst[m] = 2.0 * ((2.0 - 0.5 * X.d[i] - Y.d[j]) * eq(q, fac, m) - Y.l[j] * eq(q, fac, m + (jm - j)) -
                            Y.h[j] * eq(q, fac, m + (jp - j))) -
                     X.l[i] * eq(q, fac, base + im * st) - X.h[i] * eq(q, fac, base + ip * st);
        }
    } else {
        for (int i = 0; i < X.n; i++) {
            const int im = nb_lo(X, i), ip = nb_hi(X, i);
            dst[base + i * st] = (2.0 - X.d[i]) * eq(q, fac, base + i * st) - X.l[i] * eq(q, fac, base + im * st) -
                                 X.h[i] * eq(q, fac, base + ip * st);
        }
    }
    solve_line(X, dst + base, st);
    if (DIM == 1)
        for (int i = 0; i < X.n; i++) {
            const double f = fac[base + i * st];
            dst[base + i * st] *= f * f;
        }
}

// Later sweep along padded axis A (CpuSolverReal.cpp:250-275 and :277-306,
// 2D :382-400): right-hand side prev + (d - 1) e q + l e q[-] + h e q[+] along
// A; the solution goes to dst; last sweep (dst = q_out) then times e.
template <int A, bool LAST>
__global__ void __launch_bounds__(NTHR) k_rs_next(GridPlan g, const lfts_step_job *__restrict__ jobs, int s, int src_half) {
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const long long nlines = g.M / (A == 0 ? g.n0 : A == 1 ? g.n1 : g.n2);
    const long long line = blockIdx.x * (long long)NTHR + threadIdx.x;
    if (line >= nlines) return;
    const double *q = (const double *)jb.in + s * jb.in_stride;
    const double *fac = (const double *)jb.fac;
    const double *prev = (const double *)jb.spec + (src_half ? g.M : 0);
    double *dst = LAST ? (double *)jb.out + s * jb.out_stride : (double *)jb.spec + (src_half ? 0 : g.M);
    long long base, st;
    line_of(g, A, line, base, st);
    const Axis Y = axis((const double *)jb.bond, g, A);
    for (int j = 0; j < Y.n; j++) {
        const int jm = nb_lo(Y, j), jp = nb_hi(Y, j);
        const long long m = base + j * st;
        dst[m] = prev[m] + (Y.d[j] - 1.0) * eq(q, fac, m) + Y.l[j] * eq(q, fac, base + jm * st) + Y.h[j] * eq(q, fac, base + jp * st);
    }
    solve_line(Y, dst + base, st);
    if (LAST)
        for (int j = 0; j < Y.n; j++) {
            const double f = fac[base + j * st];
            dst[base + j * st] *= f * f;
        }
}

// The sweep along the last axis (lines contiguous in memory), tiled: a block
// of ZL threads takes ZL consecutive lines, loads e q and the previous sweep
// into shared memory with coalesced accesses (rows padded to n + 1 doubles so
// the threads' line walks fall in different banks), solves one line per
// thread there, and writes the lines back coalesced (times e when LAST).
constexpr int ZL = 64;
template <bool LAST>
__global__ void __launch_bounds__(ZL) k_rs_last_axis(GridPlan g, const lfts_step_job *__restrict__ jobs, int s, int src_half) {
    extern __shared__ double sm_rs[];
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int n = g.n2, ld = n + 1;
    const long long nlines = g.M / n, line0 = (long long)blockIdx.x * ZL;
    const int nl = nlines - line0 < ZL ? (int)(nlines - line0) : ZL;
    const double *q = (const double *)jb.in + s * jb.in_stride;
    const double *fac = (const double *)jb.fac;
    const double *prev = (const double *)jb.spec + (src_half ? g.M : 0);
    double *dst = LAST ? (double *)jb.out + s * jb.out_stride : (double *)jb.spec + (src_half ? 0 : g.M);
    double *E = sm_rs, *X = sm_rs + ZL * ld;
    const Axis Z = axis((const double *)jb.bond, g, 2);
    const long long base = line0 * n;
    for (int t = threadIdx.x; t < nl * n; t += ZL) {
        const int r = t / n, k = t - r * n;
        E[r * ld + k] = eq(q, fac, base + t);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nl * n; t += ZL) {
        const int r = t / n, k = t - r * n;
        const double *e = E + r * ld;
        const int km = nb_lo(Z, k), kp = nb_hi(Z, k);
        X[r * ld + k] = prev[base + t] + (Z.d[k] - 1.0) * e[k] + Z.l[k] * e[km] + Z.h[k] * e[kp];
    }
    __syncthreads();
    if (threadIdx.x < nl) solve_line(Z, X + threadIdx.x * ld, 1);
    __syncthreads();
    for (int t = threadIdx.x; t < nl * n; t += ZL) {
        const int r = t / n, k = t - r * n;
        double v = X[r * ld + k];
        if (LAST) {
            const double f = fac[base + t];
            v *= f * f;
        }
        dst[base + t] = v;
    }
}

}  // namespace rs
}  // namespace lfts
