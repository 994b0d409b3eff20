// Specialised step kernels for cubic grids N^3 with N in {32, 48, 64, 96, 128}.
//
// Same five passes as lfts_step_kernels.cuh (and the same results), with the
// transform plan fixed at compile time:
//   * radices, spans and line strides are constants, so butterfly indexing is
//     shifts and multiplies instead of runtime integer division;
//   * z-lines are padded (element e stored at e + e/8, lines 9/8 N + 1 long),
//     which removes the shared-memory bank conflicts of the first radix-8
//     stage (lanes 8 elements apart) and between lines of one warp;
//   * stage twiddles come from a per-stage table laid out [j-1][k1], so the
//     lanes of a warp read consecutive entries;
//   * every warp loads its rows with independent loads first (memory-level
//     parallelism), then transforms.
#pragma once
#include "lfts_step_kernels.cuh"

namespace lfts {
namespace fast {

// ---- compile-time plan, same factorisation rule as the runtime one (8s, 4s, 2s, 3s, 5s)
__host__ __device__ constexpr int nrad(int n) {
    int c = 0;
    while (n % 8 == 0) { n /= 8; c++; }
    while (n % 4 == 0) { n /= 4; c++; }
    while (n % 2 == 0) { n /= 2; c++; }
    while (n % 3 == 0) { n /= 3; c++; }
    while (n % 5 == 0) { n /= 5; c++; }
    return n == 1 ? c : -1;
}
// i-th radix, outermost first
__host__ __device__ constexpr int rad(int n, int i) {
    int c = 0;
    const int rs[5] = {8, 4, 2, 3, 5};
    for (int k = 0; k < 5; k++) {
        while (n % rs[k] == 0) {
            if (c == i) return rs[k];
            n /= rs[k];
            c++;
        }
    }
    return 1;
}
// product of the innermost s radices (= span M of stage s, innermost-first)
__host__ __device__ constexpr int span_inner(int n, int s) {
    int p = 1;
    const int nf = nrad(n);
    for (int k = 0; k < s; k++) p *= rad(n, nf - 1 - k);
    return p;
}
// stage twiddle table: stage s holds (R_s - 1) x M_s entries
__host__ __device__ constexpr int stw_offset(int n, int s) {
    int o = 0;
    const int nf = nrad(n);
    for (int k = 0; k < s; k++) o += (rad(n, nf - 1 - k) - 1) * span_inner(n, k);
    return o;
}
__host__ __device__ constexpr int stw_size(int n) { return stw_offset(n, nrad(n)); }
__host__ __device__ constexpr int padded(int n) { return n + n / 8 + 1; }
__host__ __device__ constexpr int zlines(int n) { return (256 / n) < 1 ? 1 : (256 / n); }

template <int N>
__device__ __forceinline__ int perm_ct(int t) {
    int pos = 0, len = N;
#pragma unroll
    for (int f = 0; f < nrad(N); f++) {
        const int r = rad(N, f);
        len /= r;
        pos += (t % r) * len;
        t /= r;
    }
    return pos;
}

template <typename C>
__device__ __forceinline__ C twc(C w, int sign) {
    if (sign > 0) w.y = -w.y;
    return w;
}

// Line geometry: line l starts at base(l), element e at off(e).
template <int NL_, int INNER, int PS, int ES, bool PAD, bool LINE_FAST_>
struct Lines {
    static constexpr int NL = NL_;
    static constexpr bool LINE_FAST = LINE_FAST_;
    __device__ __forceinline__ static int base(int l) { return INNER == 1 ? l * PS : (l % INNER) + (l / INNER) * PS; }
    __device__ __forceinline__ static int off(int e) { return PAD ? e + (e >> 3) : e * ES; }
};

template <class LN, int N, int S, bool DIT, typename C>
__device__ __forceinline__ void stage(C *buf, const C *stw, int sign, int tid, int nthr) {
    constexpr int NF = nrad(N);
    constexpr int R = rad(N, NF - 1 - S);
    constexpr int M = span_inner(N, S);
    constexpr int L = M * R;
    constexpr int NBF = N / R;
    constexpr int TOT = LN::NL * NBF;
    constexpr int OFF = stw_offset(N, S);
    for (int t = tid; t < TOT; t += nthr) {
        int l, b;
        if (LN::LINE_FAST) {
            l = t % LN::NL;
            b = t / LN::NL;
        } else {
            b = t % NBF;
            l = t / NBF;
        }
        const int blk = b / M, k1 = b - blk * M;
        const int p0 = blk * L + k1;
        C *lp = buf + LN::base(l);
        C a[R];
#pragma unroll
        for (int j = 0; j < R; j++) a[j] = lp[LN::off(p0 + j * M)];
        if (DIT && M > 1) {
#pragma unroll
            for (int j = 1; j < R; j++) a[j] = cmul(a[j], twc(stw[OFF + (j - 1) * M + k1], sign));
        }
        SmallDFT<R, C>::run(a, sign, nullptr, 0);
        if (!DIT && M > 1) {
#pragma unroll
            for (int k = 1; k < R; k++) a[k] = cmul(a[k], twc(stw[OFF + (k - 1) * M + k1], sign));
        }
#pragma unroll
        for (int k = 0; k < R; k++) lp[LN::off(p0 + k * M)] = a[k];
    }
}

template <class LN, int N, bool BS, int S = 0, typename C>
__device__ __forceinline__ void dit(C *buf, const C *stw, int sign, int tid, int nthr) {
    if constexpr (S < nrad(N)) {
        stage<LN, N, S, true>(buf, stw, sign, tid, nthr);
        if (BS) __syncthreads(); else __syncwarp();
        dit<LN, N, BS, S + 1>(buf, stw, sign, tid, nthr);
    }
}
template <class LN, int N, bool BS, int S = nrad(N) - 1, typename C>
__device__ __forceinline__ void dif(C *buf, const C *stw, int sign, int tid, int nthr) {
    if constexpr (S >= 0) {
        stage<LN, N, S, false>(buf, stw, sign, tid, nthr);
        if (BS) __syncthreads(); else __syncwarp();
        dif<LN, N, BS, S - 1>(buf, stw, sign, tid, nthr);
    }
}

// shared-memory layout of the fast plane kernels
template <typename C, int N, int NBR, int NZL, int NT = NTHR>
struct FSmem {
    static constexpr int NZC = N / 2 + 1;
    static constexpr int PL = padded(N);
    static constexpr int ZB = zlines(N);
    static constexpr size_t P_ELEMS = (size_t)NBR * N * NZC;
    static constexpr size_t Z_ELEMS = (size_t)NZL * (NT / 32) * ZB * PL;
    static constexpr size_t BYTES = sizeof(C) * (P_ELEMS + Z_ELEMS + stw_size(N) + 1);
};

template <typename C, int N, int NT = NTHR>
__device__ __forceinline__ void load_stw(C *dst, const void *src) {
    for (int i = threadIdx.x; i < stw_size(N); i += NT) dst[i] = ((const C *)src)[i];
}

// ------------------------------------------------------------------------
// K1 (fast): forward zy transform of one x-plane
template <typename T, int NBR, int N, int NT = NTHR>
__global__ void __launch_bounds__(NT) kf_plane_forward(GridPlan g, const lfts_step_job *__restrict__ jobs, int s,
                                                         int fm0, int fm1, int spec_out0) {
    using C = typename CT<T>::type;
    using SM = FSmem<C, N, NBR, 1, NT>;
    constexpr int NZC = SM::NZC, PL = SM::PL, ZB = SM::ZB, NU = (NBR == 2) ? N : N / 2;
    using LZ = Lines<ZB, 1, PL, 1, true, false>;
    using LY = Lines<NBR * NZC, NZC, N * NZC, NZC, false, true>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *P = (C *)smem_raw;
    C *zl = P + SM::P_ELEMS;
    C *stw = zl + SM::Z_ELEMS;
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    load_stw<C, N, NT>(stw, g.stw);
    const long long poff = (long long)x * N * N;
    const T *qin = (const T *)jb.in + s * jb.in_stride + poff;
    const T *fac = (const T *)jb.fac + poff;
    C *zw = zl + warp * ZB * PL;
    for (int u0 = warp * ZB; u0 < NU; u0 += (NT / 32) * ZB) {
        constexpr int PER = (N + 31) / 32;
        T qa[ZB][PER], qb[ZB][PER], fa[ZB][PER], fb[ZB][PER];
#pragma unroll
        for (int b = 0; b < ZB; b++) {
            const int u = u0 + b;
            const int ya = (NBR == 2) ? u : 2 * u, yb = (NBR == 2) ? u : 2 * u + 1;
#pragma unroll
            for (int i = 0; i < PER; i++) {
                const int t = lane + 32 * i;
                if (u < NU && t < N) {
                    qa[b][i] = qin[ya * N + t];
                    fa[b][i] = fm0 == FM_NONE ? (T)1 : fac[ya * N + t];
                    if (NBR == 1) {
                        qb[b][i] = qin[yb * N + t];
                        fb[b][i] = fm0 == FM_NONE ? (T)1 : fac[yb * N + t];
                    }
                }
            }
        }
#pragma unroll
        for (int b = 0; b < ZB; b++) {
#pragma unroll
            for (int i = 0; i < PER; i++) {
                const int t = lane + 32 * i;
                if (u0 + b < NU && t < N) {
                    C z;
                    if (NBR == 2) {
                        const T f0 = fm0 == FM_FAC_SQ ? fa[b][i] * fa[b][i] : fa[b][i];
                        const T f1 = fm1 == FM_FAC_SQ ? fa[b][i] * fa[b][i] : (fm1 == FM_NONE ? (T)1 : fa[b][i]);
                        z.x = qa[b][i] * f0;
                        z.y = qa[b][i] * f1;
                    } else {
                        const T f0 = fm0 == FM_FAC_SQ ? fa[b][i] * fa[b][i] : fa[b][i];
                        const T f1 = fm0 == FM_FAC_SQ ? fb[b][i] * fb[b][i] : fb[b][i];
                        z.x = qa[b][i] * f0;
                        z.y = qb[b][i] * f1;
                    }
                    zw[b * PL + LZ::off(perm_ct<N>(t))] = z;
                }
            }
        }
        __syncwarp();
        dit<LZ, N, false>(zw, stw, -1, lane, 32);
#pragma unroll
        for (int b = 0; b < ZB; b++) {
            const int u = u0 + b;
            if (u >= NU) break;
            const int ya = (NBR == 2) ? u : 2 * u, yb = (NBR == 2) ? u : 2 * u + 1;
            C *rowA = P + perm_ct<N>(ya) * NZC;
            C *rowB = P + (NBR == 2 ? N * NZC : 0) + perm_ct<N>(yb) * NZC;
            const C *z = zw + b * PL;
            for (int k = lane; k < NZC; k += 32) {
                C A, B;
                split_pair(z[LZ::off(k)], cconj(z[LZ::off(k == 0 ? 0 : N - k)]), A, B);
                rowA[k] = A;
                rowB[k] = B;
            }
        }
        __syncwarp();
    }
    __syncthreads();
    dit<LY, N, true>(P, stw, -1, tid, NT);
#pragma unroll
    for (int b = 0; b < NBR; b++) {
        C *out = (C *)jb.spec + (size_t)(spec_out0 + b) * g.Mc + (size_t)x * N * NZC;
        const C *src = P + b * N * NZC;
        for (int i = tid; i < N * NZC; i += NT) out[i] = src[i];
    }
}

// ------------------------------------------------------------------------
// K2/K4 (fast): x-transform of TJ columns, bond multiply, inverse
template <typename T, int NBR, int N>
__global__ void __launch_bounds__(NTHR) kf_xpass(GridPlan g, const lfts_step_job *__restrict__ jobs, int spec_in0,
                                                 int bsel0, int bsel1) {
    using C = typename CT<T>::type;
    constexpr int TJ = sizeof(T) == 8 ? 16 : 32;
    constexpr int NZC = N / 2 + 1;
    constexpr long long PLANE = (long long)N * NZC;
    using LX = Lines<NBR * TJ, TJ, N * TJ, TJ, false, true>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tile = (C *)smem_raw;
    C *stw = tile + NBR * N * TJ;
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int tid = threadIdx.x;
    load_stw<C, N>(stw, g.stw);
    const long long j0 = (long long)blockIdx.x * TJ;
    const C *spec = (const C *)jb.spec;
    constexpr int TOT = NBR * N * TJ;
#pragma unroll 4
    for (int i = tid; i < TOT; i += NTHR) {
        const int jj = i % TJ, xr = (i / TJ) % N, b = i / (TJ * N);
        C v = cmk<C>(0, 0);
        if (j0 + jj < PLANE) v = spec[(size_t)(spec_in0 + b) * g.Mc + xr * PLANE + j0 + jj];
        tile[(b * N + perm_ct<N>(xr)) * TJ + jj] = v;
    }
    __syncthreads();
    dit<LX, N, true>(tile, stw, -1, tid, NTHR);
    const T *bt0 = (const T *)(bsel0 ? jb.bond_half : jb.bond);
    const T *bt1 = (const T *)(bsel1 ? jb.bond_half : jb.bond);
    for (int i = tid; i < TOT; i += NTHR) {
        const int jj = i % TJ, xr = (i / TJ) % N, b = i / (TJ * N);
        if (j0 + jj < PLANE) {
            const T bv = (b == 0 ? bt0 : bt1)[xr * PLANE + j0 + jj];
            C &v = tile[(b * N + xr) * TJ + jj];
            v.x *= bv;
            v.y *= bv;
        }
    }
    __syncthreads();
    dif<LX, N, true>(tile, stw, +1, tid, NTHR);
    C *specw = (C *)jb.spec;
    for (int i = tid; i < TOT; i += NTHR) {
        const int jj = i % TJ, xr = (i / TJ) % N, b = i / (TJ * N);
        if (j0 + jj < PLANE) specw[(size_t)(spec_in0 + b) * g.Mc + xr * PLANE + j0 + jj] = tile[(b * N + perm_ct<N>(xr)) * TJ + jj];
    }
}

// load NBR spectra planes and run the inverse y transform (rows end at perm positions)
template <typename C, int N, int NBR, int NT>
__device__ __forceinline__ void fload_inverse_y(const GridPlan &g, const lfts_step_job &jb, int spec_in0, C *P, const C *stw) {
    constexpr int NZC = N / 2 + 1;
    using LY = Lines<NBR * NZC, NZC, N * NZC, NZC, false, true>;
#pragma unroll
    for (int b = 0; b < NBR; b++) {
        const C *src = (const C *)jb.spec + (size_t)(spec_in0 + b) * g.Mc + (size_t)blockIdx.x * N * NZC;
        C *dst = P + b * N * NZC;
#pragma unroll 4
        for (int i = threadIdx.x; i < N * NZC; i += NT) dst[i] = src[i];
    }
    __syncthreads();
    dif<LY, N, true>(P, stw, +1, threadIdx.x, NT);
}

// ------------------------------------------------------------------------
// K3 (fast): inverse zy, multiply by e = fac^2, forward zy, in place on a spectrum slot
template <typename T, int N, int NT = NTHR>
__global__ void __launch_bounds__(NT) kf_plane_mid(GridPlan g, const lfts_step_job *__restrict__ jobs, int spec_idx) {
    using C = typename CT<T>::type;
    using SM = FSmem<C, N, 1, 1, NT>;
    constexpr int NZC = SM::NZC, PL = SM::PL, ZB = SM::ZB, NU = N / 2;
    using LZ = Lines<ZB, 1, PL, 1, true, false>;
    using LY = Lines<NZC, NZC, N * NZC, NZC, false, true>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *P = (C *)smem_raw;
    C *zl = P + SM::P_ELEMS;
    C *stw = zl + SM::Z_ELEMS;
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    load_stw<C, N, NT>(stw, g.stw);
    __syncthreads();
    fload_inverse_y<C, N, 1, NT>(g, jb, spec_idx, P, stw);
    const T *fac = (const T *)jb.fac + (long long)x * N * N;
    C *zw = zl + warp * ZB * PL;
    constexpr int PER = (N + 31) / 32;
    for (int u0 = warp * ZB; u0 < NU; u0 += (NT / 32) * ZB) {
        T ea[ZB][PER], eb[ZB][PER];
#pragma unroll
        for (int b = 0; b < ZB; b++) {
            const int ya = 2 * (u0 + b);
#pragma unroll
            for (int i = 0; i < PER; i++) {
                const int t = lane + 32 * i;
                if (u0 + b < NU && t < N) {
                    ea[b][i] = fac[ya * N + t];
                    eb[b][i] = fac[(ya + 1) * N + t];
                }
            }
        }
#pragma unroll
        for (int b = 0; b < ZB; b++) {
            if (u0 + b >= NU) break;
            const int ya = 2 * (u0 + b);
            const C *rowA = P + perm_ct<N>(ya) * NZC, *rowB = P + perm_ct<N>(ya + 1) * NZC;
            for (int k = lane; k < N; k += 32) zw[b * PL + LZ::off(perm_ct<N>(k))] = pack_pair(rowA, rowB, k, N, NZC);
        }
        __syncwarp();
        dit<LZ, N, false>(zw, stw, +1, lane, 32);
#pragma unroll
        for (int b = 0; b < ZB; b++) {
            if (u0 + b >= NU) break;
            C v[PER];
#pragma unroll
            for (int i = 0; i < PER; i++) {
                const int t = lane + 32 * i;
                if (t < N) {
                    const C z = zw[b * PL + LZ::off(t)];
                    v[i].x = z.x * ea[b][i] * ea[b][i];
                    v[i].y = z.y * eb[b][i] * eb[b][i];
                }
            }
            __syncwarp();
#pragma unroll
            for (int i = 0; i < PER; i++) {
                const int t = lane + 32 * i;
                if (t < N) zw[b * PL + LZ::off(perm_ct<N>(t))] = v[i];
            }
        }
        __syncwarp();
        dit<LZ, N, false>(zw, stw, -1, lane, 32);
#pragma unroll
        for (int b = 0; b < ZB; b++) {
            if (u0 + b >= NU) break;
            const int ya = 2 * (u0 + b);
            C *rowA = P + perm_ct<N>(ya) * NZC, *rowB = P + perm_ct<N>(ya + 1) * NZC;
            const C *z = zw + b * PL;
            for (int k = lane; k < NZC; k += 32) {
                C A, B;
                split_pair(z[LZ::off(k)], cconj(z[LZ::off(k == 0 ? 0 : N - k)]), A, B);
                rowA[k] = A;
                rowB[k] = B;
            }
        }
        __syncwarp();
    }
    __syncthreads();
    dit<LY, N, true>(P, stw, -1, tid, NT);
    C *out = (C *)jb.spec + (size_t)spec_idx * g.Mc + (size_t)x * N * NZC;
    for (int i = tid; i < N * NZC; i += NT) out[i] = P[i];
}

// ------------------------------------------------------------------------
// K5 (fast): inverse zy of NBR planes with the step epilogue (see k_plane_inverse)
template <typename T, int NBR, int EPI, int N, int NT = NTHR>
__global__ void __launch_bounds__(NT) kf_plane_inverse(GridPlan g, const lfts_step_job *__restrict__ jobs, int s,
                                                         int spec_in0, int fm0) {
    using C = typename CT<T>::type;
    using SM = FSmem<C, N, NBR, 1, NT>;
    constexpr int NZC = SM::NZC, PL = SM::PL, ZB = SM::ZB, NU = (NBR == 2) ? N : N / 2;
    using LZ = Lines<ZB, 1, PL, 1, true, false>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *P = (C *)smem_raw;
    C *zl = P + SM::P_ELEMS;
    C *stw = zl + SM::Z_ELEMS;
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    load_stw<C, N, NT>(stw, g.stw);
    __syncthreads();
    fload_inverse_y<C, N, NBR, NT>(g, jb, spec_in0, P, stw);
    const long long poff = (long long)x * N * N;
    const T *fac = (const T *)jb.fac + poff;
    T *qout = (T *)jb.out + s * jb.out_stride + poff;
    C *zw = zl + warp * ZB * PL;
    constexpr int PER = (N + 31) / 32;
    for (int u0 = warp * ZB; u0 < NU; u0 += (NT / 32) * ZB) {
        T fa[ZB][PER], fb[ZB][PER], qa[ZB][PER], qb[ZB][PER];
#pragma unroll
        for (int b = 0; b < ZB; b++) {
            const int u = u0 + b;
            const int ya = (NBR == 2) ? u : 2 * u;
#pragma unroll
            for (int i = 0; i < PER; i++) {
                const int t = lane + 32 * i;
                if (u < NU && t < N) {
                    if (EPI != EPI_SCALE || fm0 != FM_NONE) fa[b][i] = fac[ya * N + t];
                    if (NBR == 1 && (EPI != EPI_SCALE || fm0 != FM_NONE)) fb[b][i] = fac[(ya + 1) * N + t];
                    if (EPI == EPI_RICH_ACC) {
                        qa[b][i] = qout[ya * N + t];
                        qb[b][i] = qout[(ya + 1) * N + t];
                    }
                }
            }
        }
#pragma unroll
        for (int b = 0; b < ZB; b++) {
            const int u = u0 + b;
            if (u >= NU) break;
            const int ya = (NBR == 2) ? u : 2 * u, yb = (NBR == 2) ? u : 2 * u + 1;
            const C *rowA = P + perm_ct<N>(ya) * NZC;
            const C *rowB = (NBR == 2) ? P + N * NZC + perm_ct<N>(ya) * NZC : P + perm_ct<N>(yb) * NZC;
            for (int k = lane; k < N; k += 32) zw[b * PL + LZ::off(perm_ct<N>(k))] = pack_pair(rowA, rowB, k, N, NZC);
        }
        __syncwarp();
        dit<LZ, N, false>(zw, stw, +1, lane, 32);
#pragma unroll
        for (int b = 0; b < ZB; b++) {
            const int u = u0 + b;
            if (u >= NU) break;
            const int ya = (NBR == 2) ? u : 2 * u;
#pragma unroll
            for (int i = 0; i < PER; i++) {
                const int t = lane + 32 * i;
                if (t >= N) continue;
                const C z = zw[b * PL + LZ::off(t)];
                if (EPI == EPI_RICH) {
                    const T eh = fa[b][i];
                    qout[ya * N + t] = ((T)4 * eh * z.y - eh * eh * z.x) / (T)3;
                } else if (EPI == EPI_RICH_ACC) {
                    qout[ya * N + t] = ((T)4 * fa[b][i] * z.x - qa[b][i]) / (T)3;
                    qout[(ya + 1) * N + t] = ((T)4 * fb[b][i] * z.y - qb[b][i]) / (T)3;
                } else {
                    const T f0 = fm0 == FM_NONE ? (T)1 : (fm0 == FM_FAC_SQ ? fa[b][i] * fa[b][i] : fa[b][i]);
                    const T f1 = fm0 == FM_NONE ? (T)1 : (fm0 == FM_FAC_SQ ? fb[b][i] * fb[b][i] : fb[b][i]);
                    qout[ya * N + t] = z.x * f0;
                    qout[(ya + 1) * N + t] = z.y * f1;
                }
            }
        }
        __syncwarp();
    }
}

}  // namespace fast
}  // namespace lfts
