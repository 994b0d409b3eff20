// Register-resident step kernels for 64^3 grids (64 = 8 x 8).
//
// The same five passes as lfts_step_fast.cuh, with the same spectra layout in
// HBM ([x][ky][kz], natural order), but every 64-point line transform is held
// by the 8 lanes of one lane group: lane j keeps elements j + 8m in registers,
// runs an 8-point DFT over m, applies the twiddle w64^(j k1), exchanges once
// through shared memory and runs an 8-point DFT over j.  A line therefore
// passes through shared memory once per transform instead of once per radix
// stage, which is what bounded the staged kernels (their shared-memory pipe
// ran at ~70 % while DRAM ran at ~1/3).
//
// Plane kernels keep one x-plane in shared memory, rows of PR = 73 complex
// (element e of a row at e + e/8, so row reads of eight consecutive elements
// and column reads of eight rows 73 apart are both free of bank conflicts).
// Exchanges run in place: a z-line in its own row, a y-column task in its own
// columns (kz and 64 - kz), with a skewed slot order down the column.
//
// Pairings used to halve the real transforms:
//   * two branches of one row (continuous K1/K5): z = q (f0 + i f1);
//   * rows y and y + 32 (K3, discrete K1/K5): lane j of a y-task holds rows
//     j + 8m, so rows y and y + 32 of the same kz sit in the same lane.
#pragma once
#include "lfts_step_kernels.cuh"

namespace lfts {
namespace r8 {

constexpr int N = 64, NZC = N / 2 + 1, PLANE = N * NZC;
constexpr int PR = 73;  // plane row stride (complex elements)
constexpr int XG = 72;  // exchange slots per lane group in the x-pass
constexpr int GROUPS = NTHR / 8;
static_assert(GROUPS == 32, "one lane group of 8 per 64-point line, 32 lines per CTA");
static_assert(PLANE % GROUPS == 0, "x-pass tiles cover the plane exactly");

template <typename C> constexpr size_t plane_smem() { return sizeof(C) * (size_t)N * PR; }
template <typename C> constexpr size_t xpass_smem() { return sizeof(C) * (size_t)GROUPS * XG; }

__device__ __forceinline__ int xpad(int e) { return e + (e >> 3); }

// w64^j = exp(sign * 2 pi i j / 64)
template <typename C>
__device__ __forceinline__ C tw_base(int j, int sign) {
    double sn, cs;
    sincospi((double)j / 32.0, &sn, &cs);
    C w;
    w.x = cs;
    w.y = sign * sn;
    return w;
}

// exchange slots along a row: element (k, j) at b + 9k + j
template <typename C> struct RowX {
    C *b;
    __device__ __forceinline__ C &ref(int k, int j) const { return b[9 * k + j]; }
};
// exchange slots down a plane column (row stride PR), skewed: (k, j) at row 8k + ((j + k) & 7)
template <typename C> struct ColS {
    C *b;
    __device__ __forceinline__ C &ref(int k, int j) const { return b[(8 * k + ((j + k) & 7)) * PR]; }
};

// One 64-point transform held by the 8 lanes of a group (mask = the group's
// lanes).  On entry lane j holds x[j + 8m] in a[m]; on exit lane t holds
// X[t + 8k] in a[k], X[k] = sum_n x[n] exp(SIGN 2 pi i n k / 64).
// w1 = tw_base(j, SIGN).
template <int SIGN, class AT, typename C>
__device__ __forceinline__ void fft64(C (&a)[8], const AT &at, int j, C w1, unsigned mask) {
    SmallDFT<8, C>::run(a, SIGN, nullptr, 0);
    C w = w1;
#pragma unroll
    for (int k = 1; k < 8; k++) {
        a[k] = cmul(a[k], w);
        if (k < 7) w = cmul(w, w1);
    }
#pragma unroll
    for (int k = 0; k < 8; k++) at.ref(k, j) = a[k];
    __syncwarp(mask);
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = at.ref(j, k);
    __syncwarp(mask);
    SmallDFT<8, C>::run(a, SIGN, nullptr, 0);
}

template <typename T>
__device__ __forceinline__ T fmul_mode(int mode, T f) {
    return mode == FM_NONE ? (T)1 : (mode == FM_FAC_SQ ? f * f : f);
}

// y-phase, forward, rows paired (y, y + 32): lines u = 0..31 of the plane hold
// Z_u = F_z[row u] + i F_z[row u + 32]; task kz splits them and transforms
// column kz over y, then stores it to out (column kz of one spectrum plane).
template <typename C>
__device__ __forceinline__ void y_forward_paired(C *P, int kz, int j, C wf, unsigned mask, C *out) {
    const int kc = (N - kz) & (N - 1);
    C a[8];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const int u = j + 8 * m;
        split_pair(P[u * PR + xpad(kz)], cconj(P[u * PR + xpad(kc)]), a[m], a[m + 4]);
    }
    __syncwarp(mask);
    fft64<-1>(a, ColS<C>{P + xpad(kz)}, j, wf, mask);
#pragma unroll
    for (int k = 0; k < 8; k++) out[(j + 8 * k) * NZC] = a[k];
}

// y-phase, inverse, rows paired (y, y + 32): column kz of one spectrum plane
// (in) is transformed over ky; lane j then holds rows j + 8k and packs rows
// u and u + 32 into the z-line u: Z_u[kz] = A_u + i A_{u+32} and, at 64 - kz,
// the Hermitian extension (imaginary parts of DC and Nyquist dropped).
template <typename C>
__device__ __forceinline__ void y_inverse_paired(C *P, int kz, int j, C wi, unsigned mask, const C *in) {
    const int kc = (N - kz) & (N - 1);
    C a[8];
#pragma unroll
    for (int m = 0; m < 8; m++) a[m] = in[(j + 8 * m) * NZC];
    fft64<+1>(a, ColS<C>{P + xpad(kz)}, j, wi, mask);
    if (kz == 0 || kz == N / 2) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k].y = 0;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int u = j + 8 * k;
        const C a0 = a[k], a1 = a[k + 4];
        C z;
        z.x = a0.x - a1.y;
        z.y = a0.y + a1.x;
        P[u * PR + xpad(kz)] = z;
        if (kc != kz) {
            z.x = a0.x + a1.y;
            z.y = -a0.y + a1.x;
            P[u * PR + xpad(kc)] = z;
        }
    }
}

// ------------------------------------------------------------------------
// K1: forward zy transform of one x-plane.
//   NBR = 2: spectra of f0(fac) q and f1(fac) q (slots spec_out0, +1);
//   NBR = 1: spectrum of f0(fac) q (slot spec_out0).
template <typename T, int NBR>
__global__ void __launch_bounds__(NTHR, 2) kr_plane_forward(GridPlan g, const lfts_step_job *__restrict__ jobs, int s,
                                                            int fm0, int fm1, int spec_out0) {
    using C = typename CT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *P = (C *)smem_raw;
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x, tid = threadIdx.x, lane = tid & 31, j = lane & 7, grp = tid >> 3;
    const unsigned mask = 0xFFu << (lane & 24);
    const C wf = tw_base<C>(j, -1);
    const long long poff = (long long)x * N * N;
    const T *qin = (const T *)jb.in + s * jb.in_stride + poff;
    const T *fac = (const T *)jb.fac + poff;
    C *out = (C *)jb.spec + (size_t)spec_out0 * g.Mc + (size_t)x * PLANE;
    if (NBR == 2) {
        // z-lines: row y, branches packed as real / imaginary part
        for (int y = grp; y < N; y += GROUPS) {
            T qv[8], fv[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                qv[m] = qin[y * N + j + 8 * m];
                fv[m] = fm0 == FM_NONE ? (T)1 : fac[y * N + j + 8 * m];
            }
            C a[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const T f0 = fm0 == FM_FAC_SQ ? fv[m] * fv[m] : fv[m];
                const T f1 = fm1 == FM_FAC_SQ ? fv[m] * fv[m] : (fm1 == FM_NONE ? (T)1 : fv[m]);
                a[m].x = qv[m] * f0;
                a[m].y = qv[m] * f1;
            }
            fft64<-1>(a, RowX<C>{P + y * PR}, j, wf, mask);
#pragma unroll
            for (int k = 0; k < 8; k++) P[y * PR + 9 * k + j] = a[k];
        }
        __syncthreads();
        // y-columns: task kz splits the branches and transforms both
        for (int kz = grp; kz <= N / 2; kz += GROUPS) {
            const int kc = (N - kz) & (N - 1);
            C A[8], B[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const int y = j + 8 * m;
                split_pair(P[y * PR + xpad(kz)], cconj(P[y * PR + xpad(kc)]), A[m], B[m]);
            }
            __syncwarp(mask);
            fft64<-1>(A, ColS<C>{P + xpad(kz)}, j, wf, mask);
            fft64<-1>(B, ColS<C>{P + xpad(kc)}, j, wf, mask);
            C *o0 = out + kz, *o1 = out + g.Mc + kz;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                o0[(j + 8 * k) * NZC] = A[k];
                o1[(j + 8 * k) * NZC] = B[k];
            }
        }
    } else {
        // z-lines: rows u and u + 32 packed as real / imaginary part
        {
            const int u = grp;
            T qa[8], qb[8], fa[8], fb[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                qa[m] = qin[u * N + j + 8 * m];
                qb[m] = qin[(u + 32) * N + j + 8 * m];
                fa[m] = fm0 == FM_NONE ? (T)1 : fac[u * N + j + 8 * m];
                fb[m] = fm0 == FM_NONE ? (T)1 : fac[(u + 32) * N + j + 8 * m];
            }
            C a[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                a[m].x = qa[m] * fmul_mode(fm0, fa[m]);
                a[m].y = qb[m] * fmul_mode(fm0, fb[m]);
            }
            fft64<-1>(a, RowX<C>{P + u * PR}, j, wf, mask);
#pragma unroll
            for (int k = 0; k < 8; k++) P[u * PR + 9 * k + j] = a[k];
        }
        __syncthreads();
        for (int kz = grp; kz <= N / 2; kz += GROUPS) y_forward_paired(P, kz, j, wf, mask, out + kz);
    }
}

// ------------------------------------------------------------------------
// K2 / K4: x-transform of 32 columns, bond multiply, inverse x-transform
template <typename T, int NBR>
__global__ void __launch_bounds__(NTHR, 2) kr_xpass(GridPlan g, const lfts_step_job *__restrict__ jobs, int spec_in0,
                                                 int bsel0, int bsel1) {
    using C = typename CT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int tid = threadIdx.x, lane = tid & 31, j = lane & 7, grp = tid >> 3;
    const unsigned mask = 0xFFu << (lane & 24);
    const C wf = tw_base<C>(j, -1), wi = tw_base<C>(j, +1);
    const RowX<C> at{(C *)smem_raw + grp * XG};
    const int col = blockIdx.x * GROUPS + grp;
    C *s0 = (C *)jb.spec + (size_t)spec_in0 * g.Mc + col;
    const T *bt0 = (const T *)(bsel0 ? jb.bond_half : jb.bond) + col;
    const T *bt1 = (const T *)(bsel1 ? jb.bond_half : jb.bond) + col;
#pragma unroll
    for (int b = 0; b < NBR; b++) {
        C *sb = s0 + (size_t)b * g.Mc;
        const T *bt = b == 0 ? bt0 : bt1;
        C a[8];
        T bv[8];
#pragma unroll
        for (int m = 0; m < 8; m++) a[m] = sb[(j + 8 * m) * PLANE];
#pragma unroll
        for (int k = 0; k < 8; k++) bv[k] = bt[(j + 8 * k) * PLANE];
        fft64<-1>(a, at, j, wf, mask);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            a[k].x *= bv[k];
            a[k].y *= bv[k];
        }
        fft64<+1>(a, at, j, wi, mask);
#pragma unroll
        for (int m = 0; m < 8; m++) sb[(j + 8 * m) * PLANE] = a[m];
    }
}

// ------------------------------------------------------------------------
// K3: inverse zy, multiply by e = fac^2, forward zy, in place on slot spec_idx
template <typename T>
__global__ void __launch_bounds__(NTHR, 2) kr_plane_mid(GridPlan g, const lfts_step_job *__restrict__ jobs, int spec_idx) {
    using C = typename CT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *P = (C *)smem_raw;
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x, tid = threadIdx.x, lane = tid & 31, j = lane & 7, grp = tid >> 3;
    const unsigned mask = 0xFFu << (lane & 24);
    const C wf = tw_base<C>(j, -1), wi = tw_base<C>(j, +1);
    C *sp = (C *)jb.spec + (size_t)spec_idx * g.Mc + (size_t)x * PLANE;
    const T *fac = (const T *)jb.fac + (long long)x * N * N;
    for (int kz = grp; kz <= N / 2; kz += GROUPS) y_inverse_paired(P, kz, j, wi, mask, sp + kz);
    __syncthreads();
    {
        const int u = grp;
        T ea[8], eb[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            ea[k] = fac[u * N + j + 8 * k];
            eb[k] = fac[(u + 32) * N + j + 8 * k];
        }
        C a[8];
#pragma unroll
        for (int m = 0; m < 8; m++) a[m] = P[u * PR + 9 * m + j];
        __syncwarp(mask);
        fft64<+1>(a, RowX<C>{P + u * PR}, j, wi, mask);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            a[k].x = a[k].x * ea[k] * ea[k];
            a[k].y = a[k].y * eb[k] * eb[k];
        }
        fft64<-1>(a, RowX<C>{P + u * PR}, j, wf, mask);
#pragma unroll
        for (int k = 0; k < 8; k++) P[u * PR + 9 * k + j] = a[k];
    }
    __syncthreads();
    for (int kz = grp; kz <= N / 2; kz += GROUPS) y_forward_paired(P, kz, j, wf, mask, sp + kz);
}

// ------------------------------------------------------------------------
// K5: inverse zy of NBR spectrum planes with the step epilogue.
//   NBR = 2, EPI_RICH: q' = (4 e_h v2 - e_h^2 v1) / 3 (v1 from slot spec_in0);
//   NBR = 1, EPI_SCALE: q' = f(fac) v.
template <typename T, int NBR, int EPI>
__global__ void __launch_bounds__(NTHR, 2) kr_plane_inverse(GridPlan g, const lfts_step_job *__restrict__ jobs, int s,
                                                            int spec_in0, int fm0) {
    static_assert((NBR == 2 && EPI == EPI_RICH) || (NBR == 1 && EPI == EPI_SCALE), "supported epilogues");
    using C = typename CT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *P = (C *)smem_raw;
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x, tid = threadIdx.x, lane = tid & 31, j = lane & 7, grp = tid >> 3;
    const unsigned mask = 0xFFu << (lane & 24);
    const C wi = tw_base<C>(j, +1);
    const C *in = (const C *)jb.spec + (size_t)spec_in0 * g.Mc + (size_t)x * PLANE;
    const long long poff = (long long)x * N * N;
    const T *fac = (const T *)jb.fac + poff;
    T *qout = (T *)jb.out + s * jb.out_stride + poff;
    if (NBR == 2) {
        for (int kz = grp; kz <= N / 2; kz += GROUPS) {
            const int kc = (N - kz) & (N - 1);
            C A[8], B[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                A[m] = in[(j + 8 * m) * NZC + kz];
                B[m] = in[g.Mc + (j + 8 * m) * NZC + kz];
            }
            fft64<+1>(A, ColS<C>{P + xpad(kz)}, j, wi, mask);
            fft64<+1>(B, ColS<C>{P + xpad(kc)}, j, wi, mask);
            if (kz == 0 || kz == N / 2) {
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    A[k].y = 0;
                    B[k].y = 0;
                }
            }
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int y = j + 8 * k;
                C z;
                z.x = A[k].x - B[k].y;
                z.y = A[k].y + B[k].x;
                P[y * PR + xpad(kz)] = z;
                if (kc != kz) {
                    z.x = A[k].x + B[k].y;
                    z.y = -A[k].y + B[k].x;
                    P[y * PR + xpad(kc)] = z;
                }
            }
        }
        __syncthreads();
        for (int y = grp; y < N; y += GROUPS) {
            T eh[8];
#pragma unroll
            for (int k = 0; k < 8; k++) eh[k] = fac[y * N + j + 8 * k];
            C a[8];
#pragma unroll
            for (int m = 0; m < 8; m++) a[m] = P[y * PR + 9 * m + j];
            __syncwarp(mask);
            fft64<+1>(a, RowX<C>{P + y * PR}, j, wi, mask);
#pragma unroll
            for (int k = 0; k < 8; k++) qout[y * N + j + 8 * k] = ((T)4 * eh[k] * a[k].y - eh[k] * eh[k] * a[k].x) / (T)3;
        }
    } else {
        for (int kz = grp; kz <= N / 2; kz += GROUPS) y_inverse_paired(P, kz, j, wi, mask, in + kz);
        __syncthreads();
        const int u = grp;
        T fa[8], fb[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            fa[k] = fm0 == FM_NONE ? (T)1 : fac[u * N + j + 8 * k];
            fb[k] = fm0 == FM_NONE ? (T)1 : fac[(u + 32) * N + j + 8 * k];
        }
        C a[8];
#pragma unroll
        for (int m = 0; m < 8; m++) a[m] = P[u * PR + 9 * m + j];
        __syncwarp(mask);
        fft64<+1>(a, RowX<C>{P + u * PR}, j, wi, mask);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            qout[u * N + j + 8 * k] = a[k].x * fmul_mode(fm0, fa[k]);
            qout[(u + 32) * N + j + 8 * k] = a[k].y * fmul_mode(fm0, fb[k]);
        }
    }
}

}  // namespace r8
}  // namespace lfts
