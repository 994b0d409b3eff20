// 64^3 plane kernels with bulk-copy staging (K1, K3, K5 of the step).
//
// Same transforms as the kr_* plane kernels of lfts_step_r8.cuh, with two
// changes that take the global-memory latency and the second task round off
// the critical path:
//   * all HBM traffic of a plane moves by cp.async.bulk: q / fac rows into the
//     plane rows, spectrum planes as one dense 64 x 33 copy, results back the
//     same way; the kernel computes from shared memory only;
//   * the DC (kz = 0) and Nyquist (kz = 32) y-columns are real sequences in y,
//     so they travel as one complex column a + i b (a Hermitian split at the
//     end recovers both): 32 y-tasks for 32 lane groups, one round.
//
// Shared-memory map (bytes, FP64 / FP32):
//   P       plane rows, stride PRB complex (73 / 74), z-lines at e + e/8;
//   stage   dense spectrum planes [ky][kz] at the start of P (phases that
//           read or write whole spectrum planes);
//   fstage  fac / q' rows, stride FS = 72 reals: at the end of P (K3, K5
//           NBR=1: disjoint from P rows 0..31 and from one dense plane) or
//           after P (K5 NBR=2, whose two input planes fill P).
#pragma once
#include "lfts_step_r8.cuh"

namespace lfts {
namespace r8 {

template <typename C> struct BGeo {
    using T = decltype(C::x);
    static constexpr int PRB = sizeof(C) == 16 ? 73 : 74;  // rows 16-byte aligned, columns conflict-free
    static constexpr int FS = 72;                          // staged real rows: 4 rows of a warp hit 2 bank halves
    static constexpr size_t P_BYTES = sizeof(C) * (size_t)N * PRB;
    static constexpr size_t F_BYTES = sizeof(T) * (size_t)N * FS;
    static constexpr size_t F_END = P_BYTES - F_BYTES;  // fac stage at the end of P
    static_assert(F_END % 16 == 0, "fac stage 16-byte aligned");
    static_assert(F_END >= sizeof(C) * (size_t)(N / 2) * PRB, "fac stage clear of z-lines 0..31");
    static_assert(F_END >= sizeof(C) * (size_t)PLANE, "fac stage clear of one dense spectrum plane");
    static_assert(2 * sizeof(C) * (size_t)PLANE <= P_BYTES, "two dense spectrum planes fit in P");
    static_assert((sizeof(C) * PRB) % 16 == 0, "plane rows 16-byte aligned");
};

template <typename C> constexpr size_t kb_plane_smem(bool fac_after) {
    return BGeo<C>::P_BYTES + (fac_after ? BGeo<C>::F_BYTES : 0) + 16;
}

// row owned by group g of warp w in round r (two rounds cover rows 0..63):
// rows 8w + 2r + {0, 4, 1, 5}, so the four 64-byte row reads of a warp fall
// into two full bank sets.
__device__ __forceinline__ int row_of(int w, int g, int r) { return 8 * w + 2 * r + (g >> 1) + 4 * (g & 1); }
// z-line (0..31) owned by group g of warp w, same bank property
__device__ __forceinline__ int line_of(int w, int g) { return 8 * (w & 3) + 2 * (w >> 2) + (g >> 1) + 4 * (g & 1); }

// Issue the bulk loads of one CTA (warp 0): n row copies described by the
// caller, all completing on bar.  expect = total bytes.
#define LFTS_BULK_ISSUE(expect, ...)                             \
    if (w == 0) {                                                \
        if (lane == 0) mbar_arrive_expect_tx(bar, (expect));     \
        __syncwarp();                                            \
        __VA_ARGS__                                              \
    }

// inverse y-transform of task kz's column(s) of a dense staged plane st,
// exchanging in its own staging column
template <typename C>
__device__ __forceinline__ void yinv_task(C *st, int kz, int j, C wi, unsigned mask, C (&c)[8]) {
    get_columns(st, kz, c, j);
    __syncwarp(mask);
    fft64<+1>(c, ColX<C, NZC>{st + kz}, j, wi, mask);
}

// ------------------------------------------------------------------------
// K1: forward zy transform of one x-plane (see kr_plane_forward)
template <typename T, int NBR>
__global__ void __launch_bounds__(NTHR, 2) kb_plane_forward(GridPlan g, const lfts_step_job *__restrict__ jobs, int s,
                                                            int fm0, int fm1, int spec_out0) {
    using C = typename CT<T>::type;
    using G = BGeo<C>;
    constexpr int S = G::PRB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *P = (C *)smem_raw;
    uint64_t *bar = (uint64_t *)(smem_raw + G::P_BYTES);
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5, gw = (tid >> 3) & 3, j = lane & 7;
    const int grp = tid >> 3;
    const unsigned mask = 0xFFu << (lane & 24);
    const long long poff = (long long)x * N * N;
    const T *qin = (const T *)jb.in + s * jb.in_stride + poff;
    const T *fac = (const T *)jb.fac + poff;
    const bool wfac = fm0 != FM_NONE || (NBR == 2 && fm1 != FM_NONE);
    C *out = (C *)jb.spec + (size_t)spec_out0 * g.Mc + (size_t)x * PLANE;
    if (((uintptr_t)qin | (wfac ? (uintptr_t)fac : 0) | (uintptr_t)out | (uintptr_t)g.Mc * sizeof(C)) & 15) {
        if (tid == 0) kerr_set(KERR_MISALIGNED);
        return;
    }
    if (tid == 0) mbar_init(bar, 1);
    __syncthreads();
    // q row y -> bytes [0, 64 s) of plane row y, fac row y -> [64 s, 128 s)
    constexpr uint32_t RB = N * sizeof(T);
    LFTS_BULK_ISSUE(N * RB * (wfac ? 2u : 1u), for (int r = lane; r < N; r += 32) {
        bulk_load(P + r * S, qin + r * N, RB, bar);
        if (wfac) bulk_load((T *)(P + r * S) + N, fac + r * N, RB, bar);
    })
    if (!mbar_wait(bar, 0)) {
        mbar_wait(bar, 0);
        return;
    }
    const C wf = tw_base<C>(j, -1);
    if (NBR == 2) {
#pragma unroll 1
        for (int r = 0; r < 2; r++) {
            const int y = row_of(w, gw, r);
            const T *row = (const T *)(P + y * S);
            C a[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const T q = row[j + 8 * m], f = wfac ? row[N + j + 8 * m] : (T)1;
                const T f0 = fm0 == FM_FAC_SQ ? f * f : (fm0 == FM_NONE ? (T)1 : f);
                const T f1 = fm1 == FM_FAC_SQ ? f * f : (fm1 == FM_NONE ? (T)1 : f);
                a[m].x = q * f0;
                a[m].y = q * f1;
            }
            __syncwarp(mask);
            fft64<-1>(a, RowX<C>{P + y * S}, j, wf, mask);
#pragma unroll
            for (int k = 0; k < 8; k++) P[y * S + 9 * k + j] = a[k];
        }
        __syncthreads();
        // y-columns: task kz (kz = 0: merged DC / Nyquist) splits the branches
        const int kz = grp;
        C A[8], B[8];
        if (kz != 0) {
            const int kc = N - kz;
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const int y = j + 8 * m;
                split_pair(P[y * S + xpad(kz)], cconj(P[y * S + xpad(kc)]), A[m], B[m]);
            }
        } else {
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const int y = j + 8 * m;
                const C z0 = P[y * S], z32 = P[y * S + xpad(N / 2)];
                A[m].x = z0.x;  // branch 0 at kz = 0 + i branch 0 at kz = 32
                A[m].y = z32.x;
                B[m].x = z0.y;
                B[m].y = z32.y;
            }
        }
        __syncwarp(mask);
        fft64<-1>(A, ColX<C, S>{P + xpad(kz)}, j, wf, mask);
        fft64<-1>(B, ColX<C, S>{P + xpad(kz == 0 ? N / 2 : N - kz)}, j, wf, mask);
        __syncthreads();
        put_columns(P, kz, A, j, lane, mask);
        put_columns(P + PLANE, kz, B, j, lane, mask);
    } else {
        {
            const int u = line_of(w, gw);
            const T *ra = (const T *)(P + u * S), *rb = (const T *)(P + (u + 32) * S);
            C a[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                a[m].x = ra[j + 8 * m] * fmul_mode(fm0, wfac ? ra[N + j + 8 * m] : (T)1);
                a[m].y = rb[j + 8 * m] * fmul_mode(fm0, wfac ? rb[N + j + 8 * m] : (T)1);
            }
            __syncwarp(mask);
            fft64<-1>(a, RowX<C>{P + u * S}, j, wf, mask);
#pragma unroll
            for (int k = 0; k < 8; k++) P[u * S + 9 * k + j] = a[k];
        }
        __syncthreads();
        C c[8];
        yfwd_paired_task<C, S>(P, grp, j, wf, mask, c);
        __syncthreads();
        put_columns(P, grp, c, j, lane, mask);
    }
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
        for (int b = 0; b < NBR; b++) bulk_store(out + (size_t)b * g.Mc, P + b * PLANE, PLANE * sizeof(C));
        bulk_commit();
        bulk_wait_read();
    }
}

// ------------------------------------------------------------------------
// K3: inverse zy, multiply by e = fac^2, forward zy, in place on slot spec_idx
template <typename T>
__global__ void __launch_bounds__(NTHR, 2) kb_plane_mid(GridPlan g, const lfts_step_job *__restrict__ jobs, int spec_idx) {
    using C = typename CT<T>::type;
    using G = BGeo<C>;
    constexpr int S = G::PRB, FS = G::FS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *P = (C *)smem_raw;
    T *fst = (T *)(smem_raw + G::F_END);
    uint64_t *bar = (uint64_t *)(smem_raw + G::P_BYTES);
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5, gw = (tid >> 3) & 3, j = lane & 7;
    const int grp = tid >> 3;
    const unsigned mask = 0xFFu << (lane & 24);
    C *sp = (C *)jb.spec + (size_t)spec_idx * g.Mc + (size_t)x * PLANE;
    const T *fac = (const T *)jb.fac + (long long)x * N * N;
    if (((uintptr_t)sp | (uintptr_t)fac) & 15) {
        if (tid == 0) kerr_set(KERR_MISALIGNED);
        return;
    }
    if (tid == 0) mbar_init(bar, 1);
    __syncthreads();
    constexpr uint32_t RB = N * sizeof(T);
    LFTS_BULK_ISSUE(PLANE * sizeof(C) + N * RB, {
        if (lane == 0) bulk_load(P, sp, PLANE * sizeof(C), bar);
        for (int r = lane; r < N; r += 32) bulk_load(fst + r * FS, fac + r * N, RB, bar);
    })
    if (!mbar_wait(bar, 0)) {
        mbar_wait(bar, 0);
        return;
    }
    const C wf = tw_base<C>(j, -1), wi = tw_base<C>(j, +1);
    {
        C c[8];
        yinv_task(P, grp, j, wi, mask, c);
        __syncthreads();
        put_zlines_paired<C, S>(P, grp, j, c);
    }
    __syncthreads();
    {
        const int u = line_of(w, gw);
        C a[8];
#pragma unroll
        for (int m = 0; m < 8; m++) a[m] = P[u * S + 9 * m + j];
        __syncwarp(mask);
        fft64<+1>(a, RowX<C>{P + u * S}, j, wi, mask);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const T ea = fst[u * FS + j + 8 * k], eb = fst[(u + 32) * FS + j + 8 * k];
            a[k].x = a[k].x * ea * ea;
            a[k].y = a[k].y * eb * eb;
        }
        fft64<-1>(a, RowX<C>{P + u * S}, j, wf, mask);
#pragma unroll
        for (int k = 0; k < 8; k++) P[u * S + 9 * k + j] = a[k];
    }
    __syncthreads();
    C c[8];
    yfwd_paired_task<C, S>(P, grp, j, wf, mask, c);
    __syncthreads();
    put_columns(P, grp, c, j, lane, mask);
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
        bulk_store(sp, P, PLANE * sizeof(C));
        bulk_commit();
        bulk_wait_read();
    }
}

// ------------------------------------------------------------------------
// K5: inverse zy with the step epilogue (see kr_plane_inverse)
template <typename T, int NBR, int EPI>
__global__ void __launch_bounds__(NTHR, 2) kb_plane_inverse(GridPlan g, const lfts_step_job *__restrict__ jobs, int s,
                                                            int spec_in0, int fm0) {
    static_assert((NBR == 2 && EPI == EPI_RICH) || (NBR == 1 && EPI == EPI_SCALE), "supported epilogues");
    using C = typename CT<T>::type;
    using G = BGeo<C>;
    constexpr int S = G::PRB, FS = G::FS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *P = (C *)smem_raw;
    T *fst = (T *)(smem_raw + (NBR == 2 ? G::P_BYTES : G::F_END));
    uint64_t *bar = (uint64_t *)(smem_raw + G::P_BYTES + (NBR == 2 ? G::F_BYTES : 0));
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5, gw = (tid >> 3) & 3, j = lane & 7;
    const int grp = tid >> 3;
    const unsigned mask = 0xFFu << (lane & 24);
    const C *in = (const C *)jb.spec + (size_t)spec_in0 * g.Mc + (size_t)x * PLANE;
    const long long poff = (long long)x * N * N;
    const T *fac = (const T *)jb.fac + poff;
    T *qout = (T *)jb.out + s * jb.out_stride + poff;
    const bool wfac = NBR == 2 || fm0 != FM_NONE;
    if (((uintptr_t)in | (uintptr_t)qout | (wfac ? (uintptr_t)fac : 0) | (uintptr_t)g.Mc * sizeof(C)) & 15) {
        if (tid == 0) kerr_set(KERR_MISALIGNED);
        return;
    }
    if (tid == 0) mbar_init(bar, 1);
    __syncthreads();
    constexpr uint32_t RB = N * sizeof(T);
    LFTS_BULK_ISSUE(NBR * PLANE * sizeof(C) + (wfac ? N * RB : 0u), {
        if (lane < NBR) bulk_load(P + lane * PLANE, in + (size_t)lane * g.Mc, PLANE * sizeof(C), bar);
        if (wfac)
            for (int r = lane; r < N; r += 32) bulk_load(fst + r * FS, fac + r * N, RB, bar);
    })
    if (!mbar_wait(bar, 0)) {
        mbar_wait(bar, 0);
        return;
    }
    const C wi = tw_base<C>(j, +1);
    if (NBR == 2) {
        const int kz = grp;
        C A[8], B[8];
        yinv_task(P, kz, j, wi, mask, A);
        yinv_task(P + PLANE, kz, j, wi, mask, B);
        __syncthreads();
        // z-lines: row y = j + 8k holds A + i B (Hermitian extension at 64 - kz)
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int y = j + 8 * k;
            C z;
            if (kz != 0) {
                z.x = A[k].x - B[k].y;
                z.y = A[k].y + B[k].x;
                P[y * S + xpad(kz)] = z;
                z.x = A[k].x + B[k].y;
                z.y = -A[k].y + B[k].x;
                P[y * S + xpad(N - kz)] = z;
            } else {
                z.x = A[k].x;  // A(kz=0) + i B(kz=0)
                z.y = B[k].x;
                P[y * S] = z;
                z.x = A[k].y;  // A(kz=32) + i B(kz=32)
                z.y = B[k].y;
                P[y * S + xpad(N / 2)] = z;
            }
        }
        __syncthreads();
#pragma unroll 1
        for (int r = 0; r < 2; r++) {
            const int y = row_of(w, gw, r);
            C a[8];
#pragma unroll
            for (int m = 0; m < 8; m++) a[m] = P[y * S + 9 * m + j];
            __syncwarp(mask);
            fft64<+1>(a, RowX<C>{P + y * S}, j, wi, mask);
#pragma unroll
            for (int k = 0; k < 8; k++) {
                T *f = fst + y * FS + j + 8 * k;
                const T eh = *f;
                *f = ((T)4 * eh * a[k].y - eh * eh * a[k].x) * (T)(1.0 / 3.0);
            }
        }
    } else {
        {
            C c[8];
            yinv_task(P, grp, j, wi, mask, c);
            __syncthreads();
            put_zlines_paired<C, S>(P, grp, j, c);
        }
        __syncthreads();
        const int u = line_of(w, gw);
        C a[8];
#pragma unroll
        for (int m = 0; m < 8; m++) a[m] = P[u * S + 9 * m + j];
        __syncwarp(mask);
        fft64<+1>(a, RowX<C>{P + u * S}, j, wi, mask);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            T *fa = fst + u * FS + j + 8 * k, *fb = fst + (u + 32) * FS + j + 8 * k;
            const T va = a[k].x * fmul_mode(fm0, wfac ? *fa : (T)1);
            const T vb = a[k].y * fmul_mode(fm0, wfac ? *fb : (T)1);
            *fa = va;
            *fb = vb;
        }
    }
    fence_proxy_async();
    __syncthreads();
    if (w == 0) {
        for (int r = lane; r < N; r += 32) bulk_store(qout + r * N, fst + r * FS, RB);
        bulk_commit();
        bulk_wait_read();
    }
}

#undef LFTS_BULK_ISSUE

}  // namespace r8
}  // namespace lfts
