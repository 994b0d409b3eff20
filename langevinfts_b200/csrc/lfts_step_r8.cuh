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
// Plane kernels keep one x-plane in shared memory, 64 rows of 64 complex
// elements, in a layout chosen per element size (PlaneLayout) so that the
// row and column accesses of a warp are free of bank conflicts.  Exchanges
// run in place: a z-line in its own row, a y-column task in its own columns
// (kz and 64 - kz), with a skewed slot order down the column.
//
// Pairings used to halve the real transforms:
//   * two branches of one row (continuous K1/K5): z = q (f0 + i f1);
//   * rows y and y + 32 (K3, discrete K1/K5): lane j of a y-task holds rows
//     j + 8m, so rows y and y + 32 of the same kz sit in the same lane.
#pragma once
#include "lfts_step_kernels.cuh"
#include "lfts_bulk.cuh"

// resident CTAs per SM the plane kernels are compiled for (register budget)
#ifndef LFTS_R8_MINB
#define LFTS_R8_MINB 2
#endif
#ifndef LFTS_R8_MINB_F32
#define LFTS_R8_MINB_F32 4
#endif

namespace lfts {

namespace r8 {

constexpr int N = 64, NZC = N / 2 + 1, PLANE = N * NZC;
constexpr int GROUPS = NTHR / 8;
static_assert(GROUPS == 32, "one lane group of 8 per 64-point line, 32 lines per CTA");
static_assert(PLANE % GROUPS == 0, "x-pass tiles cover the plane exactly");

// Slot of element e (0..63) of row r of the plane in shared memory.  The
// accesses to serve: a row's lanes j write 8k + j and read 8j + k (fixed k;
// the four groups of a warp take four consecutive rows), and a column's lanes
// read rows j + 8m or 8k + ((j + k) & 7) (the four groups of a warp take four
// consecutive columns).
//   16-byte complex (FP64): a wavefront serves one lane group; rows of 73
//     with e at e + e/8 keep each group's eight slots in distinct banks.
//   8-byte complex (FP32): a wavefront serves two lane groups, so the two
//     must also avoid each other: rows of 64, e XOR 8 (row parity) XOR
//     (e / 8 mod 8) XOR (r AND 6).  Every pattern above then costs the
//     minimum two wavefronts per warp access (column kc of a y-task: 1.25x),
//     against 1.5-2x in the padded layout.
template <typename C> struct PlaneLayout;
template <> struct PlaneLayout<double2> {
    static constexpr int RS = 73;
    __device__ __forceinline__ static int at(int r, int e) { return r * RS + e + (e >> 3); }
};
template <> struct PlaneLayout<float2> {
    static constexpr int RS = 64;
    __device__ __forceinline__ static int at(int r, int e) { return r * RS + (e ^ ((r & 1) << 3) ^ ((e >> 3) & 7) ^ (r & 6)); }
};
template <typename C> __device__ __forceinline__ int at(int r, int e) { return PlaneLayout<C>::at(r, e); }
template <typename C> constexpr size_t plane_smem() { return sizeof(C) * (size_t)N * PlaneLayout<C>::RS; }

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

// exchange slots along row r of plane P: (k, j) at element 8k + j
template <typename C> struct RowX {
    C *P;
    int r;
    __device__ __forceinline__ C &ref(int k, int j) const { return P[at<C>(r, 8 * k + j)]; }
};
// exchange slots down column e of plane P, skewed: (k, j) at row
// 8k + ((j + k) & 7), so both the writes (fixed k) and the reads (fixed j) of
// a lane group touch eight different banks
template <typename C> struct ColS {
    C *P;
    int e;
    __device__ __forceinline__ C &ref(int k, int j) const { return P[at<C>(8 * k + ((j + k) & 7), e)]; }
};

// One 64-point transform held by the 8 lanes of a group (mask = the group's
// lanes).  On entry lane j holds x[j + 8m] in a[m]; on exit lane t holds
// X[t + 8k] in a[k], X[k] = sum_n x[n] exp(SIGN 2 pi i n k / 64).
// w1 = tw_base(j, SIGN).
// a[k] *= w1^k for k = 1..7; the powers come from a tree of depth 3
// (w2 = w1 w1, w3 = w2 w1, w4 = w2 w2, w5 = w4 w1, w6 = w3 w3, w7 = w4 w3),
// not a serial chain of six dependent multiplies
template <typename C>
__device__ __forceinline__ void twiddle8(C (&a)[8], C w1) {
    const C w2 = cmul(w1, w1);
    const C w3 = cmul(w2, w1), w4 = cmul(w2, w2);
    a[1] = cmul(a[1], w1);
    a[2] = cmul(a[2], w2);
    a[3] = cmul(a[3], w3);
    a[4] = cmul(a[4], w4);
    a[5] = cmul(a[5], cmul(w4, w1));
    a[6] = cmul(a[6], cmul(w3, w3));
    a[7] = cmul(a[7], cmul(w4, w3));
}

template <int SIGN, class AT, typename C>
__device__ __forceinline__ void fft64(C (&a)[8], const AT &at, int j, C w1, unsigned mask) {
    SmallDFT<8, C>::run(a, SIGN, nullptr, 0);
    twiddle8(a, w1);
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

// The y-phase has 32 tasks, one per lane group: task kz in 1..31 owns the
// columns kz and 64 - kz of the z-transformed plane, and task 0 owns the DC
// and Nyquist columns 0 and 32.  Those two are real sequences in y, so task 0
// carries them as one complex column c = a + i b.

// Lane t holds c[k] = C[t + 8k] with C = F[a] + i F[b] (a, b real sequences);
// p[k] = C[-(t + 8k) mod 64], fetched from lane (8 - t) & 7 of the group.
template <typename C>
__device__ __forceinline__ void herm_partner(const C (&c)[8], C (&p)[8], int t, int lane, unsigned mask) {
    const int src = (lane & 24) | ((8 - t) & 7);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        C v;
        v.x = __shfl_sync(mask, c[7 - k].x, src);
        v.y = __shfl_sync(mask, c[7 - k].y, src);
        p[k] = t == 0 ? c[(8 - k) & 7] : v;
    }
}

// After the forward y-transform: write task kz's column(s) (c[k] at ky = j + 8k)
// to a spectrum plane st ([ky][kz], row stride NZC; global or shared).  Task 0
// splits c = F[col0] + i F[col32] into the two columns.
template <typename C>
__device__ __forceinline__ void put_columns(C *st, int kz, const C (&c)[8], int j, int lane, unsigned mask) {
    if (kz != 0) {
        C *col = st + j * NZC + kz;  // rows j + 8k at constant offsets
#pragma unroll
        for (int k = 0; k < 8; k++) col[8 * k * NZC] = c[k];
    } else {
        C p[8];
        herm_partner(c, p, j, lane, mask);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            C a, b;
            split_pair(c[k], cconj(p[k]), a, b);
            C *row = st + (j + 8 * k) * NZC;
            row[0] = a;
            row[N / 2] = b;
        }
    }
}

// Read task kz's column(s) of a spectrum plane st for an inverse y-transform
// (task 0: c = col0 + i col32).
template <typename C>
__device__ __forceinline__ void get_columns(const C *st, int kz, C (&c)[8], int j) {
    if (kz != 0) {
        const C *col = st + j * NZC + kz;
#pragma unroll
        for (int m = 0; m < 8; m++) c[m] = col[8 * m * NZC];
    } else {
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const C *row = st + (j + 8 * m) * NZC;
            const C a = row[0], b = row[N / 2];
            c[m].x = a.x - b.y;
            c[m].y = a.y + b.x;
        }
    }
}

// y-phase forward on rows paired (u, u + 32): z-lines u = 0..31 of P hold
// Z_u = F_z[row u] + i F_z[row u + 32].  Task kz splits them, transforms over
// y and leaves the column(s) in c (lane j: ky = j + 8k).
template <typename C>
__device__ __forceinline__ void yfwd_paired_task(C *P, int kz, int j, C wf, unsigned mask, C (&c)[8]) {
    if (kz != 0) {
        const int kc = N - kz;
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const int u = j + 8 * m;
            split_pair(P[at<C>(u, kz)], cconj(P[at<C>(u, kc)]), c[m], c[m + 4]);
        }
    } else {
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const int u = j + 8 * m;
            const C z0 = P[at<C>(u, 0)], z32 = P[at<C>(u, N / 2)];
            c[m].x = z0.x;  // row u: DC + i Nyquist
            c[m].y = z32.x;
            c[m + 4].x = z0.y;  // row u + 32
            c[m + 4].y = z32.y;
        }
    }
    __syncwarp(mask);
    fft64<-1>(c, ColS<C>{P, kz}, j, wf, mask);
}

// Pack rows u, u + 32 (lane j holds rows j + 8k, k < 8) of the inverse
// y-transformed column(s) of task kz into the z-lines u of P (imaginary parts
// of DC and Nyquist dropped, Hermitian extension at 64 - kz).
template <typename C>
__device__ __forceinline__ void put_zlines_paired(C *P, int kz, int j, const C (&a)[8]) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int u = j + 8 * k;
        const C a0 = a[k], a1 = a[k + 4];
        C z;
        if (kz != 0) {
            z.x = a0.x - a1.y;
            z.y = a0.y + a1.x;
            P[at<C>(u, kz)] = z;
            z.x = a0.x + a1.y;
            z.y = -a0.y + a1.x;
            P[at<C>(u, N - kz)] = z;
        } else {
            z.x = a0.x;  // s0(u) + i s0(u + 32)
            z.y = a1.x;
            P[at<C>(u, 0)] = z;
            z.x = a0.y;  // s32(u) + i s32(u + 32)
            z.y = a1.y;
            P[at<C>(u, N / 2)] = z;
        }
    }
}

// y-phase forward, rows paired, column(s) stored to a global spectrum plane
template <typename C>
__device__ __forceinline__ void y_forward_paired(C *P, int kz, int j, int lane, C wf, unsigned mask, C *plane) {
    C a[8];
    yfwd_paired_task<C>(P, kz, j, wf, mask, a);
    put_columns(plane, kz, a, j, lane, mask);
}

// y-phase inverse, rows paired, from a global spectrum plane into z-lines
template <typename C>
__device__ __forceinline__ void y_inverse_paired(C *P, int kz, int j, C wi, unsigned mask, const C *plane) {
    C a[8];
    get_columns(plane, kz, a, j);
    fft64<+1>(a, ColS<C>{P, kz}, j, wi, mask);
    put_zlines_paired<C>(P, kz, j, a);
}

// ------------------------------------------------------------------------
// K1: forward zy transform of one x-plane.
//   NBR = 2: spectra of f0(fac) q and f1(fac) q (slots spec_out0, +1);
//   NBR = 1: spectrum of f0(fac) q (slot spec_out0).
// The factor modes are template arguments (FM0, FM1): the continuous step
// uses <2, FM_FAC_SQ, FM_FAC>, the discrete step <1, FM_NONE, FM_NONE>.
template <typename T, int NBR, int FM0, int FM1>
__global__ void __launch_bounds__(NTHR, (sizeof(T) == 4 ? LFTS_R8_MINB_F32 : LFTS_R8_MINB)) kr_plane_forward(GridPlan g, const lfts_step_job *__restrict__ jobs, int s,
                                                                       int spec_out0) {
    using C = typename CT<T>::type;
    constexpr int fm0 = FM0, fm1 = FM1;
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
            const T *qrow = qin + y * N + j, *frow = fac + y * N + j;  // elements j + 8m at constant offsets
            T qv[8], fv[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                qv[m] = qrow[8 * m];
                fv[m] = fm0 == FM_NONE ? (T)1 : frow[8 * m];
            }
            C a[8];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const T f0 = fm0 == FM_FAC_SQ ? fv[m] * fv[m] : fv[m];
                const T f1 = fm1 == FM_FAC_SQ ? fv[m] * fv[m] : (fm1 == FM_NONE ? (T)1 : fv[m]);
                a[m].x = qv[m] * f0;
                a[m].y = qv[m] * f1;
            }
            fft64<-1>(a, RowX<C>{P, y}, j, wf, mask);
#pragma unroll
            for (int k = 0; k < 8; k++) P[at<C>(y, 8 * k + j)] = a[k];
        }
        __syncthreads();
        // y-columns: task kz splits the branches; branch 1 waits in its own
        // column (ekc) while branch 0 is transformed and stored
        const int kz = grp, ekz = kz, ekc = kz == 0 ? N / 2 : N - kz;
        C A[8];
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const int y = j + 8 * m;
            const C zk = P[at<C>(y, ekz)], zc = P[at<C>(y, ekc)];
            C b;
            if (kz != 0) {
                split_pair(zk, cconj(zc), A[m], b);
            } else {
                A[m].x = zk.x;  // branch 0: DC + i Nyquist
                A[m].y = zc.x;
                b.x = zk.y;  // branch 1
                b.y = zc.y;
            }
            P[at<C>(y, ekc)] = b;
        }
        __syncwarp(mask);
        fft64<-1>(A, ColS<C>{P, ekz}, j, wf, mask);
        put_columns(out, kz, A, j, lane, mask);
#pragma unroll
        for (int m = 0; m < 8; m++) A[m] = P[at<C>(j + 8 * m, ekc)];
        __syncwarp(mask);
        fft64<-1>(A, ColS<C>{P, ekc}, j, wf, mask);
        put_columns(out + g.Mc, kz, A, j, lane, mask);
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
            fft64<-1>(a, RowX<C>{P, u}, j, wf, mask);
#pragma unroll
            for (int k = 0; k < 8; k++) P[at<C>(u, 8 * k + j)] = a[k];
        }
        __syncthreads();
        y_forward_paired(P, grp, j, lane, wf, mask, out);
    }
}

// ------------------------------------------------------------------------
// x-pass geometry: items of XT columns (FP64) or 2 XT (FP32) by 64 rows
constexpr int XT = 32;
static_assert(PLANE % XT == 0, "x-pass tiles cover the plane exactly");

// ------------------------------------------------------------------------
// K2 / K4, persistent and pipelined: work items are (job, branch, 32-column
// tile); each CTA walks items blockIdx.x, + gridDim.x, ... with two shared
// stages, so the bulk load of its next item and the bulk store of its previous
// one run while it transforms the current one.  Warp 0 issues all copies.
// columns per thread: 2 in FP32 (items of 64 columns, 512-byte row copies and
// twice the work per barrier), 1 in FP64 (32 columns, 512-byte rows)
template <typename C> __host__ __device__ constexpr int xpipe_cpt() { return sizeof(C) == 8 ? 2 : 1; }
template <typename C> __host__ __device__ constexpr int xpipe_width() { return XT * xpipe_cpt<C>(); }
template <typename C> __host__ __device__ constexpr int xpipe_tiles() { return PLANE / xpipe_width<C>(); }
template <typename C> constexpr size_t xpipe_smem() { return 2 * sizeof(C) * (size_t)N * xpipe_width<C>() + 16; }
static_assert(PLANE % (2 * XT) == 0, "64-column items cover the plane exactly");

// fft64_tile for CPT columns per thread (columns l + 32c of a tile of row stride XW)
template <int SIGN, int CPT, int XW, typename C>
__device__ __forceinline__ void fft64_tile_n(C (&a)[CPT][8], C *tb, int w, int l, C w1) {
#pragma unroll
    for (int c = 0; c < CPT; c++) {
        SmallDFT<8, C>::run(a[c], SIGN, nullptr, 0);
        twiddle8(a[c], w1);
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < CPT; c++)
#pragma unroll
        for (int k = 0; k < 8; k++) tb[(8 * k + w) * XW + l + 32 * c] = a[c][k];
    __syncthreads();
#pragma unroll
    for (int c = 0; c < CPT; c++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[c][k] = tb[(8 * w + k) * XW + l + 32 * c];
        SmallDFT<8, C>::run(a[c], SIGN, nullptr, 0);
    }
}

template <typename T, int NBR>
__global__ void __launch_bounds__(NTHR, 3) kp_xpass(GridPlan g, const lfts_step_job *__restrict__ jobs, int nj,
                                                    int spec_in0, int bsel0, int bsel1) {
    using C = typename CT<T>::type;
    constexpr int CPT = xpipe_cpt<C>(), XW = xpipe_width<C>(), XTILES = xpipe_tiles<C>();
    constexpr uint32_t ROWB = XW * sizeof(C), TILEB = N * ROWB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *stage = (C *)smem_raw;
    uint64_t *bar = (uint64_t *)(stage + 2 * N * XW);
    const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
    const int nitems = nj * NBR * XTILES;  // < 2^31 for nj <= 65535
    // first item at or after it whose job is active and aligned (>= nitems: none)
    auto next_item = [&](int it) -> int {
        for (; it < nitems; it += (int)gridDim.x) {
            const lfts_step_job &jb = jobs[it / (NBR * XTILES)];
            if (jb.active && !jb.active[jb.replica]) continue;
            if (((uintptr_t)jb.spec | (uintptr_t)g.Mc * sizeof(C)) & 15) {
                if (tid == 0) kerr_set(KERR_MISALIGNED);
                continue;
            }
            return it;
        }
        return nitems;
    };
    // spectrum column block of an item: rows x at + x * PLANE
    auto item_base = [&](int it) -> C * {
        const int job = it / (NBR * XTILES), rem = it - job * (NBR * XTILES);
        const int b = rem / XTILES, t = rem - b * XTILES;
        return (C *)jobs[job].spec + (size_t)(spec_in0 + b) * g.Mc + (size_t)t * XW;
    };
    auto issue_load = [&](int it, int st) {  // warp 0
        C *src = item_base(it);
        if (l == 0) mbar_arrive_expect_tx(bar + st, TILEB);
        __syncwarp();
        for (int r = l; r < N; r += 32) bulk_load(stage + (st * N + r) * XW, src + (size_t)r * PLANE, ROWB, bar + st);
    };
    int cur = next_item(blockIdx.x);
    if (cur >= nitems) return;
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
    }
    __syncthreads();
    if (w == 0) issue_load(cur, 0);
    const C wf = tw_base<C>(w, -1), wi = tw_base<C>(w, +1);
    for (int u = 0; cur < nitems; u++) {
        const int st = u & 1;
        const int nxt = next_item(cur + (int)gridDim.x);
        if (w == 0 && nxt < nitems) {
            bulk_wait_read();  // the previous store out of stage st ^ 1 has read it
            __syncwarp();
            issue_load(nxt, st ^ 1);
        }
        const int job = cur / (NBR * XTILES), rem = cur - job * (NBR * XTILES);
        const int b = rem / XTILES, t = rem - b * XTILES;
        const lfts_step_job &jb = jobs[job];
        const T *bt = (const T *)((b == 0 ? bsel0 : bsel1) ? jb.bond_half : jb.bond) + t * XW + l;
        T bv[CPT][8];
#pragma unroll
        for (int c = 0; c < CPT; c++)
#pragma unroll
            for (int k = 0; k < 8; k++) bv[c][k] = bt[(w + 8 * k) * PLANE + 32 * c];
        if (!mbar_wait(bar + st, (u >> 1) & 1)) {
            mbar_wait(bar + st, (u >> 1) & 1);
            if (w == 0) bulk_wait_read();
            return;
        }
        C *tb = stage + st * N * XW;
        C a[CPT][8];
#pragma unroll
        for (int c = 0; c < CPT; c++)
#pragma unroll
            for (int m = 0; m < 8; m++) a[c][m] = tb[(w + 8 * m) * XW + l + 32 * c];
        fft64_tile_n<-1, CPT, XW>(a, tb, w, l, wf);
#pragma unroll
        for (int c = 0; c < CPT; c++)
#pragma unroll
            for (int k = 0; k < 8; k++) {
                a[c][k].x *= bv[c][k];
                a[c][k].y *= bv[c][k];
            }
        fft64_tile_n<+1, CPT, XW>(a, tb, w, l, wi);
        __syncthreads();
#pragma unroll
        for (int c = 0; c < CPT; c++)
#pragma unroll
            for (int m = 0; m < 8; m++) tb[(w + 8 * m) * XW + l + 32 * c] = a[c][m];
        fence_proxy_async();
        __syncthreads();
        if (w == 0) {
            C *dst = item_base(cur);
            for (int r = l; r < N; r += 32) bulk_store(dst + (size_t)r * PLANE, tb + r * XW, ROWB);
            bulk_commit();
        }
        cur = nxt;
    }
    if (w == 0) bulk_wait_read();
}

// ------------------------------------------------------------------------
// K3: inverse zy, multiply by e = fac^2, forward zy, in place on slot spec_idx
template <typename T>
__global__ void __launch_bounds__(NTHR, (sizeof(T) == 4 ? LFTS_R8_MINB_F32 : LFTS_R8_MINB)) kr_plane_mid(GridPlan g, const lfts_step_job *__restrict__ jobs, int spec_idx) {
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
    y_inverse_paired(P, grp, j, wi, mask, sp);
    __syncthreads();
    {
        const int u = grp;
        const T *frow = fac + u * N + j;
        T ea[8], eb[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            ea[k] = frow[8 * k];
            eb[k] = frow[32 * N + 8 * k];
        }
        C a[8];
#pragma unroll
        for (int m = 0; m < 8; m++) a[m] = P[at<C>(u, 8 * m + j)];
        __syncwarp(mask);
        fft64<+1>(a, RowX<C>{P, u}, j, wi, mask);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            a[k].x = a[k].x * ea[k] * ea[k];
            a[k].y = a[k].y * eb[k] * eb[k];
        }
        fft64<-1>(a, RowX<C>{P, u}, j, wf, mask);
#pragma unroll
        for (int k = 0; k < 8; k++) P[at<C>(u, 8 * k + j)] = a[k];
    }
    __syncthreads();
    y_forward_paired(P, grp, j, lane, wf, mask, sp);
}

// ------------------------------------------------------------------------
// K5: inverse zy of NBR spectrum planes with the step epilogue.
//   NBR = 2, EPI_RICH: q' = (4 e_h v2 - e_h^2 v1) / 3 (v1 from slot spec_in0);
//   NBR = 1, EPI_SCALE: q' = f(fac) v.
template <typename T, int NBR, int EPI>
__global__ void __launch_bounds__(NTHR, (sizeof(T) == 4 ? LFTS_R8_MINB_F32 : LFTS_R8_MINB)) kr_plane_inverse(GridPlan g, const lfts_step_job *__restrict__ jobs, int s,
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
    const T THIRD = (T)(1.0 / 3.0);  // multiply, not divide: no iterative division per element
    if (NBR == 2) {
        {
            // branch 0 first; its inverse column waits in column ekz while
            // branch 1 is transformed, then both are packed into the z-lines
            const int kz = grp, ekz = kz, ekc = kz == 0 ? N / 2 : N - kz;
            C A[8];
            get_columns(in, kz, A, j);
            fft64<+1>(A, ColS<C>{P, ekz}, j, wi, mask);
#pragma unroll
            for (int k = 0; k < 8; k++) P[at<C>(j + 8 * k, ekz)] = A[k];
            get_columns(in + g.Mc, kz, A, j);
            fft64<+1>(A, ColS<C>{P, ekc}, j, wi, mask);
            // z-line y = j + 8k: A + i B (Hermitian extension at 64 - kz)
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int y = j + 8 * k;
                const C a = P[at<C>(y, ekz)], bb = A[k];
                C z;
                if (kz != 0) {
                    z.x = a.x - bb.y;
                    z.y = a.y + bb.x;
                    P[at<C>(y, ekz)] = z;
                    z.x = a.x + bb.y;
                    z.y = -a.y + bb.x;
                    P[at<C>(y, ekc)] = z;
                } else {
                    z.x = a.x;  // A(kz = 0) + i B(kz = 0)
                    z.y = bb.x;
                    P[at<C>(y, ekz)] = z;
                    z.x = a.y;  // A(kz = 32) + i B(kz = 32)
                    z.y = bb.y;
                    P[at<C>(y, ekc)] = z;
                }
            }
        }
        __syncthreads();
        for (int y = grp; y < N; y += GROUPS) {
            const T *frow = fac + y * N + j;
            T *qrow = qout + y * N + j;
            T eh[8];
#pragma unroll
            for (int k = 0; k < 8; k++) eh[k] = frow[8 * k];
            C a[8];
#pragma unroll
            for (int m = 0; m < 8; m++) a[m] = P[at<C>(y, 8 * m + j)];
            __syncwarp(mask);
            fft64<+1>(a, RowX<C>{P, y}, j, wi, mask);
#pragma unroll
            for (int k = 0; k < 8; k++) qrow[8 * k] = ((T)4 * eh[k] * a[k].y - eh[k] * eh[k] * a[k].x) * THIRD;
        }
    } else {
        y_inverse_paired(P, grp, j, wi, mask, in);
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
        for (int m = 0; m < 8; m++) a[m] = P[at<C>(u, 8 * m + j)];
        __syncwarp(mask);
        fft64<+1>(a, RowX<C>{P, u}, j, wi, mask);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            qout[u * N + j + 8 * k] = a[k].x * fmul_mode(fm0, fa[k]);
            qout[(u + 32) * N + j + 8 * k] = a[k].y * fmul_mode(fm0, fb[k]);
        }
    }
}

}  // namespace r8
}  // namespace lfts
