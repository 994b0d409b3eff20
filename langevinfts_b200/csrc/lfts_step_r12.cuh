// Register-resident plane kernels for 96^3 grids (96 = 12 x 8).
//
// The plane passes of the continuous step (K1, K3, K5 of lfts_step_fast.cuh)
// with the same spectra layout in HBM ([x][ky][kz], natural order).  Every
// 96-point line transform is held by the 8 lanes of one lane group, 12 values
// per lane, and passes through shared memory once:
//   variant A: lane j holds x[j + 8m] (m < 12).  A 12-point DFT over m (prime
//     factor map 12 = 3 x 4, no internal twiddles), the twiddle w96^(j k2),
//     one exchange, then twelve 8-point DFTs over j: lane t takes k2 = t and,
//     for t < 4, also k2 = 8 + t.  Lane t ends with X[t + 12k] (k < 8) and,
//     for t < 4, X[8 + t + 12k].
//   variant B, the transpose: lane t starts with x[t + 12k] (and x[8 + t +
//     12k]); 8-point DFTs, the twiddle w96^(n2 k1), one exchange, a 12-point
//     DFT; lane j ends with X[j + 8k] (k < 12).  The mid pass runs inverse z,
//     the field multiply and forward z on one line without another exchange.
// X[k] = sum_n x[n] exp(SIGN 2 pi i n k / 96) in both.
// The exchange slot of (k2, j) is 8 k2 + ((j + k2) & 7): the writes (fixed k2)
// and the reads (fixed j) of a lane group each touch eight banks, in a row and
// down a column alike.  Plane positions go through PlaneLayout96: FP64
// (16-byte complex, one lane group per wavefront) uses rows of stride 97;
// FP32 (8-byte complex, two groups per wavefront) uses rows of 96 with
// position p at p XOR 8 (row parity) XOR (row AND 6), which keeps the two
// groups of a wavefront apart as well (43 % fewer shared-memory wavefronts
// than stride 97 with 8-byte elements, per a count of the kernels' patterns).
//
// Plane kernels run 48 lane groups (384 threads) per CTA.  K1 and K5 keep one
// x-plane of packed z-lines (both branches as real / imaginary part, 96 rows of
// stride 97); K3 keeps 48 rows (rows y and y + 48 packed) and runs the column
// exchanges of task kz down its two columns kz and 96 - kz.
#pragma once
#include "lfts_step_r8.cuh"

namespace lfts {
namespace r12 {

constexpr int N = 96, NZC = N / 2 + 1, PLANE = N * NZC;
constexpr int GROUPS = 48, NT = 8 * GROUPS;

template <typename C> struct PlaneLayout96;
template <> struct PlaneLayout96<double2> {
    static constexpr int RS = 97;
    __device__ __forceinline__ static int at(int r, int p) { return r * RS + p; }
};
template <> struct PlaneLayout96<float2> {
    static constexpr int RS = 96;
    __device__ __forceinline__ static int at(int r, int p) { return r * RS + (p ^ ((r & 1) << 3) ^ (r & 6)); }
};
// index of position p of row r of a plane in shared memory
template <typename C> __device__ __forceinline__ int at(int r, int p) { return PlaneLayout96<C>::at(r, p); }
template <typename C> constexpr size_t plane_smem(int rows) { return sizeof(C) * (size_t)rows * PlaneLayout96<C>::RS; }

__device__ __forceinline__ int slot(int k2, int j) { return 8 * k2 + ((j + k2) & 7); }

// w96^e with the sign of the transform
template <typename C>
__device__ __forceinline__ C tw96(int e, int sign) {
    double sn, cs;
    sincospi((double)e / 48.0, &sn, &cs);
    C w;
    w.x = cs;
    w.y = sign * sn;
    return w;
}

// exchange spaces: position p of a 96-slot line
template <typename C> struct Row {  // row r of plane P
    C *P;
    int r;
    __device__ __forceinline__ C &at(int p) const { return P[lfts::r12::at<C>(r, p)]; }
    __device__ __forceinline__ C &ref(int k2, int j) const { return at(slot(k2, j)); }
};
template <typename C> struct Col {  // column c of a 96-row plane P
    C *P;
    int c;
    __device__ __forceinline__ C &at(int p) const { return P[lfts::r12::at<C>(p, c)]; }
    __device__ __forceinline__ C &ref(int k2, int j) const { return at(slot(k2, j)); }
};
template <typename C> struct Col2 {  // columns c0, c1 of a 48-row plane P (positions 0..47, 48..95)
    C *P;
    int c0, c1;
    __device__ __forceinline__ C &at(int p) const {
        return p < N / 2 ? P[lfts::r12::at<C>(p, c0)] : P[lfts::r12::at<C>(p - N / 2, c1)];
    }
    __device__ __forceinline__ C &ref(int k2, int j) const { return at(slot(k2, j)); }
};

// 12-point DFT in place, natural order: input n = (4 n1 + 3 n2) mod 12 and
// output k = (4 k1 + 9 k2) mod 12 (n1, k1 < 3; n2, k2 < 4) turn it into
// 3-point DFTs of 4-point DFTs with no twiddles between them.
template <int SIGN, typename C>
__device__ __forceinline__ void dft12(C (&a)[12]) {
    C t[3][4];
#pragma unroll
    for (int n1 = 0; n1 < 3; n1++)
#pragma unroll
        for (int n2 = 0; n2 < 4; n2++) t[n1][n2] = a[(4 * n1 + 3 * n2) % 12];
#pragma unroll
    for (int n1 = 0; n1 < 3; n1++) SmallDFT<4, C>::run(t[n1], SIGN, nullptr, 0);
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) {
        C u[3] = {t[0][k2], t[1][k2], t[2][k2]};
        SmallDFT<3, C>::run(u, SIGN, nullptr, 0);
#pragma unroll
        for (int k1 = 0; k1 < 3; k1++) a[(4 * k1 + 9 * k2) % 12] = u[k1];
    }
}

// a[k] *= w1^k for k = 1..11 (powers by a tree of depth 4)
template <typename C>
__device__ __forceinline__ void twiddle12(C (&a)[12], C w1) {
    const C w2 = cmul(w1, w1);
    const C w3 = cmul(w2, w1), w4 = cmul(w2, w2);
    const C w5 = cmul(w4, w1), w6 = cmul(w3, w3), w7 = cmul(w4, w3), w8 = cmul(w4, w4);
    a[1] = cmul(a[1], w1);
    a[2] = cmul(a[2], w2);
    a[3] = cmul(a[3], w3);
    a[4] = cmul(a[4], w4);
    a[5] = cmul(a[5], w5);
    a[6] = cmul(a[6], w6);
    a[7] = cmul(a[7], w7);
    a[8] = cmul(a[8], w8);
    a[9] = cmul(a[9], cmul(w8, w1));
    a[10] = cmul(a[10], cmul(w5, w5));
    a[11] = cmul(a[11], cmul(w8, w3));
}

// Variant A.  w1 = w96^j with the transform's sign; o1 is set for j < 4 only.
template <int SIGN, class AT, typename C>
__device__ __forceinline__ void fft96a(C (&a)[12], const AT &at, int j, C w1, unsigned mask, C (&o0)[8], C (&o1)[8]) {
    dft12<SIGN>(a);
    twiddle12(a, w1);
#pragma unroll
    for (int k2 = 0; k2 < 12; k2++) at.ref(k2, j) = a[k2];
    __syncwarp(mask);
#pragma unroll
    for (int i = 0; i < 8; i++) o0[i] = at.ref(j, i);
    if (j < 4) {
#pragma unroll
        for (int i = 0; i < 8; i++) o1[i] = at.ref(8 + j, i);
    }
    __syncwarp(mask);
    SmallDFT<8, C>::run(o0, SIGN, nullptr, 0);
    if (j < 4) SmallDFT<8, C>::run(o1, SIGN, nullptr, 0);
}

// Variant B.  v0 = w96^t, v1 = w96^(8 + t) with the transform's sign; b1 is
// read for t < 4 only.  Lane j ends with X[j + 8k] in a[k].
template <int SIGN, class AT, typename C>
__device__ __forceinline__ void fft96b(C (&b0)[8], C (&b1)[8], const AT &at, int t, C v0, C v1, unsigned mask, C (&a)[12]) {
    SmallDFT<8, C>::run(b0, SIGN, nullptr, 0);
    r8::twiddle8(b0, v0);
#pragma unroll
    for (int k1 = 0; k1 < 8; k1++) at.ref(t, k1) = b0[k1];
    if (t < 4) {
        SmallDFT<8, C>::run(b1, SIGN, nullptr, 0);
        r8::twiddle8(b1, v1);
#pragma unroll
        for (int k1 = 0; k1 < 8; k1++) at.ref(8 + t, k1) = b1[k1];
    }
    __syncwarp(mask);
#pragma unroll
    for (int n2 = 0; n2 < 12; n2++) a[n2] = at.ref(n2, t);
    __syncwarp(mask);
    dft12<SIGN>(a);
}

// Column(s) of task kz of a global spectrum plane st ([ky][kz]) for an inverse
// y-transform: lane j gets ky = j + 8m; task 0 packs c = col 0 + i col 48.
template <typename C>
__device__ __forceinline__ void get_columns(const C *st, int kz, C (&c)[12], int j) {
    if (kz != 0) {
        const C *col = st + j * NZC + kz;
#pragma unroll
        for (int m = 0; m < 12; m++) c[m] = col[8 * m * NZC];
    } else {
#pragma unroll
        for (int m = 0; m < 12; m++) {
            const C *row = st + (j + 8 * m) * NZC;
            const C a = row[0], b = row[N / 2];
            c[m].x = a.x - b.y;
            c[m].y = a.y + b.x;
        }
    }
}

// Store a forward y-transform of task kz (lane t: ky = t + 12k in o0 and, for
// t < 4, ky = 8 + t + 12k in o1) to a spectrum plane st.  Task 0 holds
// c = F[col 0] + i F[col 48] and splits it with the Hermitian partner
// c[96 - ky], fetched through its free exchange space xs.
template <typename C, class AT>
__device__ __forceinline__ void put_columns(C *st, const AT &xs, int kz, const C (&o0)[8], const C (&o1)[8], int t,
                                            unsigned mask) {
    if (kz != 0) {
        C *col = st + kz;
#pragma unroll
        for (int k = 0; k < 8; k++) col[(t + 12 * k) * NZC] = o0[k];
        if (t < 4) {
#pragma unroll
            for (int k = 0; k < 8; k++) col[(8 + t + 12 * k) * NZC] = o1[k];
        }
    } else {
#pragma unroll
        for (int k = 0; k < 8; k++) xs.at(t + 12 * k) = o0[k];
        if (t < 4) {
#pragma unroll
            for (int k = 0; k < 8; k++) xs.at(8 + t + 12 * k) = o1[k];
        }
        __syncwarp(mask);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int ky = t + 12 * k;
            C a, b;
            split_pair(o0[k], cconj(xs.at((N - ky) % N)), a, b);
            st[ky * NZC] = a;
            st[ky * NZC + N / 2] = b;
        }
        if (t < 4) {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int ky = 8 + t + 12 * k;
                C a, b;
                split_pair(o1[k], cconj(xs.at(N - ky)), a, b);
                st[ky * NZC] = a;
                st[ky * NZC + N / 2] = b;
            }
        }
        __syncwarp(mask);
    }
}

// Write A + i B of row y at columns kz and kc = 96 - kz of a packed plane
// (Hermitian extension); task 0 carries (DC, Nyquist) in (x, y) of A and B.
template <typename C>
__device__ __forceinline__ void put_packed(C *P, int y, int kz, int kc, C A, C B) {
    C z;
    if (kz != 0) {
        z.x = A.x - B.y;
        z.y = A.y + B.x;
        P[at<C>(y, kz)] = z;
        z.x = A.x + B.y;
        z.y = -A.y + B.x;
        P[at<C>(y, kc)] = z;
    } else {
        z.x = A.x;
        z.y = B.x;
        P[at<C>(y, 0)] = z;
        z.x = A.y;
        z.y = B.y;
        P[at<C>(y, N / 2)] = z;
    }
}

// resident CTAs per SM the kernels are compiled for (register budget)
template <typename T> __host__ __device__ constexpr int minb_two_branch() { return sizeof(T) == 4 ? 2 : 1; }
template <typename T> __host__ __device__ constexpr int minb_mid() { return sizeof(T) == 4 ? 2 : 1; }

// ------------------------------------------------------------------------
// K1: forward zy transform of one x-plane into the spectra of f0(fac) q and
// f1(fac) q (slots spec_out0, spec_out0 + 1).
template <typename T, int FM0, int FM1>
__global__ void __launch_bounds__(NT, minb_two_branch<T>()) kq_plane_forward(GridPlan g, const lfts_step_job *__restrict__ jobs,
                                                                          int s, int spec_out0) {
    using C = typename CT<T>::type;
    constexpr int fm0 = FM0, fm1 = FM1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *P = (C *)smem_raw;
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x, tid = threadIdx.x, lane = tid & 31, j = lane & 7, grp = tid >> 3;
    const unsigned mask = 0xFFu << (lane & 24);
    const C wf = tw96<C>(j, -1);
    const long long poff = (long long)x * N * N;
    const T *qin = (const T *)jb.in + s * jb.in_stride + poff;
    const T *fac = (const T *)jb.fac + poff;
    C *out = (C *)jb.spec + (size_t)spec_out0 * g.Mc + (size_t)x * PLANE;
    // z-lines: row y with the branches as real / imaginary part; X[k] at row position k
    for (int y = grp; y < N; y += GROUPS) {
        const T *qrow = qin + y * N + j, *frow = fac + y * N + j;
        T qv[12], fv[12];
#pragma unroll
        for (int m = 0; m < 12; m++) {
            qv[m] = qrow[8 * m];
            fv[m] = fm0 == FM_NONE ? (T)1 : frow[8 * m];
        }
        C a[12];
#pragma unroll
        for (int m = 0; m < 12; m++) {
            const T f0 = fm0 == FM_FAC_SQ ? fv[m] * fv[m] : fv[m];
            const T f1 = fm1 == FM_FAC_SQ ? fv[m] * fv[m] : (fm1 == FM_NONE ? (T)1 : fv[m]);
            a[m].x = qv[m] * f0;
            a[m].y = qv[m] * f1;
        }
        C o0[8], o1[8];
        fft96a<-1>(a, Row<C>{P, y}, j, wf, mask, o0, o1);
#pragma unroll
        for (int k = 0; k < 8; k++) P[at<C>(y, j + 12 * k)] = o0[k];
        if (j < 4) {
#pragma unroll
            for (int k = 0; k < 8; k++) P[at<C>(y, 8 + j + 12 * k)] = o1[k];
        }
    }
    __syncthreads();
    // y-columns: task kz splits columns kz and kc into the branches; branch 1
    // waits in column kc while branch 0 is transformed and stored
    const int kz = grp, kc = kz == 0 ? N / 2 : N - kz;
    C A[12];
#pragma unroll
    for (int m = 0; m < 12; m++) {
        const int y = j + 8 * m;
        const C zk = P[at<C>(y, kz)], zc = P[at<C>(y, kc)];
        C b;
        if (kz != 0) {
            split_pair(zk, cconj(zc), A[m], b);
        } else {
            A[m].x = zk.x;  // branch 0: DC + i Nyquist
            A[m].y = zc.x;
            b.x = zk.y;  // branch 1
            b.y = zc.y;
        }
        P[at<C>(y, kc)] = b;
    }
    __syncwarp(mask);
    C o0[8], o1[8];
    fft96a<-1>(A, Col<C>{P, kz}, j, wf, mask, o0, o1);
    put_columns(out, Col<C>{P, kz}, kz, o0, o1, j, mask);
#pragma unroll
    for (int m = 0; m < 12; m++) A[m] = P[at<C>(j + 8 * m, kc)];
    __syncwarp(mask);
    fft96a<-1>(A, Col<C>{P, kc}, j, wf, mask, o0, o1);
    put_columns(out + g.Mc, Col<C>{P, kc}, kz, o0, o1, j, mask);
}

// ------------------------------------------------------------------------
// K3: inverse zy, multiply by e = fac^2, forward zy, in place on slot spec_idx
template <typename T>
__global__ void __launch_bounds__(NT, minb_mid<T>()) kq_plane_mid(GridPlan g, const lfts_step_job *__restrict__ jobs, int spec_idx) {
    using C = typename CT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *P = (C *)smem_raw;  // 48 packed rows: z-line u = row u + i row (u + 48)
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x, tid = threadIdx.x, lane = tid & 31, j = lane & 7, grp = tid >> 3;
    const unsigned mask = 0xFFu << (lane & 24);
    C *sp = (C *)jb.spec + (size_t)spec_idx * g.Mc + (size_t)x * PLANE;
    const T *fac = (const T *)jb.fac + (long long)x * N * N;
    const int kz = grp, kc = kz == 0 ? N / 2 : N - kz;
    {
        // inverse y: lane t ends with rows t + 12k; rows u and u + 48 are k and k + 4
        C a[12], o0[8], o1[8];
        get_columns(sp, kz, a, j);
        fft96a<+1>(a, Col2<C>{P, kz, kc}, j, tw96<C>(j, +1), mask, o0, o1);
#pragma unroll
        for (int k = 0; k < 4; k++) put_packed(P, j + 12 * k, kz, kc, o0[k], o0[k + 4]);
        if (j < 4) {
#pragma unroll
            for (int k = 0; k < 4; k++) put_packed(P, 8 + j + 12 * k, kz, kc, o1[k], o1[k + 4]);
        }
    }
    __syncthreads();
    {
        const int u = grp;
        const T *fa = fac + u * N, *fb = fac + (u + N / 2) * N;
        T ea0[8], eb0[8], ea1[8], eb1[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            ea0[k] = fa[j + 12 * k];
            eb0[k] = fb[j + 12 * k];
        }
        if (j < 4) {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                ea1[k] = fa[8 + j + 12 * k];
                eb1[k] = fb[8 + j + 12 * k];
            }
        }
        C a[12], o0[8], o1[8];
#pragma unroll
        for (int m = 0; m < 12; m++) a[m] = P[at<C>(u, j + 8 * m)];
        __syncwarp(mask);
        fft96a<+1>(a, Row<C>{P, u}, j, tw96<C>(j, +1), mask, o0, o1);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            o0[k].x *= ea0[k] * ea0[k];
            o0[k].y *= eb0[k] * eb0[k];
        }
        if (j < 4) {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                o1[k].x *= ea1[k] * ea1[k];
                o1[k].y *= eb1[k] * eb1[k];
            }
        }
        fft96b<-1>(o0, o1, Row<C>{P, u}, j, tw96<C>(j, -1), tw96<C>(8 + j, -1), mask, a);
#pragma unroll
        for (int k = 0; k < 12; k++) P[at<C>(u, j + 8 * k)] = a[k];
    }
    __syncthreads();
    {
        // forward y: lane j takes rows u = j + 8m (m < 6) and u + 48
        C c[12];
#pragma unroll
        for (int m = 0; m < 6; m++) {
            const int u = j + 8 * m;
            if (kz != 0) {
                split_pair(P[at<C>(u, kz)], cconj(P[at<C>(u, kc)]), c[m], c[m + 6]);
            } else {
                const C z0 = P[at<C>(u, 0)], z48 = P[at<C>(u, N / 2)];
                c[m].x = z0.x;  // row u: DC + i Nyquist
                c[m].y = z48.x;
                c[m + 6].x = z0.y;  // row u + 48
                c[m + 6].y = z48.y;
            }
        }
        __syncwarp(mask);
        C o0[8], o1[8];
        fft96a<-1>(c, Col2<C>{P, kz, kc}, j, tw96<C>(j, -1), mask, o0, o1);
        put_columns(sp, Col2<C>{P, kz, kc}, kz, o0, o1, j, mask);
    }
}

// ------------------------------------------------------------------------
// K5: inverse zy of the spectra in slots spec_in0 (v1) and spec_in0 + 1 (v2),
// q' = (4 e_h v2 - e_h^2 v1) / 3 with e_h = fac
template <typename T>
__global__ void __launch_bounds__(NT, minb_two_branch<T>()) kq_plane_inverse(GridPlan g, const lfts_step_job *__restrict__ jobs,
                                                                          int s, int spec_in0) {
    using C = typename CT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *P = (C *)smem_raw;
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x, tid = threadIdx.x, lane = tid & 31, j = lane & 7, grp = tid >> 3;
    const unsigned mask = 0xFFu << (lane & 24);
    const C wi = tw96<C>(j, +1);
    const C *in = (const C *)jb.spec + (size_t)spec_in0 * g.Mc + (size_t)x * PLANE;
    const long long poff = (long long)x * N * N;
    const T *fac = (const T *)jb.fac + poff;
    T *qout = (T *)jb.out + s * jb.out_stride + poff;
    const T THIRD = (T)(1.0 / 3.0);
    {
        // branch 0 waits in column kz (rows y) while branch 1 is transformed,
        // then both are packed into the z-lines
        const int kz = grp, kc = kz == 0 ? N / 2 : N - kz;
        C A[12], o0[8], o1[8];
        get_columns(in, kz, A, j);
        fft96a<+1>(A, Col<C>{P, kz}, j, wi, mask, o0, o1);
#pragma unroll
        for (int k = 0; k < 8; k++) P[at<C>(j + 12 * k, kz)] = o0[k];
        if (j < 4) {
#pragma unroll
            for (int k = 0; k < 8; k++) P[at<C>(8 + j + 12 * k, kz)] = o1[k];
        }
        get_columns(in + g.Mc, kz, A, j);
        fft96a<+1>(A, Col<C>{P, kc}, j, wi, mask, o0, o1);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int y = j + 12 * k;
            put_packed(P, y, kz, kc, P[at<C>(y, kz)], o0[k]);
        }
        if (j < 4) {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int y = 8 + j + 12 * k;
                put_packed(P, y, kz, kc, P[at<C>(y, kz)], o1[k]);
            }
        }
    }
    __syncthreads();
    for (int y = grp; y < N; y += GROUPS) {
        const T *frow = fac + y * N;
        T *qrow = qout + y * N;
        T e0[8], e1[8];
#pragma unroll
        for (int k = 0; k < 8; k++) e0[k] = frow[j + 12 * k];
        if (j < 4) {
#pragma unroll
            for (int k = 0; k < 8; k++) e1[k] = frow[8 + j + 12 * k];
        }
        C a[12], o0[8], o1[8];
#pragma unroll
        for (int m = 0; m < 12; m++) a[m] = P[at<C>(y, j + 8 * m)];
        __syncwarp(mask);
        fft96a<+1>(a, Row<C>{P, y}, j, wi, mask, o0, o1);
#pragma unroll
        for (int k = 0; k < 8; k++) qrow[j + 12 * k] = ((T)4 * e0[k] * o0[k].y - e0[k] * e0[k] * o0[k].x) * THIRD;
        if (j < 4) {
#pragma unroll
            for (int k = 0; k < 8; k++) qrow[8 + j + 12 * k] = ((T)4 * e1[k] * o1[k].y - e1[k] * e1[k] * o1[k].x) * THIRD;
        }
    }
}

// ------------------------------------------------------------------------
// K2 / K4, persistent and pipelined: work items are (job, branch, tile of XW
// columns of the [kx][ky][kz] spectrum), 96 rows each.  Warp 0 bulk-loads the
// next item into the other of two shared stages while the CTA transforms the
// current one, and bulk-stores each finished tile.  Thread (w, l) owns column
// l of the tile: variant A forward over rows w + 8m (warps w < 4 take the
// second round of 8-point DFTs), the bond multiply on rows w + 12k and
// 8 + w + 12k, then variant B inverse, which starts from exactly those rows.
// (A split over 12 warps that balances the 8-point DFTs measured slower: one
// CTA per SM at its FP64 register need, or spills at two.)
constexpr int XW = 32;  // columns per item (512-byte rows in FP64, 256 in FP32)
constexpr int XTILES = PLANE / XW;
static_assert(PLANE % XW == 0, "x-pass tiles cover the plane exactly");
template <typename C> constexpr size_t xpipe_smem() { return 2 * sizeof(C) * (size_t)N * XW + 16; }
// resident CTAs per SM: FP32 four (64 registers, a few spills; the pass waits at
// its barriers, so more CTAs hide more of it: 0.765 against 0.777 ms a 32-job
// step at three), FP64 two
template <typename T> __host__ __device__ constexpr int minb_xpass() { return sizeof(T) == 4 ? 4 : 2; }

template <typename T, int NBR>
__global__ void __launch_bounds__(NTHR, minb_xpass<T>()) kq_xpass(GridPlan g, const lfts_step_job *__restrict__ jobs, int nj,
                                                                  int spec_in0, int bsel0, int bsel1) {
    using C = typename CT<T>::type;
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
    const C wf = tw96<C>(w, -1), vi0 = tw96<C>(w, +1), vi1 = tw96<C>(8 + w, +1);
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
        if (!mbar_wait(bar + st, (u >> 1) & 1)) {
            mbar_wait(bar + st, (u >> 1) & 1);
            if (w == 0) bulk_wait_read();
            return;
        }
        C *tb = stage + st * N * XW + l;
        // forward: rows w + 8m -> X[w + 12k] (o0), X[8 + w + 12k] (o1, w < 4)
        C a[12], o0[8], o1[8];
#pragma unroll
        for (int m = 0; m < 12; m++) a[m] = tb[(w + 8 * m) * XW];
        dft12<-1>(a);
        twiddle12(a, wf);
        __syncthreads();
#pragma unroll
        for (int k2 = 0; k2 < 12; k2++) tb[slot(k2, w) * XW] = a[k2];
        // bond factors of rows w + 12k and 8 + w + 12k (loaded here, not before
        // the forward stage, to keep the FP64 register count within two CTAs)
        T bv0[8], bv1[8];
#pragma unroll
        for (int k = 0; k < 8; k++) bv0[k] = bt[(w + 12 * k) * PLANE];
        if (w < 4) {
#pragma unroll
            for (int k = 0; k < 8; k++) bv1[k] = bt[(8 + w + 12 * k) * PLANE];
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 8; i++) o0[i] = tb[slot(w, i) * XW];
        SmallDFT<8, C>::run(o0, -1, nullptr, 0);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            o0[k].x *= bv0[k];
            o0[k].y *= bv0[k];
        }
        if (w < 4) {
#pragma unroll
            for (int i = 0; i < 8; i++) o1[i] = tb[slot(8 + w, i) * XW];
            SmallDFT<8, C>::run(o1, -1, nullptr, 0);
#pragma unroll
            for (int k = 0; k < 8; k++) {
                o1[k].x *= bv1[k];
                o1[k].y *= bv1[k];
            }
        }
        // inverse, variant B: the slots rewritten here are the ones this
        // thread has just read
        SmallDFT<8, C>::run(o0, +1, nullptr, 0);
        r8::twiddle8(o0, vi0);
#pragma unroll
        for (int k1 = 0; k1 < 8; k1++) tb[slot(w, k1) * XW] = o0[k1];
        if (w < 4) {
            SmallDFT<8, C>::run(o1, +1, nullptr, 0);
            r8::twiddle8(o1, vi1);
#pragma unroll
            for (int k1 = 0; k1 < 8; k1++) tb[slot(8 + w, k1) * XW] = o1[k1];
        }
        __syncthreads();
#pragma unroll
        for (int n2 = 0; n2 < 12; n2++) a[n2] = tb[slot(n2, w) * XW];
        dft12<+1>(a);
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 12; k++) tb[(w + 8 * k) * XW] = a[k];
        fence_proxy_async();
        __syncthreads();
        if (w == 0) {
            C *dst = item_base(cur);
            for (int r = l; r < N; r += 32) bulk_store(dst + (size_t)r * PLANE, stage + (st * N + r) * XW, ROWB);
            bulk_commit();
        }
        cur = nxt;
    }
    if (w == 0) bulk_wait_read();
}

}  // namespace r12
}  // namespace lfts
