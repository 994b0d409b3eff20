// Device FFT building blocks for the pseudo-spectral contour step (sm_100a).
//
// The reference calls a library 3D real FFT per operator-splitting sub-step
// (cufftExecD2Z/Z2D at src/platforms/cuda/CudaSolverPseudo.cu:371-396, MKL DFTI
// at src/platforms/cpu/MklFFT3D.cpp:55-79).  Here the 3D transform is split into
// shared-memory passes that the step kernels fuse with their pointwise work:
//   * a "plane" pass does the real z transform and the complex y transform of
//     one x-plane entirely in shared memory,
//   * a "column" pass does the complex x transform of a tile of (y, kz)
//     columns, applies the Boltzmann bond factor and transforms back.
// Every 1D transform is an in-place mixed-radix Cooley-Tukey transform over
// lines held in shared memory:
//   DIT: input at digit-reversed positions perm(t) -> natural-order output,
//   DIF: natural-order input -> output at digit-reversed positions perm(k),
// so a forward DIT followed by an inverse DIF needs no permutation pass and no
// ping-pong buffer.  Radices 2, 3, 4, 5, 8 are unrolled; any other prime factor
// up to LFTS_MAX_RADIX uses a direct small DFT.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define LFTS_MAX_FACTORS 8
#define LFTS_MAX_RADIX 64
#define LFTS_MAX_AXIS 1024

namespace lfts {

template <typename T> struct CT;
template <> struct CT<double> { using type = double2; };
template <> struct CT<float> { using type = float2; };

template <typename C> __device__ __forceinline__ C cmk(double re, double im) { C c; c.x = re; c.y = im; return c; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
// FP32 complex add and subtract as one packed instruction each (add / sub
// .rn.f32x2 of sm_100: each lane rounded to nearest, as two scalar adds are)
__device__ __forceinline__ unsigned long long pack2(float2 a) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 unpack2(unsigned long long r) {
    float2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pack2(a)), "l"(pack2(b)));
    return unpack2(r);
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pack2(a)), "l"(pack2(b)));
    return unpack2(r);
}
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    C c;
    c.x = a.x * b.x - a.y * b.y;
    c.y = a.x * b.y + a.y * b.x;
    return c;
}
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
// multiply by -i (sign<0) or +i (sign>0)
template <typename C> __device__ __forceinline__ C cmul_i(C a, int sign) {
    C c;
    if (sign < 0) { c.x = a.y; c.y = -a.x; } else { c.x = -a.y; c.y = a.x; }
    return c;
}

// One axis of the transform.  radix[] is outermost-first: n = radix[0]*...*radix[nf-1].
struct AxisPlan {
    int n;
    int nf;
    int radix[LFTS_MAX_FACTORS];
};

// Plan of a 3D real grid n0 x n1 x n2 (z = n2 fastest).  1D/2D boxes use
// leading extents of 1, as the reference's Pseudo.cpp:17-82 does.
struct GridPlan {
    int n0, n1, n2, nzc;     // nzc = n2/2 + 1
    long long M, Mc;         // n0*n1*n2, n0*n1*nzc
    AxisPlan ax[3];
    const void *tw[3];       // twiddles exp(-2 pi i j / n), n entries, precision T
    const short *perm[3];    // digit-reversal permutation, n entries
    const void *stw;         // per-stage twiddles of the cubic fast path (lfts_step_fast.cuh), or NULL
};

// w_n^e for the forward (sign<0) or inverse (sign>0) direction, table in shared memory
template <typename C>
__device__ __forceinline__ C twid(const C *tw, int e, int sign) {
    C t = tw[e];
    if (sign > 0) t.y = -t.y;
    return t;
}

// In-register small DFT: a[k] <- sum_j a[j] w_R^(jk), w_R = exp(sign 2 pi i / R)
template <int R, typename C> struct SmallDFT;

template <typename C> struct SmallDFT<2, C> {
    __device__ __forceinline__ static void run(C *a, int, const C *, int) {
        C t = a[0];
        a[0] = cadd(t, a[1]);
        a[1] = csub(t, a[1]);
    }
};
template <typename C> struct SmallDFT<4, C> {
    __device__ __forceinline__ static void run(C *a, int sign, const C *, int) {
        C t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
        C t2 = cadd(a[1], a[3]), t3 = cmul_i(csub(a[1], a[3]), sign);
        a[0] = cadd(t0, t2);
        a[2] = csub(t0, t2);
        a[1] = cadd(t1, t3);
        a[3] = csub(t1, t3);
    }
};
template <typename C> struct SmallDFT<8, C> {
    __device__ __forceinline__ static void run(C *a, int sign, const C *, int) {
        using T = decltype(a[0].x);
        const T h = (T)0.70710678118654752440084436210485;
        // radix-2 over pairs (j, j+4), then twiddle w_8^j, then two radix-4
        C b[8];
#pragma unroll
        for (int j = 0; j < 4; j++) { b[j] = cadd(a[j], a[j + 4]); b[j + 4] = csub(a[j], a[j + 4]); }
        // b[4+j] *= w_8^j
        {
            C t = b[5];  // * (h, sign*h)
            b[5].x = h * (t.x - (T)sign * t.y);
            b[5].y = h * (t.y + (T)sign * t.x);
            b[6] = cmul_i(b[6], sign);
            t = b[7];    // * (-h, sign*h)
            b[7].x = h * (-t.x - (T)sign * t.y);
            b[7].y = h * (-t.y + (T)sign * t.x);
        }
        C e[4] = {b[0], b[1], b[2], b[3]};
        C o[4] = {b[4], b[5], b[6], b[7]};
        SmallDFT<4, C>::run(e, sign, nullptr, 0);
        SmallDFT<4, C>::run(o, sign, nullptr, 0);
        // even outputs from e, odd outputs from o
#pragma unroll
        for (int k = 0; k < 4; k++) { a[2 * k] = e[k]; a[2 * k + 1] = o[k]; }
    }
};
template <typename C> struct SmallDFT<3, C> {
    __device__ __forceinline__ static void run(C *a, int sign, const C *, int) {
        using T = decltype(a[0].x);
        const T c = (T)-0.5, s = (T)sign * (T)0.86602540378443864676372317075294;
        C t1 = cadd(a[1], a[2]), t2 = csub(a[1], a[2]);
        C m1;
        m1.x = a[0].x + c * t1.x;
        m1.y = a[0].y + c * t1.y;
        C r2;  // s * i * t2
        r2.x = -s * t2.y;
        r2.y = s * t2.x;
        a[0] = cadd(a[0], t1);
        a[1] = cadd(m1, r2);
        a[2] = csub(m1, r2);
    }
};
template <typename C> struct SmallDFT<5, C> {
    __device__ __forceinline__ static void run(C *a, int sign, const C *, int) {
        using T = decltype(a[0].x);
        const T c1 = (T)0.30901699437494742410229341718282, c2 = (T)-0.80901699437494742410229341718282;
        const T s1 = (T)sign * (T)0.95105651629515357211643933337938;
        const T s2 = (T)sign * (T)0.58778525229247312916870595463907;
        C b1 = cadd(a[1], a[4]), b4 = csub(a[1], a[4]);
        C b2 = cadd(a[2], a[3]), b3 = csub(a[2], a[3]);
        C m1, m2;
        m1.x = a[0].x + c1 * b1.x + c2 * b2.x;
        m1.y = a[0].y + c1 * b1.y + c2 * b2.y;
        m2.x = a[0].x + c2 * b1.x + c1 * b2.x;
        m2.y = a[0].y + c2 * b1.y + c1 * b2.y;
        // n1 = i*(s1*b4 + s2*b3), n2 = i*(s2*b4 - s1*b3)
        C n1, n2;
        n1.x = -(s1 * b4.y + s2 * b3.y);
        n1.y = s1 * b4.x + s2 * b3.x;
        n2.x = -(s2 * b4.y - s1 * b3.y);
        n2.y = s2 * b4.x - s1 * b3.x;
        a[0] = cadd(a[0], cadd(b1, b2));
        a[1] = cadd(m1, n1);
        a[4] = csub(m1, n1);
        a[2] = cadd(m2, n2);
        a[3] = csub(m2, n2);
    }
};

// Line addressing inside shared memory: line l lives at
//   base + (l % inner) * 1 + (l / inner) * plane_stride, element e at + e*es
struct LineMap {
    int nl, inner, plane_stride, es;
    __device__ __forceinline__ int off(int l) const { return (l % inner) + (l / inner) * plane_stride; }
};

// DIT stage of radix R.  m = L/R = span of the sub-transforms being merged.
template <int R, typename C>
__device__ __forceinline__ void dit_stage(C *base, const LineMap lm, int n, int L, int m, const C *tw, int sign,
                                          int tid, int nthr) {
    const int nbf = n / R;
    const int total = lm.nl * nbf;
    const int twstep = n / L;
    for (int t = tid; t < total; t += nthr) {
        const int l = t % lm.nl;
        const int b = t / lm.nl;
        const int blk = b / m, k1 = b - blk * m;
        const int p0 = blk * L + k1;
        C *lp = base + lm.off(l);
        C a[R];
#pragma unroll
        for (int j = 0; j < R; j++) a[j] = lp[(p0 + j * m) * lm.es];
        if (k1 != 0) {
#pragma unroll
            for (int j = 1; j < R; j++) a[j] = cmul(a[j], twid(tw, (j * k1 * twstep) % n, sign));
        }
        SmallDFT<R, C>::run(a, sign, tw, n);
#pragma unroll
        for (int k = 0; k < R; k++) lp[(p0 + k * m) * lm.es] = a[k];
    }
}

template <int R, typename C>
__device__ __forceinline__ void dif_stage(C *base, const LineMap lm, int n, int L, int m, const C *tw, int sign,
                                          int tid, int nthr) {
    const int nbf = n / R;
    const int total = lm.nl * nbf;
    const int twstep = n / L;
    for (int t = tid; t < total; t += nthr) {
        const int l = t % lm.nl;
        const int b = t / lm.nl;
        const int blk = b / m, i = b - blk * m;
        const int p0 = blk * L + i;
        C *lp = base + lm.off(l);
        C a[R];
#pragma unroll
        for (int j = 0; j < R; j++) a[j] = lp[(p0 + j * m) * lm.es];
        SmallDFT<R, C>::run(a, sign, tw, n);
        if (i != 0) {
#pragma unroll
            for (int k = 1; k < R; k++) a[k] = cmul(a[k], twid(tw, (k * i * twstep) % n, sign));
        }
#pragma unroll
        for (int k = 0; k < R; k++) lp[(p0 + k * m) * lm.es] = a[k];
    }
}

// Generic prime radix (direct DFT through the twiddle table), used for
// factors other than 2, 3, 4, 5, 8 (e.g. 7, 23, 31 in the reference's tests).
template <typename C>
__device__ void generic_stage(bool dit, int R, C *base, const LineMap lm, int n, int L, int m, const C *tw,
                              int sign, int tid, int nthr) {
    const int nbf = n / R;
    const int total = lm.nl * nbf;
    const int twstep = n / L;
    const int wstep = n / R;
    for (int t = tid; t < total; t += nthr) {
        const int l = t % lm.nl;
        const int b = t / lm.nl;
        const int blk = b / m, k1 = b - blk * m;
        const int p0 = blk * L + k1;
        C *lp = base + lm.off(l);
        C a[LFTS_MAX_RADIX], o[LFTS_MAX_RADIX];
        for (int j = 0; j < R; j++) {
            a[j] = lp[(p0 + j * m) * lm.es];
            if (dit && k1 != 0 && j != 0) a[j] = cmul(a[j], twid(tw, (j * k1 * twstep) % n, sign));
        }
        for (int k = 0; k < R; k++) {
            C acc = a[0];
            for (int j = 1; j < R; j++) acc = cadd(acc, cmul(a[j], twid(tw, wstep * ((j * k) % R), sign)));
            if (!dit && k1 != 0 && k != 0) acc = cmul(acc, twid(tw, (k * k1 * twstep) % n, sign));
            o[k] = acc;
        }
        for (int k = 0; k < R; k++) lp[(p0 + k * m) * lm.es] = o[k];
    }
}

// Full in-place DIT over all lines (input at perm positions -> natural).
// BLOCK_SYNC: __syncthreads between stages (block-wide lines) or __syncwarp
// (warp-private lines).  GEN: compile the direct-DFT path for prime factors
// other than 2, 3, 5 (kernels for grids without such factors leave it out and
// carry no per-thread scratch frame).
template <typename C, bool BLOCK_SYNC, bool GEN>
__device__ void dit_lines(C *base, const LineMap lm, const AxisPlan &ap, const C *tw, int sign, int tid, int nthr) {
    const int n = ap.n;
    int L = 1;
    for (int s = ap.nf - 1; s >= 0; s--) {
        const int R = ap.radix[s];
        const int m = L;
        L *= R;
        switch (R) {
            case 2: dit_stage<2, C>(base, lm, n, L, m, tw, sign, tid, nthr); break;
            case 3: dit_stage<3, C>(base, lm, n, L, m, tw, sign, tid, nthr); break;
            case 4: dit_stage<4, C>(base, lm, n, L, m, tw, sign, tid, nthr); break;
            case 5: dit_stage<5, C>(base, lm, n, L, m, tw, sign, tid, nthr); break;
            case 8: dit_stage<8, C>(base, lm, n, L, m, tw, sign, tid, nthr); break;
            default: if (GEN) generic_stage<C>(true, R, base, lm, n, L, m, tw, sign, tid, nthr); break;
        }
        if (BLOCK_SYNC) __syncthreads(); else __syncwarp();
    }
}

// Full in-place DIF over all lines (natural -> output at perm positions).
template <typename C, bool BLOCK_SYNC, bool GEN>
__device__ void dif_lines(C *base, const LineMap lm, const AxisPlan &ap, const C *tw, int sign, int tid, int nthr) {
    const int n = ap.n;
    int L = n;
    for (int s = 0; s < ap.nf; s++) {
        const int R = ap.radix[s];
        const int m = L / R;
        switch (R) {
            case 2: dif_stage<2, C>(base, lm, n, L, m, tw, sign, tid, nthr); break;
            case 3: dif_stage<3, C>(base, lm, n, L, m, tw, sign, tid, nthr); break;
            case 4: dif_stage<4, C>(base, lm, n, L, m, tw, sign, tid, nthr); break;
            case 5: dif_stage<5, C>(base, lm, n, L, m, tw, sign, tid, nthr); break;
            case 8: dif_stage<8, C>(base, lm, n, L, m, tw, sign, tid, nthr); break;
            default: if (GEN) generic_stage<C>(false, R, base, lm, n, L, m, tw, sign, tid, nthr); break;
        }
        L = m;
        if (BLOCK_SYNC) __syncthreads(); else __syncwarp();
    }
}

}  // namespace lfts
