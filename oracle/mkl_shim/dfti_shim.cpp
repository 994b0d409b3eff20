/*
 * Oracle infrastructure (test-only; never linked into the product).
 *
 * Project-written FP64 FFT behind the MKL-DFTI stand-in, so that the reference
 * CPU platform (src/platforms/cpu/MklFFT{1,2,3}D.cpp) compiles and runs
 * unchanged here.  Semantics follow what those files configure:
 *   forward : real [n0][n1]..[nd-1] -> complex [n0]..[nd-1/2+1] (r2c, unscaled)
 *   backward: complex half spectrum -> real (c2r, unscaled; MklFFT*D divides
 *             by the grid size itself, MklFFT3D.cpp:77-78)
 *
 * Algorithm (own restatement of textbook methods):
 *   - complex transforms use a mixed-radix Stockham auto-sort decimation in
 *     frequency, radices 4 and 2 hand-coded and any other prime by a direct
 *     small DFT, twiddles hoisted out of the inner loop.  A strided axis of a row-major array is transformed in place
 *     of its layout: element i of column q sits at q + B*i, which is exactly
 *     the interleaved form Stockham works on, so no transposes are needed.
 *   - the last (contiguous) axis is real: two real rows a, b are packed into
 *     one complex row a + i b (16 such pairs at a time, interleaved, so the
 *     same Stockham inner loop runs over them), transformed once, and separated with
 *     A[k] = (Z[k] + conj Z[n-k])/2, B[k] = (Z[k] - conj Z[n-k])/(2i).
 *     The inverse rebuilds Z = A + iB from the Hermitian halves (imaginary
 *     parts of the DC and Nyquist bins are dropped, as a c2r transform does).
 */
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <vector>

#include "mkl_dfti.h"
#include "mkl_service.h"

namespace {

struct cpx {
    double re, im;
};
inline cpx cadd(cpx a, cpx b) { return {a.re + b.re, a.im + b.im}; }
inline cpx csub(cpx a, cpx b) { return {a.re - b.re, a.im - b.im}; }
inline cpx cmul(cpx a, cpx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cpx cconj(cpx a) { return {a.re, -a.im}; }

struct Plan1D {
    int n = 0;
    std::vector<int> radices;
    std::vector<cpx> tw;  // tw[j] = exp(-2 pi i j / n)

    explicit Plan1D(int n_) : n(n_) {
        int m = n;
        while (m % 4 == 0) { radices.push_back(4); m /= 4; }
        while (m % 2 == 0) { radices.push_back(2); m /= 2; }
        for (int p = 3; m > 1; p += 2) {
            while (m % p == 0) { radices.push_back(p); m /= p; }
        }
        tw.resize(n);
        for (int j = 0; j < n; j++) {
            // angles reduced to [0, 2pi) exactly through the integer j
            double a = -2.0 * M_PI * (double)j / (double)n;
            tw[j] = {std::cos(a), std::sin(a)};
        }
    }
    // w_n^e for the forward sign; sign=+1 flips to the conjugate
    inline cpx w(long e, int sign) const {
        cpx t = tw[e % n];
        return sign > 0 ? cconj(t) : t;
    }
};

// One Stockham DIF pass over B interleaved sequences of length n.
// x and y have n*B elements; returns the buffer holding the result.
cpx *stockham(const Plan1D &p, long B, cpx *x, cpx *y, int sign) {
    const int N = p.n;
    long s = B;
    int ncur = N;
    for (int r : p.radices) {
        const int m = ncur / r;
        const long stride_tw = N / ncur;  // w_ncur^e = w_N^(e*stride_tw)
        // small-DFT matrix w_r^(jk) for generic radices
        std::vector<cpx> wr((size_t)r * r);
        for (int j = 0; j < r; j++)
            for (int k = 0; k < r; k++) wr[(size_t)j * r + k] = p.w((long)(N / r) * ((j * k) % r), sign);
        std::vector<cpx> twk(r), a(r), b(r);
        for (int pp = 0; pp < m; pp++) {
            for (int k = 0; k < r; k++) twk[k] = p.w((long)pp * k * stride_tw, sign);
            const cpx *xs = x + s * pp;
            cpx *ys = y + s * (long)r * pp;
            if (r == 2) {
                const cpx t1 = twk[1];
                for (long q = 0; q < s; q++) {
                    const cpx a0 = xs[q], a1 = xs[q + s * m];
                    ys[q] = cadd(a0, a1);
                    ys[q + s] = cmul(csub(a0, a1), t1);
                }
            } else if (r == 4) {
                const cpx t1 = twk[1], t2 = twk[2], t3 = twk[3];
                for (long q = 0; q < s; q++) {
                    const cpx a0 = xs[q], a1 = xs[q + s * m], a2 = xs[q + 2 * s * m], a3 = xs[q + 3 * s * m];
                    const cpx u0 = cadd(a0, a2), u1 = csub(a0, a2), u2 = cadd(a1, a3), d = csub(a1, a3);
                    const cpx u3 = sign < 0 ? cpx{d.im, -d.re} : cpx{-d.im, d.re};
                    ys[q] = cadd(u0, u2);
                    ys[q + s] = cmul(cadd(u1, u3), t1);
                    ys[q + 2 * s] = cmul(csub(u0, u2), t2);
                    ys[q + 3 * s] = cmul(csub(u1, u3), t3);
                }
            } else {
                for (long q = 0; q < s; q++) {
                    for (int j = 0; j < r; j++) a[j] = xs[q + s * (long)j * m];
                    for (int k = 0; k < r; k++) {
                        cpx acc = a[0];
                        for (int j = 1; j < r; j++) acc = cadd(acc, cmul(a[j], wr[(size_t)j * r + k]));
                        b[k] = acc;
                    }
                    for (int k = 0; k < r; k++) ys[q + s * k] = k ? cmul(b[k], twk[k]) : b[k];
                }
            }
        }
        cpx *t = x; x = y; y = t;
        s *= r;
        ncur = m;
    }
    return x;
}

struct Descriptor {
    int dim = 0;
    long len[3] = {1, 1, 1};
    bool committed = false;
    std::vector<Plan1D> plans;  // one per axis
};

// Transform axis `ax` (complex, not the last real axis) of a complex array of
// shape cshape[0..dim-1] in place, using `work` as scratch.
void c2c_axis(const Descriptor &d, const long *cshape, int ax, cpx *data, std::vector<cpx> &work, int sign) {
    long outer = 1, inner = 1;
    for (int i = 0; i < ax; i++) outer *= cshape[i];
    for (int i = ax + 1; i < d.dim; i++) inner *= cshape[i];
    const long n = cshape[ax];
    const long block = n * inner;
    work.resize(block);
    for (long o = 0; o < outer; o++) {
        cpx *x = data + o * block;
        cpx *res = stockham(d.plans[ax], inner, x, work.data(), sign);
        if (res != x) std::memcpy(x, res, sizeof(cpx) * block);
    }
}

constexpr long GROUP = 16;  // row pairs transformed together as interleaved columns

void forward(const Descriptor &d, const double *in, cpx *out) {
    const long nz = d.len[d.dim - 1];
    const long nzc = nz / 2 + 1;
    long rows = 1;
    for (int i = 0; i < d.dim - 1; i++) rows *= d.len[i];
    const Plan1D &pz = d.plans[d.dim - 1];
    const long pairs = (rows + 1) / 2;
    std::vector<cpx> zl(nz * GROUP), wk(nz * GROUP);
    for (long g0 = 0; g0 < pairs; g0 += GROUP) {
        const long G = std::min(GROUP, pairs - g0);
        for (long g = 0; g < G; g++) {
            const long r = 2 * (g0 + g);
            const double *ra = in + r * nz;
            const double *rb = (r + 1 < rows) ? in + (r + 1) * nz : nullptr;
            for (long t = 0; t < nz; t++) zl[t * G + g] = {ra[t], rb ? rb[t] : 0.0};
        }
        cpx *Z = stockham(pz, G, zl.data(), wk.data(), -1);
        for (long g = 0; g < G; g++) {
            const long r = 2 * (g0 + g);
            const bool pair = r + 1 < rows;
            for (long k = 0; k < nzc; k++) {
                cpx zk = Z[k * G + g], zn = cconj(Z[((nz - k) % nz) * G + g]);
                out[r * nzc + k] = {0.5 * (zk.re + zn.re), 0.5 * (zk.im + zn.im)};
                if (pair) out[(r + 1) * nzc + k] = {0.5 * (zk.im - zn.im), -0.5 * (zk.re - zn.re)};
            }
        }
    }
    long cshape[3];
    for (int i = 0; i < d.dim; i++) cshape[i] = d.len[i];
    cshape[d.dim - 1] = nzc;
    std::vector<cpx> work;
    for (int ax = d.dim - 2; ax >= 0; ax--) c2c_axis(d, cshape, ax, out, work, -1);
}

void backward(const Descriptor &d, const cpx *in, double *out) {
    const long nz = d.len[d.dim - 1];
    const long nzc = nz / 2 + 1;
    long rows = 1;
    for (int i = 0; i < d.dim - 1; i++) rows *= d.len[i];
    long cshape[3];
    for (int i = 0; i < d.dim; i++) cshape[i] = d.len[i];
    cshape[d.dim - 1] = nzc;
    std::vector<cpx> buf(in, in + rows * nzc);
    std::vector<cpx> work;
    for (int ax = 0; ax <= d.dim - 2; ax++) c2c_axis(d, cshape, ax, buf.data(), work, +1);
    const Plan1D &pz = d.plans[d.dim - 1];
    const long pairs = (rows + 1) / 2;
    std::vector<cpx> zl(nz * GROUP), wk(nz * GROUP);
    for (long g0 = 0; g0 < pairs; g0 += GROUP) {
        const long G = std::min(GROUP, pairs - g0);
        for (long g = 0; g < G; g++) {
            const long r = 2 * (g0 + g);
            const bool pair = (r + 1 < rows);
            for (long k = 0; k < nz; k++) {
                cpx a, b = {0.0, 0.0};
                if (k < nzc) {
                    a = buf[r * nzc + k];
                    if (pair) b = buf[(r + 1) * nzc + k];
                } else {
                    a = cconj(buf[r * nzc + (nz - k)]);
                    if (pair) b = cconj(buf[(r + 1) * nzc + (nz - k)]);
                }
                if (k == 0 || (nz % 2 == 0 && k == nz / 2)) { a.im = 0.0; b.im = 0.0; }
                zl[k * G + g] = {a.re - b.im, a.im + b.re};  // Z = a + i b
            }
        }
        cpx *z = stockham(pz, G, zl.data(), wk.data(), +1);
        for (long g = 0; g < G; g++) {
            const long r = 2 * (g0 + g);
            const bool pair = (r + 1 < rows);
            for (long t = 0; t < nz; t++) {
                out[r * nz + t] = z[t * G + g].re;
                if (pair) out[(r + 1) * nz + t] = z[t * G + g].im;
            }
        }
    }
}

}  // namespace

struct lfts_dfti_descriptor : Descriptor {};

extern "C" {

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE *handle, enum DFTI_CONFIG_VALUE precision,
                              enum DFTI_CONFIG_VALUE domain, MKL_LONG dimension, ...) {
    if (precision != DFTI_DOUBLE || domain != DFTI_REAL || dimension < 1 || dimension > 3) return 1;
    auto *d = new lfts_dfti_descriptor();
    d->dim = (int)dimension;
    va_list ap;
    va_start(ap, dimension);
    if (dimension == 1) {
        d->len[0] = va_arg(ap, MKL_LONG);
    } else {
        const MKL_LONG *l = va_arg(ap, const MKL_LONG *);
        for (int i = 0; i < dimension; i++) d->len[i] = l[i];
    }
    va_end(ap);
    for (int i = 0; i < d->dim; i++) {
        if (d->len[i] < 1) { delete d; return 2; }
        d->plans.emplace_back((int)d->len[i]);
    }
    *handle = d;
    return 0;
}

MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE handle, enum DFTI_CONFIG_PARAM param, ...) {
    if (!handle) return 1;
    va_list ap;
    va_start(ap, param);
    MKL_LONG status = 0;
    if (param == DFTI_PLACEMENT) {
        int v = va_arg(ap, int);
        if (v != DFTI_NOT_INPLACE) status = 3;
    } else if (param == DFTI_CONJUGATE_EVEN_STORAGE) {
        int v = va_arg(ap, int);
        if (v != DFTI_COMPLEX_COMPLEX) status = 3;
    } else if (param == DFTI_INPUT_STRIDES || param == DFTI_OUTPUT_STRIDES) {
        // Only the default contiguous row-major layout is supported; check it.
        const MKL_LONG *st = va_arg(ap, const MKL_LONG *);
        const int dim = handle->dim;
        bool real_side = (param == DFTI_INPUT_STRIDES);  // forward descriptors; backward swaps
        // Accept either the real or the complex contiguous layout.
        MKL_LONG expect_r = 1, expect_c = 1;
        bool ok_r = st[0] == 0, ok_c = st[0] == 0;
        for (int i = dim; i >= 1; i--) {
            ok_r = ok_r && st[i] == expect_r;
            ok_c = ok_c && st[i] == expect_c;
            expect_r *= handle->len[i - 1];
            expect_c *= (i == dim) ? (handle->len[i - 1] / 2 + 1) : handle->len[i - 1];
        }
        (void)real_side;
        if (!(ok_r || ok_c)) status = 4;
    } else {
        status = 5;
    }
    va_end(ap);
    return status;
}

MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE handle) {
    if (!handle) return 1;
    handle->committed = true;
    return 0;
}

MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE handle, void *in, ...) {
    if (!handle || !handle->committed) return 1;
    va_list ap;
    va_start(ap, in);
    void *out = va_arg(ap, void *);
    va_end(ap);
    forward(*handle, (const double *)in, (cpx *)out);
    return 0;
}

MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE handle, void *in, ...) {
    if (!handle || !handle->committed) return 1;
    va_list ap;
    va_start(ap, in);
    void *out = va_arg(ap, void *);
    va_end(ap);
    backward(*handle, (const cpx *)in, (double *)out);
    return 0;
}

MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE *handle) {
    if (!handle) return 1;
    delete *handle;
    *handle = nullptr;
    return 0;
}

void mkl_get_version(MKLVersion *v) {
    v->MajorVersion = 0;
    v->MinorVersion = 0;
    v->UpdateVersion = 0;
    v->ProductStatus = "langevinfts-b200 oracle FFT shim (not Intel MKL)";
    v->Build = "project-written FP64 mixed-radix FFT";
    v->Processor = "generic";
    v->Platform = "x86_64";
}

}  // extern "C"
