// Fused pseudo-spectral step kernels (sm_100a).
//
// One continuous Richardson step (reference: CudaSolverPseudo.cu:345-412, six
// cuFFT calls and ~12 pointwise kernels) is five launches here, each a single
// pass over HBM:
//   K1 plane_forward<2>  read q, fac          -> zy-spectra of e*q and e_h*q
//   K2 xpass<2>          x-FFT, *b and *b_h, inverse x-FFT (both spectra)
//   K3 plane_mid         inverse zy, *e (= e_h^2), forward zy  (half-step seam)
//   K4 xpass<1>          x-FFT, *b_h, inverse x-FFT
//   K5 plane_inverse<2>  inverse zy of both, q' = (4 e_h v2 - e v1)/3
// The discrete step is K1<1>, K2<1>, K5<1>.  Every kernel handles a batch of
// independent jobs (grid.y), so all propagators of a schedule slot and all
// replicas advance in one launch.
#pragma once
#include "lfts_fft.cuh"
#include "../../include/lfts_b200.h"

namespace lfts {

constexpr int NTHR = 256;
constexpr int NWARP = NTHR / 32;

// factor modes for the real-space multiply
enum { FM_NONE = 0, FM_FAC = 1, FM_FAC_SQ = 2 };

template <typename T>
__device__ __forceinline__ T fac_value(int mode, const T *fac, long long idx) {
    if (mode == FM_NONE) return (T)1;
    T f = fac[idx];
    return mode == FM_FAC ? f : f * f;
}

// shared-memory layout shared by the plane kernels
// Each warp transforms zb z-lines at a time (zl: zb lines of n2 per warp), so
// all 32 lanes have butterflies even when one line has only n2/8 of them.
template <typename C>
struct PlaneSmem {
    C *P, *zl, *zl2, *twy, *twz;
    short *py, *pz;
    __device__ PlaneSmem(unsigned char *raw, int nbr, int n1, int n2, int nzc, bool two_lines, int zb) {
        P = (C *)raw;
        zl = P + nbr * n1 * nzc;
        zl2 = zl + NWARP * zb * n2;
        twy = zl2 + (two_lines ? NWARP * zb * n2 : 0);
        twz = twy + n1;
        py = (short *)(twz + n2);
        pz = py + n1;
    }
    static size_t bytes(int nbr, int n1, int n2, int nzc, bool two_lines, int zb) {
        return sizeof(C) * ((size_t)nbr * n1 * nzc + (size_t)NWARP * zb * n2 * (two_lines ? 2 : 1) + n1 + n2) +
               sizeof(short) * (n1 + n2);
    }
};

template <typename C>
__device__ __forceinline__ void load_plane_tables(const GridPlan &g, PlaneSmem<C> &sm) {
    for (int i = threadIdx.x; i < g.n1; i += NTHR) { sm.twy[i] = ((const C *)g.tw[1])[i]; sm.py[i] = g.perm[1][i]; }
    for (int i = threadIdx.x; i < g.n2; i += NTHR) { sm.twz[i] = ((const C *)g.tw[2])[i]; sm.pz[i] = g.perm[2][i]; }
}

// Separate the transform Z of (a + i b) into the half spectra of a and b.
template <typename C>
__device__ __forceinline__ void split_pair(C zk, C zn_conj, C &A, C &B) {
    A.x = (zk.x + zn_conj.x) * 0.5f;
    A.y = (zk.y + zn_conj.y) * 0.5f;
    B.x = (zk.y - zn_conj.y) * 0.5f;
    B.y = -(zk.x - zn_conj.x) * 0.5f;
}

// Hermitian extension of the half spectra A, B of two real rows at full index
// k, packed as Z = A + i B (imaginary parts of DC / Nyquist dropped as c2r does).
template <typename C>
__device__ __forceinline__ C pack_pair(const C *rowA, const C *rowB, int k, int n2, int nzc) {
    C A, B;
    if (k < nzc) {
        A = rowA[k];
        B = rowB ? rowB[k] : cmk<C>(0, 0);
    } else {
        A = cconj(rowA[n2 - k]);
        B = rowB ? cconj(rowB[n2 - k]) : cmk<C>(0, 0);
    }
    if (k == 0 || (2 * k == n2)) { A.y = 0; B.y = 0; }
    C Z;
    Z.x = A.x - B.y;
    Z.y = A.y + B.x;
    return Z;
}

// ------------------------------------------------------------------------
// K1: forward zy transform of one x-plane.  NBR=2: both branches of one input
// (factors fm0, fm1), z-work unit = one row.  NBR=1: z-work unit = row pair.
template <typename T, int NBR, bool GEN>
__global__ void __launch_bounds__(NTHR) k_plane_forward(GridPlan g, const lfts_step_job *__restrict__ jobs, int s,
                                                        int fm0, int fm1, int spec_out0, int zb) {
    using C = typename CT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n1 = g.n1, n2 = g.n2, nzc = g.nzc;
    PlaneSmem<C> sm(smem_raw, NBR, n1, n2, nzc, false, zb);
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    load_plane_tables(g, sm);
    __syncthreads();

    const long long poff = (long long)x * n1 * n2;
    const T *qin = (const T *)jb.in + s * jb.in_stride + poff;
    const T *fac = (const T *)jb.fac;
    const int nunits = (NBR == 2) ? n1 : (n1 + 1) / 2;
    C *zw = sm.zl + warp * zb * n2;
    for (int u0 = warp * zb; u0 < nunits; u0 += NWARP * zb) {
        const int nb = min(zb, nunits - u0);
        for (int b = 0; b < nb; b++) {
            const int u = u0 + b;
            const int ya = (NBR == 2) ? u : 2 * u;
            const int yb = (NBR == 2) ? u : 2 * u + 1;
            const bool hasb = (NBR == 2) || (yb < n1);
            for (int t = lane; t < n2; t += 32) {
                const long long ia = poff + (long long)ya * n2 + t;
                const T qa = qin[ya * n2 + t];
                T va, vb;
                if (NBR == 2) {
                    va = qa * fac_value(fm0, fac, ia);
                    vb = qa * fac_value(fm1, fac, ia);
                } else {
                    va = qa * fac_value(fm0, fac, ia);
                    vb = hasb ? qin[yb * n2 + t] * fac_value(fm0, fac, ia + n2) : (T)0;
                }
                C z;
                z.x = va;
                z.y = vb;
                zw[b * n2 + sm.pz[t]] = z;
            }
        }
        __syncwarp();
        const LineMap lmz = {nb, 1, n2, 1};
        dit_lines<C, false, GEN>(zw, lmz, g.ax[2], sm.twz, -1, lane, 32);
        for (int b = 0; b < nb; b++) {
            const int u = u0 + b;
            const int ya = (NBR == 2) ? u : 2 * u;
            const int yb = (NBR == 2) ? u : 2 * u + 1;
            const bool hasb = (NBR == 2) || (yb < n1);
            const int pb = (NBR == 2) ? 1 : 0;
            C *rowA = sm.P + (size_t)sm.py[ya] * nzc;
            C *rowB = sm.P + (size_t)pb * n1 * nzc + (size_t)sm.py[yb < n1 ? yb : ya] * nzc;
            const C *z = zw + b * n2;
            for (int k = lane; k < nzc; k += 32) {
                C A, B;
                split_pair(z[k], cconj(z[k == 0 ? 0 : n2 - k]), A, B);
                rowA[k] = A;
                if (hasb) rowB[k] = B;
            }
        }
        __syncwarp();
    }
    __syncthreads();
    const LineMap lmy = {NBR * nzc, nzc, n1 * nzc, nzc};
    dit_lines<C, true, GEN>(sm.P, lmy, g.ax[1], sm.twy, -1, tid, NTHR);
    for (int b = 0; b < NBR; b++) {
        C *out = (C *)jb.spec + (size_t)(spec_out0 + b) * g.Mc + (size_t)x * n1 * nzc;
        const C *src = sm.P + (size_t)b * n1 * nzc;
        for (int i = tid; i < n1 * nzc; i += NTHR) out[i] = src[i];
    }
}

// ------------------------------------------------------------------------
// K2/K4: x-transform of a tile of TJ (y, kz) columns, bond multiply, inverse.
// bsel[b] selects the bond table of branch b: 0 = bond, 1 = bond_half.
template <typename T, int NBR, bool GEN>
__global__ void __launch_bounds__(NTHR) k_xpass(GridPlan g, const lfts_step_job *__restrict__ jobs, int spec_in0,
                                                int bsel0, int bsel1, int TJ) {
    using C = typename CT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n0 = g.n0;
    C *tile = (C *)smem_raw;
    C *twx = tile + NBR * n0 * TJ;
    short *px = (short *)(twx + n0);
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int tid = threadIdx.x;
    for (int i = tid; i < n0; i += NTHR) { twx[i] = ((const C *)g.tw[0])[i]; px[i] = g.perm[0][i]; }
    __syncthreads();
    const long long plane = (long long)g.n1 * g.nzc;
    const long long j0 = (long long)blockIdx.x * TJ;
    const int tot = NBR * n0 * TJ;
    const C *spec = (const C *)jb.spec;
    for (int i = tid; i < tot; i += NTHR) {
        const int jj = i % TJ, x = (i / TJ) % n0, b = i / (TJ * n0);
        C v = cmk<C>(0, 0);
        if (j0 + jj < plane) v = spec[(size_t)(spec_in0 + b) * g.Mc + x * plane + j0 + jj];
        tile[(b * n0 + px[x]) * TJ + jj] = v;
    }
    __syncthreads();
    const LineMap lmx = {NBR * TJ, TJ, n0 * TJ, TJ};
    dit_lines<C, true, GEN>(tile, lmx, g.ax[0], twx, -1, tid, NTHR);
    const T *bt0 = (const T *)(bsel0 ? jb.bond_half : jb.bond);
    const T *bt1 = (const T *)(bsel1 ? jb.bond_half : jb.bond);
    for (int i = tid; i < tot; i += NTHR) {
        const int jj = i % TJ, x = (i / TJ) % n0, b = i / (TJ * n0);
        if (j0 + jj < plane) {
            const T bv = (b == 0 ? bt0 : bt1)[x * plane + j0 + jj];
            C &v = tile[(b * n0 + x) * TJ + jj];
            v.x *= bv;
            v.y *= bv;
        }
    }
    __syncthreads();
    dif_lines<C, true, GEN>(tile, lmx, g.ax[0], twx, +1, tid, NTHR);
    C *specw = (C *)jb.spec;
    for (int i = tid; i < tot; i += NTHR) {
        const int jj = i % TJ, x = (i / TJ) % n0, b = i / (TJ * n0);
        if (j0 + jj < plane) specw[(size_t)(spec_in0 + b) * g.Mc + x * plane + j0 + jj] = tile[(b * n0 + px[x]) * TJ + jj];
    }
}

// Forward x-transform only (no bond factor, no inverse) of one spectrum slot:
// completes the r2c 3D transform that k_plane_forward<T, 1> began.
template <typename T, bool GEN>
__global__ void __launch_bounds__(NTHR) k_xpass_forward(GridPlan g, const lfts_step_job *__restrict__ jobs, int spec_in0,
                                                        int TJ) {
    using C = typename CT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n0 = g.n0;
    C *tile = (C *)smem_raw;
    C *twx = tile + n0 * TJ;
    short *px = (short *)(twx + n0);
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int tid = threadIdx.x;
    for (int i = tid; i < n0; i += NTHR) { twx[i] = ((const C *)g.tw[0])[i]; px[i] = g.perm[0][i]; }
    __syncthreads();
    const long long plane = (long long)g.n1 * g.nzc;
    const long long j0 = (long long)blockIdx.x * TJ;
    const int tot = n0 * TJ;
    C *spec = (C *)jb.spec + (size_t)spec_in0 * g.Mc;
    for (int i = tid; i < tot; i += NTHR) {
        const int jj = i % TJ, x = i / TJ;
        C v = cmk<C>(0, 0);
        if (j0 + jj < plane) v = spec[x * plane + j0 + jj];
        tile[px[x] * TJ + jj] = v;
    }
    __syncthreads();
    const LineMap lmx = {TJ, TJ, n0 * TJ, TJ};
    dit_lines<C, true, GEN>(tile, lmx, g.ax[0], twx, -1, tid, NTHR);
    for (int i = tid; i < tot; i += NTHR) {
        const int jj = i % TJ, x = i / TJ;
        if (j0 + jj < plane) spec[x * plane + j0 + jj] = tile[x * TJ + jj];
    }
}

// inverse y transform of NBR planes loaded from spec (natural -> perm rows)
template <typename T, int NBR, bool GEN>
__device__ __forceinline__ void load_and_inverse_y(const GridPlan &g, const lfts_step_job &jb, int spec_in0,
                                                   PlaneSmem<typename CT<T>::type> &sm) {
    using C = typename CT<T>::type;
    const int n1 = g.n1, nzc = g.nzc, x = blockIdx.x;
    for (int b = 0; b < NBR; b++) {
        const C *src = (const C *)jb.spec + (size_t)(spec_in0 + b) * g.Mc + (size_t)x * n1 * nzc;
        C *dst = sm.P + (size_t)b * n1 * nzc;
        for (int i = threadIdx.x; i < n1 * nzc; i += NTHR) dst[i] = src[i];
    }
    __syncthreads();
    const LineMap lmy = {NBR * nzc, nzc, n1 * nzc, nzc};
    dif_lines<C, true, GEN>(sm.P, lmy, g.ax[1], sm.twy, +1, threadIdx.x, NTHR);
}

// ------------------------------------------------------------------------
// K3: half-step seam of the continuous step: inverse zy, multiply by
// e = fac^2 (exp(-w ds/4)^2 = exp(-w ds/2)), forward zy, in place on spec slot.
template <typename T, bool GEN>
__global__ void __launch_bounds__(NTHR) k_plane_mid(GridPlan g, const lfts_step_job *__restrict__ jobs, int spec_idx,
                                                    int zb) {
    using C = typename CT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n1 = g.n1, n2 = g.n2, nzc = g.nzc;
    PlaneSmem<C> sm(smem_raw, 1, n1, n2, nzc, true, zb);
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    load_plane_tables(g, sm);
    __syncthreads();
    load_and_inverse_y<T, 1, GEN>(g, jb, spec_idx, sm);
    __syncthreads();
    const T *fac = (const T *)jb.fac;
    const long long poff = (long long)x * n1 * n2;
    C *zw = sm.zl + warp * zb * n2;
    C *zw2 = sm.zl2 + warp * zb * n2;
    const int nunits = (n1 + 1) / 2;
    for (int u0 = warp * zb; u0 < nunits; u0 += NWARP * zb) {
        const int nb = min(zb, nunits - u0);
        const LineMap lmz = {nb, 1, n2, 1};
        for (int b = 0; b < nb; b++) {
            const int ya = 2 * (u0 + b), yb = ya + 1;
            const C *rowA = sm.P + (size_t)sm.py[ya] * nzc;
            const C *rowB = yb < n1 ? sm.P + (size_t)sm.py[yb] * nzc : nullptr;
            for (int k = lane; k < n2; k += 32) zw[b * n2 + sm.pz[k]] = pack_pair(rowA, rowB, k, n2, nzc);
        }
        __syncwarp();
        dit_lines<C, false, GEN>(zw, lmz, g.ax[2], sm.twz, +1, lane, 32);
        for (int b = 0; b < nb; b++) {
            const int ya = 2 * (u0 + b), yb = ya + 1;
            const bool hasb = yb < n1;
            for (int t = lane; t < n2; t += 32) {
                const C z = zw[b * n2 + t];
                C v;
                v.x = z.x * fac_value(FM_FAC_SQ, fac, poff + (long long)ya * n2 + t);
                v.y = hasb ? z.y * fac_value(FM_FAC_SQ, fac, poff + (long long)yb * n2 + t) : (T)0;
                zw2[b * n2 + sm.pz[t]] = v;
            }
        }
        __syncwarp();
        dit_lines<C, false, GEN>(zw2, lmz, g.ax[2], sm.twz, -1, lane, 32);
        for (int b = 0; b < nb; b++) {
            const int ya = 2 * (u0 + b), yb = ya + 1;
            const bool hasb = yb < n1;
            C *rowA = sm.P + (size_t)sm.py[ya] * nzc;
            C *rowB = hasb ? sm.P + (size_t)sm.py[yb] * nzc : nullptr;
            const C *z = zw2 + b * n2;
            for (int k = lane; k < nzc; k += 32) {
                C A, B;
                split_pair(z[k], cconj(z[k == 0 ? 0 : n2 - k]), A, B);
                rowA[k] = A;
                if (hasb) rowB[k] = B;
            }
        }
        __syncwarp();
    }
    __syncthreads();
    const LineMap lmy = {nzc, nzc, n1 * nzc, nzc};
    dit_lines<C, true, GEN>(sm.P, lmy, g.ax[1], sm.twy, -1, tid, NTHR);
    C *out = (C *)jb.spec + (size_t)spec_idx * g.Mc + (size_t)x * n1 * nzc;
    for (int i = tid; i < n1 * nzc; i += NTHR) out[i] = sm.P[i];
}

// ------------------------------------------------------------------------
// K5: inverse zy of NBR planes with the step epilogue.
//   EPI_SCALE (NBR=1): out = v * factor(fm0)              (discrete / half bond)
//   EPI_RICH  (NBR=2): out = (4 e_h v_half - e v_full)/3   (Richardson)
//   EPI_RICH_ACC (NBR=1, branch 2 only): out = (4 e_h v - out)/3, where out
//                      already holds e v_full (large-plane fallback)
enum { EPI_SCALE = 0, EPI_RICH = 1, EPI_RICH_ACC = 2 };

template <typename T, int NBR, int EPI, bool GEN>
__global__ void __launch_bounds__(NTHR) k_plane_inverse(GridPlan g, const lfts_step_job *__restrict__ jobs, int s,
                                                        int spec_in0, int fm0, int zb) {
    using C = typename CT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n1 = g.n1, n2 = g.n2, nzc = g.nzc;
    PlaneSmem<C> sm(smem_raw, NBR, n1, n2, nzc, false, zb);
    const lfts_step_job jb = jobs[blockIdx.y];
    if (jb.active && !jb.active[jb.replica]) return;
    const int x = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    load_plane_tables(g, sm);
    __syncthreads();
    load_and_inverse_y<T, NBR, GEN>(g, jb, spec_in0, sm);
    __syncthreads();
    const T *fac = (const T *)jb.fac;
    const long long poff = (long long)x * n1 * n2;
    T *qout = (T *)jb.out + s * jb.out_stride + poff;
    C *zw = sm.zl + warp * zb * n2;
    const int nunits = (NBR == 2) ? n1 : (n1 + 1) / 2;
    for (int u0 = warp * zb; u0 < nunits; u0 += NWARP * zb) {
        const int nb = min(zb, nunits - u0);
        for (int b = 0; b < nb; b++) {
            const int u = u0 + b;
            const int ya = (NBR == 2) ? u : 2 * u;
            const int yb = (NBR == 2) ? u : 2 * u + 1;
            const bool hasb = (NBR == 2) || (yb < n1);
            const C *rowA = sm.P + (size_t)sm.py[ya] * nzc;
            const C *rowB = (NBR == 2) ? sm.P + (size_t)n1 * nzc + (size_t)sm.py[ya] * nzc
                                       : (hasb ? sm.P + (size_t)sm.py[yb] * nzc : nullptr);
            for (int k = lane; k < n2; k += 32) zw[b * n2 + sm.pz[k]] = pack_pair(rowA, rowB, k, n2, nzc);
        }
        __syncwarp();
        const LineMap lmz = {nb, 1, n2, 1};
        dit_lines<C, false, GEN>(zw, lmz, g.ax[2], sm.twz, +1, lane, 32);
        for (int b = 0; b < nb; b++) {
            const int u = u0 + b;
            const int ya = (NBR == 2) ? u : 2 * u;
            const int yb = (NBR == 2) ? u : 2 * u + 1;
            const bool hasb = (NBR == 2) || (yb < n1);
            for (int t = lane; t < n2; t += 32) {
                const C z = zw[b * n2 + t];
                const long long ia = poff + (long long)ya * n2 + t;
                if (EPI == EPI_RICH) {
                    const T eh = fac[ia];
                    qout[ya * n2 + t] = ((T)4 * eh * z.y - eh * eh * z.x) / (T)3;
                } else if (EPI == EPI_RICH_ACC) {
                    const T eh = fac[ia];
                    qout[ya * n2 + t] = ((T)4 * eh * z.x - qout[ya * n2 + t]) / (T)3;
                    if (hasb) {
                        const T ehb = fac[ia + n2];
                        qout[yb * n2 + t] = ((T)4 * ehb * z.y - qout[yb * n2 + t]) / (T)3;
                    }
                } else {
                    qout[ya * n2 + t] = z.x * fac_value(fm0, fac, ia);
                    if (hasb) qout[yb * n2 + t] = z.y * fac_value(fm0, fac, ia + n2);
                }
            }
        }
        __syncwarp();
    }
}

}  // namespace lfts
