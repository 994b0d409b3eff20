// Periodic 3D convolution for the learned saddle-point start (U-Net), as an
// implicit GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
//   out[p][co] = act(bias[co] + sum_{tap, ci} w[tap][co][ci] in[p + tap][ci])
//
// Activations are channels-last BF16 ([B][D][H][W][C], C a multiple of 16),
// the box is periodic (p + tap wraps), accumulation is FP32 in tensor memory.
// One CTA of 128 threads owns 128 consecutive output positions (the GEMM's M)
// and all COUT channels (N).  Per tap the threads gather the shifted input
// rows (K = CIN) and copy the tap's packed weights into one of two shared
// stages, in the K-major no-swizzle layout of the MMA: 16-byte core-matrix
// rows, chunk kc of row m at (kc * ROWS + m) * 16 bytes.  Thread 0 issues the
// CIN/16 MMAs of the tap (M = 128, N = COUT, K = 16 each) and commits them to
// the stage's mbarrier; a stage is refilled only after that commit arrived.
// Waits are bounded (lfts_bulk.cuh): a wait that gives up sets the device
// error word, waits once more for the tensor core, frees the tensor memory
// and returns.  Included by lfts_engine.cu (one device error word).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "lfts_bulk.cuh"

namespace lfts {
namespace unet {

constexpr int CONV_M = 128;  // output positions per CTA (MMA M)

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    // K-major, no swizzle: start, leading (K-chunk) and stride (8-row group)
    // byte offsets in 16-byte units; version 1 (bits 46-47)
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 16-byte global -> shared copy that does not wait for the data (cp.async,
// completed by cp_async_wait_all), so a thread keeps many loads in flight
__device__ __forceinline__ void cp_async16(void *dst_smem, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst_smem)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ uint16_t to_bf16(float f) {
    // round to nearest even (finite values; NaN stays NaN)
    uint32_t u = __float_as_uint(f);
    if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)((u >> 16) | ((u & 0xFFFF) ? 0x40 : 0));
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

// in: [npos][cin] BF16 (npos = B*D*H*W), wpk: [taps][cin/8][cout][8] BF16,
// bias: [cout] FP32, out: [npos][cout] BF16.
__global__ void __launch_bounds__(CONV_M) k_conv3d_umma(const uint4 *__restrict__ in, const uint4 *__restrict__ wpk,
                                                        const float *__restrict__ bias, uint16_t *__restrict__ out, int B,
                                                        int D, int H, int W, int cin, int cout, int taps, int relu,
                                                        uint32_t tmem_cols) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int kc_n = cin / 8;                       // 16-byte chunks per row (K / 8)
    const int a_units = kc_n * CONV_M, b_units = kc_n * cout;
    uint4 *stage0 = (uint4 *)smem_raw;              // [2][a_units + b_units] 16-byte units
    uint64_t *bar = (uint64_t *)(stage0 + 2 * (a_units + b_units));
    uint32_t *tmem_slot = (uint32_t *)(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5;
    const long long npos = (long long)B * D * H * W;
    const long long p = (long long)blockIdx.x * CONV_M + tid;
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    // this thread's output position
    int n = 0, z = 0, y = 0, x = 0;
    const bool valid = p < npos;
    if (valid) {
        long long q = p;
        x = (int)(q % W);
        q /= W;
        y = (int)(q % H);
        q /= H;
        z = (int)(q % D);
        n = (int)(q / D);
    }
    // instruction descriptor: FP32 accumulate, BF16 A and B, both K-major, N = cout, M = 128
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(cout >> 3) << 17) | ((uint32_t)(CONV_M >> 4) << 24);
    bool ok = true;
    for (int t = 0; t < taps; t++) {
        const int st = t & 1;
        // every thread takes the same branch: the wait results are combined
        if (t >= 2 && !__syncthreads_and(mbar_wait(bar + st, ((t >> 1) - 1) & 1))) {
            ok = false;
            break;
        }
        uint4 *sa = stage0 + st * (a_units + b_units), *sb = sa + a_units;
        // A: the input row at this position shifted by the tap (periodic)
        {
            uint4 *dst = sa + tid;
            if (valid) {
                int dz = 0, dy = 0, dx = 0;
                if (taps == 27) {
                    dz = t / 9 - 1;
                    dy = (t / 3) % 3 - 1;
                    dx = t % 3 - 1;
                }
                const int zz = (z + dz + D) % D, yy = (y + dy + H) % H, xx = (x + dx + W) % W;
                const uint4 *src = in + ((((long long)n * D + zz) * H + yy) * W + xx) * kc_n;
                for (int kc = 0; kc < kc_n; kc++) cp_async16(dst + kc * CONV_M, src + kc);
            } else {
                for (int kc = 0; kc < kc_n; kc++) dst[kc * CONV_M] = make_uint4(0, 0, 0, 0);
            }
        }
        // B: the tap's packed weights
        {
            const uint4 *src = wpk + (long long)t * b_units;
            for (int i = tid; i < b_units; i += CONV_M) cp_async16(sb + i, src + i);
        }
        cp_async_wait_all();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_addr(sa), b0 = smem_addr(sb);
            for (int s = 0; s < kc_n / 2; s++) {
                const uint64_t da = umma_desc(a0 + (uint32_t)(2 * s * CONV_M * 16), CONV_M * 16, 128);
                const uint64_t db = umma_desc(b0 + (uint32_t)(2 * s * cout * 16), (uint32_t)cout * 16, 128);
                umma_bf16(tmem, da, db, idesc, (t > 0 || s > 0) ? 1u : 0u);
            }
            umma_commit(bar + st);
        }
    }
    {
        const bool fin = ok ? mbar_wait(bar + ((taps - 1) & 1), ((taps - 1) >> 1) & 1) : false;
        ok = __syncthreads_and(fin);
    }
    if (!ok) {
        // give the tensor core a second bounded wait, then release and leave
        mbar_wait(bar + ((taps - 1) & 1), ((taps - 1) >> 1) & 1);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // epilogue: warp w reads accumulator rows 32w..32w+31 (tensor-memory lanes)
        for (int c0 = 0; c0 < cout; c0 += 16) {
            uint32_t v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
            if (valid) {
                uint16_t h[16];
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    float f = __uint_as_float(v[i]) + bias[c0 + i];
                    if (relu && f < 0.f) f = 0.f;
                    h[i] = to_bf16(f);
                }
                uint4 *o = (uint4 *)(out + p * cout + c0);
                o[0] = make_uint4(h[0] | (h[1] << 16), h[2] | (h[3] << 16), h[4] | (h[5] << 16), h[6] | (h[7] << 16));
                o[1] = make_uint4(h[8] | (h[9] << 16), h[10] | (h[11] << 16), h[12] | (h[13] << 16), h[14] | (h[15] << 16));
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
}

// ------------------------------------------------------------------------
// 3x3x3 convolution with the input of a tile staged once: the tile is 1 x 16
// x 8 output positions (z, y, x) and its halo 3 x 18 x 10 positions sits in
// shared memory as planes [kc][zh][yh][xh] of 16-byte units.  For tap (dz, dy,
// dx) the A operand of the MMA is read in place: the 8 output positions of a
// y row map to 8 consecutive halo rows (one core matrix), the 16 y rows are
// HX units apart (SBO), the channel chunks a plane apart (LBO); only the
// tap's weights are copied per tap.  Needs H % 16 == 0 and W % 8 == 0.
constexpr int HT_Y = 16, HT_X = 8, HZ = 3, HY = HT_Y + 2, HX = HT_X + 2, HPLANE = HZ * HY * HX;

// Warp roles after the halo is staged: warps 1-3 copy the tap weights into a
// ring of NS stages (full[st]: 96 producer arrivals), lane 0 of warp 0 issues
// each tap's MMAs once its stage is full and commits them to empty[st], which
// frees the stage; a last commit to bar_done releases the epilogue.
__global__ void __launch_bounds__(CONV_M) k_conv3d_halo_umma(const uint4 *__restrict__ in, const uint4 *__restrict__ wpk,
                                                             const float *__restrict__ bias, uint16_t *__restrict__ out,
                                                             int B, int D, int H, int W, int cin, int cout, int relu,
                                                             uint32_t tmem_cols, int NS) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int kc_n = cin / 8, b_units = kc_n * cout;
    uint4 *halo = (uint4 *)smem_raw;                 // kc_n * HPLANE units
    uint4 *wst = halo + kc_n * HPLANE;               // NS weight stages
    uint64_t *full = (uint64_t *)(wst + (size_t)NS * b_units), *empty = full + NS, *done = empty + NS;
    uint32_t *tmem_slot = (uint32_t *)(done + 1);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int x0 = blockIdx.x * HT_X, y0 = blockIdx.y * HT_Y, z = blockIdx.z % D, n = blockIdx.z / D;
    if (tid == 0) {
        for (int i = 0; i < NS; i++) {
            mbar_init(full + i, CONV_M - 32);
            mbar_init(empty + i, 1);
        }
        mbar_init(done, 1);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // the halo, periodic
    for (int i = tid; i < kc_n * HPLANE; i += CONV_M) {
        const int kc = i / HPLANE, r = i - kc * HPLANE;
        const int zh = r / (HY * HX), yh = (r / HX) % HY, xh = r % HX;
        const int zz = (z + zh - 1 + D) % D, yy = (y0 + yh - 1 + H) % H, xx = (x0 + xh - 1 + W) % W;
        cp_async16(halo + i, in + ((((long long)n * D + zz) * H + yy) * W + xx) * kc_n + kc);
    }
    cp_async_wait_all();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    bool ok = true;
    if (warp > 0) {
        // producers: tap t into stage t % NS once the MMAs of tap t - NS freed it
        const int pt = tid - 32;
        for (int t = 0; t < 27 && ok; t++) {
            const int st = t % NS, u = t / NS;
            if (u > 0 && !mbar_wait(empty + st, (u - 1) & 1)) {
                ok = false;
                break;
            }
            uint4 *sb = wst + (size_t)st * b_units;
            const uint4 *src = wpk + (long long)t * b_units;
            for (int i = pt; i < b_units; i += CONV_M - 32) cp_async16(sb + i, src + i);
            cp_async_wait_all();
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(full + st)) : "memory");
        }
    } else if (tid == 0) {
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(cout >> 3) << 17) | ((uint32_t)(CONV_M >> 4) << 24);
        const uint32_t halo0 = smem_addr(halo);
        for (int t = 0; t < 27; t++) {
            const int st = t % NS, u = t / NS;
            if (!mbar_wait(full + st, u & 1)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;  // halo offsets of the tap (0..2)
            const uint32_t a_tap = halo0 + (uint32_t)(((dz * HY + dy) * HX + dx) * 16);
            const uint32_t b0 = smem_addr(wst + (size_t)st * b_units);
            for (int s = 0; s < kc_n / 2; s++) {
                const uint64_t da = umma_desc(a_tap + (uint32_t)(2 * s * HPLANE * 16), HPLANE * 16, HX * 16);
                const uint64_t db = umma_desc(b0 + (uint32_t)(2 * s * cout * 16), (uint32_t)cout * 16, 128);
                umma_bf16(tmem, da, db, idesc, (t > 0 || s > 0) ? 1u : 0u);
            }
            umma_commit(empty + st);
        }
        if (ok) umma_commit(done);
    }
    {
        // every thread: the accumulator is complete (or some wait gave up)
        const bool fin = __syncthreads_and(ok) ? mbar_wait(done, 0) : false;
        ok = __syncthreads_and(fin);
    }
    if (!ok) {
        mbar_wait(done, 0);  // a second bounded wait for MMAs still in flight
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int m = tid;  // accumulator row = 8 j + l: position (y0 + j, x0 + l)
        const long long p = (((long long)n * D + z) * H + (y0 + m / 8)) * W + (x0 + m % 8);
        for (int c0 = 0; c0 < cout; c0 += 16) {
            uint32_t v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
            uint16_t h[16];
#pragma unroll
            for (int i = 0; i < 16; i++) {
                float f = __uint_as_float(v[i]) + bias[c0 + i];
                if (relu && f < 0.f) f = 0.f;
                h[i] = to_bf16(f);
            }
            uint4 *o = (uint4 *)(out + p * cout + c0);
            o[0] = make_uint4(h[0] | (h[1] << 16), h[2] | (h[3] << 16), h[4] | (h[5] << 16), h[6] | (h[7] << 16));
            o[1] = make_uint4(h[8] | (h[9] << 16), h[10] | (h[11] << 16), h[12] | (h[13] << 16), h[14] | (h[15] << 16));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
}

// ------------------------------------------------------------------------
// Weight gradient of the periodic convolution:
//   dw[tap][co][ci] += sum_p gy[p][co] x[p + tap][ci]
// per tap a GEMM with M = co (padded to 128 rows), N = cin, K = positions.
// Both operands are MN-major in channels-last memory (16 bytes = 8 channels of
// one position), so they are staged without transposition: chunk c of
// position k at (c * WG_K + k) * 16 bytes; 8 consecutive positions form a core
// matrix (LBO = 128 bytes), channel chunks are WG_K * 16 bytes apart (SBO).
// A CTA takes one (kz, ky) row of taps (kx = 0..2; the single tap of a 1x1x1
// kernel) over WG_CHUNK positions, keeps one accumulator per tap in tensor
// memory, and adds them to dw (FP32, zeroed by the caller) with atomics.
constexpr int WG_K = 64;        // positions per stage (4 MMA K-steps)
constexpr int WG_CHUNK = 2048;  // positions per CTA

__global__ void __launch_bounds__(CONV_M) k_conv3d_wgrad_umma(const uint4 *__restrict__ x, const uint4 *__restrict__ gy,
                                                              float *__restrict__ dw, int B, int D, int H, int W, int cin,
                                                              int cout, int taps, uint32_t tmem_cols) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int ntap = taps == 27 ? 3 : 1;
    const int xc = cin / 8, gc = cout / 8;             // 16-byte chunks per position
    const int a_units = 16 * WG_K, b_units = xc * WG_K; // A: 128 rows (16 chunks), B per tap
    const int st_units = a_units + ntap * b_units;
    uint4 *stage0 = (uint4 *)smem_raw;
    uint64_t *bar = (uint64_t *)(stage0 + 2 * st_units);
    uint32_t *tmem_slot = (uint32_t *)(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5;
    const long long npos = (long long)B * D * H * W;
    const long long p0 = (long long)blockIdx.x * WG_CHUNK;
    const int g = blockIdx.y;  // tap row: kz = g / 3, ky = g % 3
    // rows of A beyond cout stay zero in both stages
    for (int i = tid; i < 2 * st_units; i += CONV_M) stage0[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    // M = 128, N = cin, both operands MN-major, FP32 accumulate
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(cin >> 3) << 17) |
                           ((uint32_t)(CONV_M >> 4) << 24);
    const int k = tid & (WG_K - 1), half = tid / WG_K;  // two threads per staged position
    const int nst = WG_CHUNK / WG_K;
    bool ok = true;
    for (int u = 0; u < nst; u++) {
        const int st = u & 1;
        if (u >= 2 && !__syncthreads_and(mbar_wait(bar + st, ((u >> 1) - 1) & 1))) {
            ok = false;
            break;
        }
        uint4 *sa = stage0 + st * st_units, *sb = sa + a_units;
        const long long p = p0 + (long long)u * WG_K + k;
        const bool valid = p < npos;
        int n = 0, z = 0, y = 0, xx = 0;
        if (valid) {
            long long q = p;
            xx = (int)(q % W);
            q /= W;
            y = (int)(q % H);
            q /= H;
            z = (int)(q % D);
            n = (int)(q / D);
        }
        for (int c = half; c < gc; c += 2) {
            if (valid) cp_async16(sa + c * WG_K + k, gy + p * gc + c);
            else sa[c * WG_K + k] = make_uint4(0, 0, 0, 0);
        }
        for (int j = 0; j < ntap; j++) {
            uint4 *dst = sb + j * b_units + k;
            if (valid) {
                int dz = 0, dy = 0, dx = 0;
                if (taps == 27) {
                    dz = g / 3 - 1;
                    dy = g % 3 - 1;
                    dx = j - 1;
                }
                const int zz = (z + dz + D) % D, yy = (y + dy + H) % H, x2 = (xx + dx + W) % W;
                const uint4 *src = x + ((((long long)n * D + zz) * H + yy) * W + x2) * xc;
                for (int c = half; c < xc; c += 2) cp_async16(dst + c * WG_K, src + c);
            } else {
                for (int c = half; c < xc; c += 2) dst[c * WG_K] = make_uint4(0, 0, 0, 0);
            }
        }
        cp_async_wait_all();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_addr(sa), b0 = smem_addr(sb);
            for (int s = 0; s < WG_K / 16; s++) {
                const uint64_t da = umma_desc(a0 + (uint32_t)(16 * s * 16), 128, WG_K * 16);
                for (int j = 0; j < ntap; j++) {
                    const uint64_t db = umma_desc(b0 + (uint32_t)((j * b_units + 16 * s) * 16), 128, WG_K * 16);
                    umma_bf16(tmem + (uint32_t)(j * cin), da, db, idesc, (u > 0 || s > 0) ? 1u : 0u);
                }
            }
            umma_commit(bar + st);
        }
    }
    {
        const bool fin = ok ? mbar_wait(bar + ((nst - 1) & 1), ((nst - 1) >> 1) & 1) : false;
        ok = __syncthreads_and(fin);
    }
    if (!ok) {
        mbar_wait(bar + ((nst - 1) & 1), ((nst - 1) >> 1) & 1);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int co = 32 * warp + (tid & 31);  // accumulator row of this thread
        for (int j = 0; j < ntap; j++) {
            const int tap = taps == 27 ? 3 * g + j : 0;
            for (int c0 = 0; c0 < cin; c0 += 16) {
                uint32_t v[16];
                tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(j * cin + c0), v);
                if (co < cout) {
                    float *o = dw + ((long long)tap * cout + co) * cin + c0;
#pragma unroll
                    for (int i = 0; i < 16; i++) atomicAdd(o + i, __uint_as_float(v[i]));
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
}
}  // namespace unet
}  // namespace lfts

extern "C" int lfts_conv3d_wgrad_bf16(void *stream, const void *x, const void *gy, float *dw, int B, int D, int H, int W,
                                      int cin, int cout, int taps) {
    if (!x || !gy || !dw) return fail("null argument");
    if (B < 1 || D < 1 || H < 1 || W < 1) return fail("conv3d wgrad: extents must be positive");
    if (cin < 16 || cin % 16 || cin > LFTS_CONV_MAX_CIN)
        return fail("conv3d wgrad: cin must be a multiple of 16 up to " + std::to_string(LFTS_CONV_MAX_CIN));
    if (cout < 16 || cout % 16 || cout > LFTS_CONV_MAX_COUT)
        return fail("conv3d wgrad: cout must be a multiple of 16 up to " + std::to_string(LFTS_CONV_MAX_COUT));
    if (taps != 1 && taps != 27) return fail("conv3d wgrad: taps must be 1 or 27");
    if (((uintptr_t)x | (uintptr_t)gy) & 15) return fail("conv3d wgrad: buffers must be 16-byte aligned");
    const long long npos = (long long)B * D * H * W;
    const long long chunks = (npos + lfts::unet::WG_CHUNK - 1) / lfts::unet::WG_CHUNK;
    if (chunks > 0x7fffffffLL) return fail("conv3d wgrad: too many positions");
    const int ntap = taps == 27 ? 3 : 1;
    uint32_t cols = 32;
    while ((int)cols < ntap * cin) cols <<= 1;
    const size_t st_units = (size_t)16 * lfts::unet::WG_K + (size_t)ntap * (cin / 8) * lfts::unet::WG_K;
    const size_t smem = 2 * 16 * st_units + 2 * sizeof(uint64_t) + 16;
    if (smem > 200 * 1024) return fail("conv3d wgrad: cin too large for the shared-memory stages");
    if (cout > 128) return fail("conv3d wgrad: cout (the accumulator rows) must be <= 128");
    {
        cudaError_t e = cudaFuncSetAttribute(lfts::unet::k_conv3d_wgrad_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return fail(std::string("conv3d wgrad: ") + cudaGetErrorString(e));
    }
    lfts::unet::k_conv3d_wgrad_umma<<<dim3((unsigned)chunks, taps == 27 ? 9 : 1), lfts::unet::CONV_M, smem,
                                      (cudaStream_t)stream>>>((const uint4 *)x, (const uint4 *)gy, dw, B, D, H, W, cin, cout,
                                                              taps, cols);
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) return fail(std::string("conv3d wgrad launch: ") + cudaGetErrorString(e));
    return 0;
}

extern "C" int lfts_conv3d_bf16(void *stream, const void *in, const void *wpk, const float *bias, void *out, int B, int D,
                                int H, int W, int cin, int cout, int taps, int relu) {
    if (!in || !wpk || !bias || !out) return fail("null argument");
    if (B < 1 || D < 1 || H < 1 || W < 1) return fail("conv3d: extents must be positive");
    if (cin < 16 || cin % 16 || cin > LFTS_CONV_MAX_CIN)
        return fail("conv3d: cin must be a multiple of 16 up to " + std::to_string(LFTS_CONV_MAX_CIN));
    if (cout < 16 || cout % 16 || cout > LFTS_CONV_MAX_COUT)
        return fail("conv3d: cout must be a multiple of 16 up to " + std::to_string(LFTS_CONV_MAX_COUT));
    if (taps != 1 && taps != 27) return fail("conv3d: taps must be 1 (1x1x1) or 27 (3x3x3)");
    if (((uintptr_t)in | (uintptr_t)wpk | (uintptr_t)out) & 15) return fail("conv3d: buffers must be 16-byte aligned");
    const long long npos = (long long)B * D * H * W;
    const long long blocks = (npos + lfts::unet::CONV_M - 1) / lfts::unet::CONV_M;
    if (blocks > 0x7fffffffLL) return fail("conv3d: too many positions");
    uint32_t cols = 32;
    while ((int)cols < cout) cols <<= 1;
    {
        // halo-staged kernel: 3x3x3, H % 16 == 0, W % 8 == 0, halo + weight stages within 200 KB
        using namespace lfts::unet;
        // weight stages: as many (2..4) as fit beside the halo in 200 KB
        auto hs = [&](int ns) {
            return (size_t)16 * ((size_t)(cin / 8) * HPLANE + (size_t)ns * (cin / 8) * cout) + (2 * (size_t)ns + 1) * sizeof(uint64_t) + 16;
        };
        int NS = 4;
        while (NS > 2 && hs(NS) > 200 * 1024) NS--;
        const size_t hsmem = hs(NS);
        if (taps == 27 && H % HT_Y == 0 && W % HT_X == 0 && hsmem <= 200 * 1024 && (long long)B * D <= 65535) {
            // per device (the attribute belongs to the current device), so set on every call
            cudaError_t e = cudaFuncSetAttribute(k_conv3d_halo_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            if (e != cudaSuccess) return fail(std::string("conv3d: ") + cudaGetErrorString(e));
            k_conv3d_halo_umma<<<dim3((unsigned)(W / HT_X), (unsigned)(H / HT_Y), (unsigned)(B * D)), CONV_M, hsmem,
                                 (cudaStream_t)stream>>>((const uint4 *)in, (const uint4 *)wpk, bias, (uint16_t *)out, B, D, H,
                                                         W, cin, cout, relu, cols, NS);
            e = cudaPeekAtLastError();
            if (e != cudaSuccess) return fail(std::string("conv3d launch: ") + cudaGetErrorString(e));
            return 0;
        }
    }
    const size_t smem = (size_t)2 * 16 * ((size_t)(cin / 8) * (lfts::unet::CONV_M + cout)) + 2 * sizeof(uint64_t) + 16;
    if (smem > 200 * 1024) return fail("conv3d: cin x (128 + cout) too large for the shared-memory stages");
    {
        cudaError_t e = cudaFuncSetAttribute(lfts::unet::k_conv3d_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return fail(std::string("conv3d: ") + cudaGetErrorString(e));
    }
    lfts::unet::k_conv3d_umma<<<(unsigned)blocks, lfts::unet::CONV_M, smem, (cudaStream_t)stream>>>(
        (const uint4 *)in, (const uint4 *)wpk, bias, (uint16_t *)out, B, D, H, W, cin, cout, taps, relu, cols);
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) return fail(std::string("conv3d launch: ") + cudaGetErrorString(e));
    return 0;
}

// ---------------------------------------------------------------- AdamW (training of the U-Net)
// Decoupled weight decay, then the Adam moments and the bias-corrected step,
// in the order torch.optim.AdamW applies them:
//   p *= 1 - lr wd;  m += (1 - b1)(g - m);  v = b2 v + (1 - b2) g^2;
//   p -= (lr / (1 - b1^t)) m / (sqrt(v) / sqrt(1 - b2^t) + eps).
__global__ void k_adamw_f32(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                            long long n, float decay, float b1, float b2, float eps, float step_size, float bc2_sqrt) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        float mi = m[i];
        mi = mi + (1.0f - b1) * (gi - mi);
        const float vi = v[i] * b2 + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] * decay;
        p[i] = pi - step_size * (mi / (sqrtf(vi) / bc2_sqrt + eps));
    }
}

extern "C" int lfts_adamw_f32(void *stream, float *p, const float *g, float *m, float *v, long long n, double lr, double b1,
                              double b2, double eps, double weight_decay, int step) {
    if (!p || !g || !m || !v) return fail("adamw: null argument");
    if (n < 0 || step < 1) return fail("adamw: n must be >= 0 and step >= 1");
    if (n == 0) return 0;
    const double bc1 = 1.0 - std::pow(b1, step), bc2 = 1.0 - std::pow(b2, step);
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_adamw_f32<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(p, g, m, v, n, (float)(1.0 - lr * weight_decay), (float)b1,
                                                                   (float)b2, (float)eps, (float)(lr / bc1),
                                                                   (float)std::sqrt(bc2));
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) return fail(std::string("adamw launch: ") + cudaGetErrorString(e));
    return 0;
}
