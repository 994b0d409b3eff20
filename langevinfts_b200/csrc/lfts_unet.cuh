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
#include <cstdlib>
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
// 3x3x3 convolution with the input of a tile staged once: the tile is TZ x 16
// x 8 output positions (z, y, x; TZ = 1 or 2) and its halo (TZ + 2) x 18 x 10
// positions sits in shared memory as planes [kc][zh][yh][xh] of 16-byte
// units (a chunk's plane padded to an odd length).  For tap (dz, dy, dx) and
// output plane j the A operand of the MMA is read in place: the 8 output
// positions of a y row map to 8 consecutive halo rows (one core matrix), the
// 16 y rows are HX units apart (SBO), the channel chunks a plane apart (LBO).  Each staged tap of weights feeds TZ MMAs (one
// per output plane, TZ accumulators of COUT columns in tensor memory).  Needs
// H % 16 == 0, W % 8 == 0 and D % TZ == 0.
constexpr int HT_Y = 16, HT_X = 8, HY = HT_Y + 2, HX = HT_X + 2, HROW = HY * HX;  // halo positions per z plane

// Thread 32 streams the tap weights with one bulk copy per tap into a ring of
// NS stages (full[st]: transaction bytes), starting before the halo is staged;
// lane 0 of warp 0 issues each tap's MMAs once its stage is full and commits
// them to empty[st], which lets the next bulk copy into the stage; a last
// commit to done releases the epilogue.
template <int TZ>
__global__ void __launch_bounds__(CONV_M) k_conv3d_halo_umma(const uint4 *__restrict__ in, const uint4 *__restrict__ wpk,
                                                             const float *__restrict__ bias, uint16_t *__restrict__ out,
                                                             int B, int D, int H, int W, int cin, int cout, int relu,
                                                             uint32_t tmem_cols, int NS) {
    // halo units per channel chunk, odd so that the chunks of one position fall in different banks
    constexpr int HPL = (TZ + 2) * HROW + 1;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int kc_n = cin / 8, b_units = kc_n * cout;
    const uint32_t b_bytes = (uint32_t)b_units * 16;
    uint4 *halo = (uint4 *)smem_raw;                 // kc_n * HPL units
    uint4 *wst = halo + kc_n * HPL;                  // NS weight stages
    uint64_t *full = (uint64_t *)(wst + (size_t)NS * b_units), *empty = full + NS, *done = empty + NS;
    uint32_t *tmem_slot = (uint32_t *)(done + 1);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int ztiles = D / TZ;
    const int x0 = blockIdx.x * HT_X, y0 = blockIdx.y * HT_Y, z0 = (blockIdx.z % ztiles) * TZ, n = blockIdx.z / ztiles;
    int issued = 0;  // taps whose bulk copy thread 32 started
    if (tid == 32) {
        for (int i = 0; i < NS; i++) {
            mbar_init(full + i, 1);
            mbar_init(empty + i, 1);
        }
        mbar_init(done, 1);
        // the first NS taps stream in while the halo is staged
        for (; issued < NS && issued < 27; issued++) {
            mbar_arrive_expect_tx(full + issued, b_bytes);
            bulk_load(wst + (size_t)issued * b_units, wpk + (long long)issued * b_units, b_bytes, full + issued);
        }
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // the halo, periodic: halo row r = zh * HY + yh holds HX positions x kc_n
    // chunks, contiguous in global memory apart from the wrapped ends; thread
    // items run chunk-fastest along a row so that a warp's copies are coalesced
    {
        const int rowu = HX * kc_n, nrows = (TZ + 2) * HY;
        const int dr = CONV_M / rowu, df = CONV_M - dr * rowu;
        const float rk = 1.0f / (float)kc_n;
        int r = tid / rowu, f = tid - r * rowu;
        while (r < nrows) {
            const int xh = (int)(((float)f + 0.5f) * rk), kc = f - xh * kc_n;
            const int zh = r / HY, yh = r - zh * HY;
            int xx = x0 + xh - 1, yy = y0 + yh - 1, zz = z0 + zh - 1;
            xx += xx < 0 ? W : 0;
            xx -= xx >= W ? W : 0;
            yy += yy < 0 ? H : 0;
            yy -= yy >= H ? H : 0;
            zz += zz < 0 ? D : 0;
            zz -= zz >= D ? D : 0;
            cp_async16(halo + kc * HPL + r * HX + xh, in + ((((long long)n * D + zz) * H + yy) * W + xx) * kc_n + kc);
            f += df;
            r += dr;
            if (f >= rowu) {
                f -= rowu;
                r++;
            }
        }
    }
    cp_async_wait_all();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    bool ok = true;
    if (tid == 32) {
        // producer: tap t into stage t % NS once the MMAs of tap t - NS freed it
        for (; issued < 27; issued++) {
            const int st = issued % NS, u = issued / NS;
            if (!mbar_wait(empty + st, (u - 1) & 1)) {
                ok = false;
                break;
            }
            mbar_arrive_expect_tx(full + st, b_bytes);
            bulk_load(wst + (size_t)st * b_units, wpk + (long long)issued * b_units, b_bytes, full + st);
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
            const uint32_t b0 = smem_addr(wst + (size_t)st * b_units);
#pragma unroll
            for (int j = 0; j < TZ; j++) {
                const uint32_t a_tap = halo0 + (uint32_t)((((j + dz) * HY + dy) * HX + dx) * 16);
                for (int s = 0; s < kc_n / 2; s++) {
                    const uint64_t da = umma_desc(a_tap + (uint32_t)(2 * s * HPL * 16), HPL * 16, HX * 16);
                    const uint64_t db = umma_desc(b0 + (uint32_t)(2 * s * cout * 16), (uint32_t)cout * 16, 128);
                    umma_bf16(tmem + (uint32_t)(j * cout), da, db, idesc, (t > 0 || s > 0) ? 1u : 0u);
                }
            }
            umma_commit(empty + st);
        }
        if (ok) umma_commit(done);
    }
    {
        // every thread: the accumulators are complete (or some wait gave up)
        const bool fin = __syncthreads_and(ok) ? mbar_wait(done, 0) : false;
        ok = __syncthreads_and(fin);
    }
    if (!ok) {
        // a second bounded wait for MMAs still in flight, and for the weight
        // copies that no MMA consumed
        mbar_wait(done, 0);
        if (tid == 32)
            for (int t = issued > NS ? issued - NS : 0; t < issued; t++) mbar_wait(full + t % NS, (t / NS) & 1);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int m = tid;  // accumulator row = 8 j + l: position (y0 + j, x0 + l)
#pragma unroll
        for (int j = 0; j < TZ; j++) {
            const long long p = (((long long)n * D + z0 + j) * H + (y0 + m / 8)) * W + (x0 + m % 8);
            for (int c0 = 0; c0 < cout; c0 += 16) {
                uint32_t v[16];
                tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(j * cout + c0), v);
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
// Weight gradient of the periodic convolution:
//   dw[tap][co][ci] += sum_p gy[p][co] x[p + tap][ci]
// per tap a GEMM with M = co (padded to 128 rows), N = cin, K = positions.
// Both operands are MN-major in channels-last memory (16 bytes = 8 channels of
// one position), so they are staged without transposition: 8 consecutive
// positions of one channel chunk form a core matrix (16-byte rows), channel
// chunks are a fixed stride apart (SBO).  gy (A): chunk c of position k at
// (c * WG_K + k) * 16 bytes.  A CTA takes one (kz, ky) row of taps (kx = 0..2;
// the single tap of a 1x1x1 kernel) over nst stages of WG_K positions, keeps one
// accumulator per tap in tensor memory, and adds them to dw (FP32, zeroed by
// the caller) with atomics.
//
// x (B), ROWS form (W % 8 == 0): the WG_K positions of a stage are R = WG_K /
// SEG segments of SEG consecutive x positions of one row (SEG = 64, 32, 16 or
// 8, dividing W), each staged once with a one-position periodic halo on both
// sides, shifted by (dz, dy): chunk c of halo position h of segment r at
// (c * XS + r * (SEG + 2) + h) * 16 bytes, XS = R * (SEG + 2).  The three kx
// taps read the same staged rows, offset by kx units; the two core matrices
// of a K-step are 128 bytes apart inside a segment (SEG >= 16) or one segment
// apart (SEG = 8).  Gather form (other W): per tap, the shifted row of each
// position, chunk c of position k at (c * WG_K + k) * 16 bytes.
//
// The stages go through a ring of WS slots.  Warps 0-3 load: every thread
// copies its share of stage v with cp.async (one commit group per stage; items
// run chunk-fastest so a warp's copies are coalesced), and at stage u waits
// only for its own group of stage u (WS - 2 newer groups may still be in
// flight), fences and arrives on full[u % WS].  Lane 0 of warp 4 does nothing
// else than issue: it waits for full[u % WS] (all 128 arrivals), issues the
// stage's MMAs and commits them to empty[u % WS], which each loading thread
// waits for before it refills the slot.  Warps 0-3 then read the accumulators
// (tensor-memory lanes 32 w .. 32 w + 31).
constexpr int WG_K = 64;        // positions per stage (4 MMA K-steps)

template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// The MMA reads A as 128 rows (16 chunks of WG_K positions from the slot's
// start): rows at and above cout read whatever follows (the slot's B, the next
// slot), and their accumulator rows are never stored.  The ring is padded so
// that the last slot's 16 chunks stay inside it.
__host__ __device__ constexpr int wgrad_ring_units(int ws, int st_units) {
    return (ws - 1) * st_units + (st_units > 16 * WG_K ? st_units : 16 * WG_K);
}
// 16-byte units of one slot: gy, then x (ROWS form: seg > 0)
__host__ __device__ constexpr int wgrad_slot_units(int cin, int cout, int ntap, int seg) {
    return (cout / 8) * WG_K + (seg > 0 ? (cin / 8) * (WG_K / seg) * (seg + 2) : ntap * (cin / 8) * WG_K);
}

constexpr int WG_THREADS = CONV_M + 32;  // 4 loading warps and the MMA warp

template <int WS, bool ROWS>
__global__ void __launch_bounds__(WG_THREADS) k_conv3d_wgrad_umma(const uint4 *__restrict__ x, const uint4 *__restrict__ gy,
                                                              float *__restrict__ dw, int B, int D, int H, int W, int cin,
                                                              int cout, int taps, uint32_t tmem_cols, int seg, int nst) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int ntap = taps == 27 ? 3 : 1;
    const int xc = cin / 8, gc = cout / 8;             // 16-byte chunks per position
    const int R = ROWS ? WG_K / seg : 0, SW = seg + 2, XS = R * SW;
    const int a_units = gc * WG_K, b_units = xc * WG_K; // A: the cout rows; B per tap (gather form)
    const int st_units = wgrad_slot_units(cin, cout, ntap, ROWS ? seg : 0);
    uint4 *stage0 = (uint4 *)smem_raw;
    uint64_t *full = (uint64_t *)(stage0 + wgrad_ring_units(WS, st_units)), *empty = full + WS;
    uint32_t *tmem_slot = (uint32_t *)(empty + WS);
    long long *seg_row = (long long *)(empty + WS + 1);  // ROWS: per (stage, segment) shifted row start, -1 past the end
    int *seg_x0 = (int *)(seg_row + nst * R);             // ROWS: x of the segment's first position
    const int tid = threadIdx.x, warp = tid >> 5;
    const long long npos = (long long)B * D * H * W;
    // the tap rows of a chunk are neighbours in the grid, so its x and gy come from DRAM once
    const long long p0 = (long long)blockIdx.y * nst * WG_K;
    const int g = blockIdx.x;  // tap row: kz = g / 3, ky = g % 3
    const int dz = taps == 27 ? g / 3 - 1 : 0, dy = taps == 27 ? g % 3 - 1 : 0;
    if (tid == 0) {
        for (int s = 0; s < WS; s++) {
            mbar_init(full + s, CONV_M);
            mbar_init(empty + s, 1);
        }
    }
    if (ROWS) {
        for (int e = tid; e < nst * R; e += WG_THREADS) {
            const long long ps = p0 + (long long)e * seg;  // stage e / R, segment e % R
            long long base = -1;
            int x0 = 0;
            if (ps < npos) {
                long long q = ps / W;
                x0 = (int)(ps - q * W);
                int y = (int)(q % H) + dy;
                q /= H;
                int z = (int)(q % D) + dz;
                const long long n = q / D;
                y += y < 0 ? H : 0;
                y -= y >= H ? H : 0;
                z += z < 0 ? D : 0;
                z -= z >= D ? D : 0;
                base = ((n * D + z) * H + y) * W;
            }
            seg_row[e] = base;
            seg_x0[e] = x0;
        }
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
    // gather form with ntap cin <= 256: all taps in one MMA (N = ntap cin, accumulator j at columns j cin as before)
    const bool stack = !ROWS && ntap * cin <= 256;
    const uint32_t idesc_stack = (idesc & ~(0x3Fu << 17)) | ((uint32_t)((ntap * cin) >> 3) << 17);
    const float rgc = 1.0f / (float)gc, rxc = 1.0f / (float)xc, rsw = 1.0f / (float)SW;
    // this thread's copies of stage v into its slot (zeros beyond the last position)
    auto load = [&](int v) {
        uint4 *sa = stage0 + (v % WS) * st_units, *sb = sa + a_units;
        const long long pv = p0 + (long long)v * WG_K;
        // gy: WG_K positions x gc chunks, contiguous in global memory
        for (int i = tid; i < WG_K * gc; i += CONV_M) {
            const int k = (int)(((float)i + 0.5f) * rgc), c = i - k * gc;
            if (pv + k < npos) cp_async16(sa + c * WG_K + k, gy + pv * gc + i);
            else sa[c * WG_K + k] = make_uint4(0, 0, 0, 0);
        }
        if (ROWS) {
            // x: R segments x (SEG + 2) halo positions x xc chunks
            for (int i = tid; i < XS * xc; i += CONV_M) {
                const int q = (int)(((float)i + 0.5f) * rxc), c = i - q * xc;
                const int r = (int)(((float)q + 0.5f) * rsw), h = q - r * SW;
                const int e = v * R + r;
                const long long base = seg_row[e];
                uint4 *dst = sb + c * XS + r * SW + h;
                if (base >= 0) {
                    int xw = seg_x0[e] + h - 1;
                    xw += xw < 0 ? W : 0;
                    xw -= xw >= W ? W : 0;
                    cp_async16(dst, x + (base + xw) * xc + c);
                } else {
                    *dst = make_uint4(0, 0, 0, 0);
                }
            }
        } else {
            // x: per tap the shifted row of each position
            for (int i = tid; i < ntap * WG_K * xc; i += CONV_M) {
                const int q = (int)(((float)i + 0.5f) * rxc), c = i - q * xc;
                const int j = q / WG_K, k = q - j * WG_K;
                uint4 *dst = sb + j * b_units + c * WG_K + k;
                const long long p = pv + k;
                if (p < npos) {
                    long long t = p / W;
                    int xx = (int)(p - t * W) + (taps == 27 ? j - 1 : 0);
                    int y = (int)(t % H) + dy;
                    t /= H;
                    int z = (int)(t % D) + dz;
                    const long long n = t / D;
                    xx += xx < 0 ? W : 0;
                    xx -= xx >= W ? W : 0;
                    y += y < 0 ? H : 0;
                    y -= y >= H ? H : 0;
                    z += z < 0 ? D : 0;
                    z -= z >= D ? D : 0;
                    cp_async16(dst, x + (((n * D + z) * H + y) * W + xx) * xc + c);
                } else {
                    *dst = make_uint4(0, 0, 0, 0);
                }
            }
        }
    };
    bool ok = true;
    int u = 0;  // the MMA thread: stages issued
    if (warp < 4) {
        // one commit group per stage (empty past the last), so group u holds stage u
        for (int v = 0; v < WS - 1; v++) {
            if (v < nst) load(v);
            cp_async_commit();
        }
        for (int w = 0; w < nst; w++) {
            cp_async_wait_group<WS - 2>();  // this thread's stage w has landed (WS - 2 newer groups may not)
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(full + w % WS);
            // refill the slot of stage w - 1 with stage w + WS - 1 once its MMAs are done
            const int v = w + WS - 1;
            if (v < nst) {
                if (v >= WS && !mbar_wait(empty + v % WS, (v / WS - 1) & 1)) {
                    ok = false;
                    break;
                }
                load(v);
            }
            cp_async_commit();
        }
        cp_async_wait_all();
    } else if (tid == CONV_M) {
        for (; u < nst; u++) {
            const int st = u % WS;
            if (!mbar_wait(full + st, (u / WS) & 1)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_addr(stage0 + st * st_units), b0 = a0 + (uint32_t)a_units * 16;
            if (!ROWS && stack) {
                // gather form: the taps' copies are chunks j * xc + c at one stride, so one MMA of N = ntap cin
                for (int s = 0; s < WG_K / 16; s++)
                    umma_bf16(tmem, umma_desc(a0 + (uint32_t)(16 * s * 16), 128, WG_K * 16),
                              umma_desc(b0 + (uint32_t)(16 * s * 16), 128, WG_K * 16), idesc_stack, (u > 0 || s > 0) ? 1u : 0u);
                umma_commit(empty + st);
                continue;
            }
            for (int s = 0; s < WG_K / 16; s++) {
                const uint64_t da = umma_desc(a0 + (uint32_t)(16 * s * 16), 128, WG_K * 16);
                for (int j = 0; j < ntap; j++) {
                    uint64_t db;
                    if (ROWS) {
                        const int k0 = 16 * s, r = k0 / seg;
                        const int unit = r * SW + (k0 - r * seg) + (taps == 27 ? j : 1);
                        db = umma_desc(b0 + (uint32_t)unit * 16, seg >= 16 ? 128u : (uint32_t)SW * 16, (uint32_t)XS * 16);
                    } else {
                        db = umma_desc(b0 + (uint32_t)((j * b_units + 16 * s) * 16), 128, WG_K * 16);
                    }
                    umma_bf16(tmem + (uint32_t)(j * cin), da, db, idesc, (u > 0 || s > 0) ? 1u : 0u);
                }
            }
            umma_commit(empty + st);
        }
    }
    {
        // the last stage's MMAs are the last to complete (one thread issues them in order)
        const bool fin = __syncthreads_and(ok) ? mbar_wait(empty + (nst - 1) % WS, ((nst - 1) / WS) & 1) : false;
        ok = __syncthreads_and(fin);
    }
    if (!ok) {
        // a second bounded wait for MMAs still in flight: the last stage the MMA thread committed
        if (tid == CONV_M && u > 0) mbar_wait(empty + (u - 1) % WS, ((u - 1) / WS) & 1);
    } else if (warp < 4) {
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
// ------------------------------------------------------------------------
// 3x3x3 convolution by slices of 16 input channels: for the tile of TZ x 16 x 8
// output positions (TZ = 1, 2 or 4 planes, one accumulator of COUT columns per
// plane) each stage of a ring of NS slots holds one slice: the halo of its two
// 16-byte channel chunks, (TZ + 2) x 18 x 10 positions as two planes of odd
// length HPLP (the layout of k_conv3d_halo_umma restricted to two chunks), and
// the 27 taps' weights of those channels, tap t at t * 2 * COUT units (two
// chunks of COUT rows).  A slice feeds 27 x TZ MMAs of K = 16.  Warps 0-3 load
// (the halo with cp.async, chunk-fastest; thread 0 also issues one bulk copy
// per tap for the weights, counted in transaction bytes on the slot's full
// barrier), wait for their own copies with a lag of NS - 2 groups, fence and
// arrive; lane 0 of warp 4 issues the MMAs of a full slot and commits them to
// its empty barrier; warps 0-3 then read the accumulators.  Against the halo
// kernel the loads overlap the MMAs inside a CTA and each weight byte staged
// serves TZ x 128 positions.  Needs H % 16 == 0, W % 8 == 0, D % TZ == 0.
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

constexpr int KS_THREADS = CONV_M + 32;  // 4 loading warps and the MMA warp

template <int TZ> __host__ __device__ constexpr int kslice_hplp() { return (TZ + 2) * HROW + 1; }
__host__ __device__ constexpr int kslice_slot_units(int hplp, int cout) { return 2 * hplp + 27 * 2 * cout; }

template <int TZ, int NS>
__global__ void __launch_bounds__(KS_THREADS) k_conv3d_kslice_umma(const uint4 *__restrict__ in, const uint4 *__restrict__ wpk,
                                                                 const float *__restrict__ bias, uint16_t *__restrict__ out,
                                                                 int B, int D, int H, int W, int cin, int cout, int relu,
                                                                 uint32_t tmem_cols) {
    constexpr int HPLP = kslice_hplp<TZ>();
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int kc_n = cin / 8, nsl = kc_n / 2, b_units = kc_n * cout;
    const int slot_units = kslice_slot_units(HPLP, cout);
    const uint32_t w_bytes = 27u * 2u * (uint32_t)cout * 16u;
    uint4 *ring = (uint4 *)smem_raw;
    uint64_t *full = (uint64_t *)(ring + (size_t)NS * slot_units), *empty = full + NS, *done = empty + NS;
    uint32_t *tmem_slot = (uint32_t *)(done + 1);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int ztiles = D / TZ;
    const int x0 = blockIdx.x * HT_X, y0 = blockIdx.y * HT_Y, z0 = (blockIdx.z % ztiles) * TZ, n = blockIdx.z / ztiles;
    if (tid == 0) {
        for (int i = 0; i < NS; i++) {
            mbar_init(full + i, CONV_M);
            mbar_init(empty + i, 1);
        }
        mbar_init(done, 1);
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
    // loading thread's copies of slice v into its slot
    auto load = [&](int v) {
        uint4 *slot = ring + (size_t)(v % NS) * slot_units;
        if (tid == 0) {
            mbar_expect_tx(full + v % NS, w_bytes);
            uint4 *wd = slot + 2 * HPLP;
            for (int t = 0; t < 27; t++)
                bulk_load(wd + t * 2 * cout, wpk + (long long)t * b_units + 2 * v * cout, 2u * (uint32_t)cout * 16u,
                          full + v % NS);
        }
        // halo items (position, chunk), chunk fastest: two consecutive threads read a position's 32 bytes
        for (int i = tid; i < 2 * (TZ + 2) * HROW; i += CONV_M) {
            const int r = i >> 1, c = i & 1;
            const int zh = r / HROW, rem = r - zh * HROW, yh = rem / HX, xh = rem - yh * HX;
            int xx = x0 + xh - 1, yy = y0 + yh - 1, zz = z0 + zh - 1;
            xx += xx < 0 ? W : 0;
            xx -= xx >= W ? W : 0;
            yy += yy < 0 ? H : 0;
            yy -= yy >= H ? H : 0;
            zz += zz < 0 ? D : 0;
            zz -= zz >= D ? D : 0;
            cp_async16(slot + c * HPLP + r, in + ((((long long)n * D + zz) * H + yy) * W + xx) * kc_n + 2 * v + c);
        }
    };
    bool ok = true;
    int u = 0;  // the MMA thread: slices issued
    if (warp < 4) {
        for (int v = 0; v < NS - 1; v++) {
            if (v < nsl) load(v);
            cp_async_commit();
        }
        for (int w = 0; w < nsl; w++) {
            cp_async_wait_group<NS - 2>();  // this thread's halo copies of slice w have landed
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(full + w % NS);
            const int v = w + NS - 1;
            if (v < nsl) {
                if (v >= NS && !mbar_wait(empty + v % NS, (v / NS - 1) & 1)) {
                    ok = false;
                    break;
                }
                load(v);
            }
            cp_async_commit();
        }
        cp_async_wait_all();
    } else if (tid == CONV_M) {
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(cout >> 3) << 17) | ((uint32_t)(CONV_M >> 4) << 24);
        for (; u < nsl; u++) {
            const int st = u % NS;
            if (!mbar_wait(full + st, (u / NS) & 1)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t h0 = smem_addr(ring + (size_t)st * slot_units), w0 = h0 + (uint32_t)(2 * HPLP) * 16u;
            for (int t = 0; t < 27; t++) {
                const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
                const uint64_t db = umma_desc(w0 + (uint32_t)(t * 2 * cout) * 16u, (uint32_t)cout * 16, 128);
#pragma unroll
                for (int j = 0; j < TZ; j++) {
                    const uint32_t a = h0 + (uint32_t)((((j + dz) * HY + dy) * HX + dx) * 16);
                    umma_bf16(tmem + (uint32_t)(j * cout), umma_desc(a, HPLP * 16, HX * 16), db, idesc,
                              (u > 0 || t > 0) ? 1u : 0u);
                }
            }
            umma_commit(empty + st);
        }
        if (ok) umma_commit(done);
    }
    {
        const bool fin = __syncthreads_and(ok) ? mbar_wait(done, 0) : false;
        ok = __syncthreads_and(fin);
    }
    if (!ok) {
        // a wait gave up after its bound (the weight copies issued have long landed by
        // then): a second bounded wait for the MMAs the MMA thread committed
        if (tid == CONV_M && u > 0) mbar_wait(empty + (u - 1) % NS, ((u - 1) / NS) & 1);
    } else if (warp < 4) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int m = tid;  // accumulator row = 8 j + l: position (y0 + j, x0 + l)
#pragma unroll
        for (int j = 0; j < TZ; j++) {
            const long long p = (((long long)n * D + z0 + j) * H + (y0 + m / 8)) * W + (x0 + m % 8);
            for (int c0 = 0; c0 < cout; c0 += 16) {
                uint32_t v[16];
                tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(j * cout + c0), v);
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
    const int ntap = taps == 27 ? 3 : 1;
    const long long rows = taps == 27 ? 9 : 1;
    uint32_t cols = 32;
    while ((int)cols < ntap * cin) cols <<= 1;
    if (cout > 128) return fail("conv3d wgrad: cout (the accumulator rows) must be <= 128");
    using namespace lfts::unet;
    // x staged as row segments with a halo when W % 8 == 0 (segment: the longest of 64, 32, 16, 8 dividing W)
    int seg = W % 64 == 0 ? 64 : W % 32 == 0 ? 32 : W % 16 == 0 ? 16 : W % 8 == 0 ? 8 : 0;
    if (const char *env = std::getenv("LFTS_CONV_WGRAD_GATHER"))  // 1: per-tap gathers at every W
        if (env[0] == '1') seg = 0;
    const int st_units = wgrad_slot_units(cin, cout, ntap, seg);
    auto smem_of = [&](int ws, int nst) {
        const size_t table = seg ? (size_t)nst * (WG_K / seg) * (sizeof(long long) + sizeof(int)) : 0;
        return (size_t)16 * wgrad_ring_units(ws, st_units) + (2 * (size_t)ws + 1) * sizeof(uint64_t) + table + 16;
    };
    // resident CTAs per SM: shared memory (228 KB per SM, 1 KB reserved per CTA) and tensor-memory columns
    auto resident = [&](size_t smem) {
        int c = (int)((228 * 1024) / (smem + 1024));
        return c < (int)(512 / cols) ? c : (int)(512 / cols);
    };
    // ring depth: the most stages in flight per SM (resident CTAs times WS - 1); ties go to the deeper ring
    int WS = 0, best = 0;
    for (int ws = 2; ws <= 4; ws++) {
        if (smem_of(ws, 64) > 200 * 1024) continue;
        const int c = resident(smem_of(ws, 64));
        if (c * (ws - 1) >= best) {
            best = c * (ws - 1);
            WS = ws;
        }
    }
    if (const char *env = std::getenv("LFTS_CONV_WGRAD_RING")) {  // 2, 3 or 4 overrides the choice
        const int ws = env[0] - '0';
        if (ws >= 2 && ws <= 4 && smem_of(ws, 64) <= 200 * 1024) WS = ws;
    }
    if (WS == 0) return fail("conv3d wgrad: cin too large for the shared-memory stages");
    // stages of WG_K positions per CTA (each CTA adds its partial sums to dw with
    // atomics): 64 while that gives at least four waves of resident CTAs, else the
    // most (32 .. 256) that still fill one wave
    auto ctas = [&](int nst) { return (npos + (long long)nst * WG_K - 1) / ((long long)nst * WG_K) * rows; };
    const long long wave = 148LL * resident(smem_of(WS, 64));
    int nst = 64;
    if (ctas(64) < 4 * wave) {
        nst = 32;
        while (nst < 256 && ctas(2 * nst) >= wave - wave / 16) nst *= 2;
    }
    if (const char *env = std::getenv("LFTS_CONV_WGRAD_STAGES")) {  // override: 32 .. 1024
        const int v = std::atoi(env);
        if (v >= 32 && v <= 1024) nst = v;
    }
    const long long chunks = (npos + (long long)nst * WG_K - 1) / ((long long)nst * WG_K);
    if (chunks > 65535) return fail("conv3d wgrad: too many positions (more than 65535 chunks of nst x 64)");
    if (smem_of(WS, nst) > 200 * 1024) return fail("conv3d wgrad: shared memory of the stages and the segment table");
    using Kern = void (*)(const uint4 *, const uint4 *, float *, int, int, int, int, int, int, int, uint32_t, int, int);
    Kern kern = seg ? (WS == 2 ? k_conv3d_wgrad_umma<2, true> : WS == 3 ? k_conv3d_wgrad_umma<3, true> : k_conv3d_wgrad_umma<4, true>)
                    : (WS == 2 ? k_conv3d_wgrad_umma<2, false> : WS == 3 ? k_conv3d_wgrad_umma<3, false> : k_conv3d_wgrad_umma<4, false>);
    cudaError_t e = cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return fail(std::string("conv3d wgrad: ") + cudaGetErrorString(e));
    kern<<<dim3(taps == 27 ? 9 : 1, (unsigned)chunks), WG_THREADS, smem_of(WS, nst), (cudaStream_t)stream>>>(
        (const uint4 *)x, (const uint4 *)gy, dw, B, D, H, W, cin, cout, taps, cols, seg, nst);
    e = cudaPeekAtLastError();
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
    if (taps == 27 && H % lfts::unet::HT_Y == 0 && W % lfts::unet::HT_X == 0 && cin >= 32) {
        // slices of 16 input channels, by default from three slices on (at two the
        // halo kernel is faster: 323 against 498 us for 32 -> 32 channels at 64^3 x 8).
        // Of the (output planes 4, 2, 1; ring of 3 or 2 slots) within 200 KB, the one
        // with the most resident CTAs per SM, then the most planes, then slots
        // (d1a 80 -> 32: 2 planes, 2 slots, two CTAs per SM 625 us against 859-891 us
        // for 4 planes at one CTA per SM and 1161 us for the halo kernel; d2a 144 -> 48:
        // 4 planes, 2 slots 210 against 378 us).  LFTS_CONV_KSLICE=0|1 (1: from two
        // slices on), LFTS_CONV_KSLICE_TZ=1|2|4 and LFTS_CONV_KSLICE_NS=2|3 override
        using namespace lfts::unet;
        bool use = cin >= 48;
        int want_tz = 0;
        if (const char *env = std::getenv("LFTS_CONV_KSLICE")) use = env[0] != '0';
        int want_ns = 0;
        if (const char *env = std::getenv("LFTS_CONV_KSLICE_TZ")) want_tz = std::atoi(env);
        if (const char *env = std::getenv("LFTS_CONV_KSLICE_NS")) want_ns = std::atoi(env);
        auto smem_of = [&](int tz, int ns) {
            const int hplp = (tz + 2) * HROW + 1;
            return (size_t)16 * ns * kslice_slot_units(hplp, cout) + (2 * (size_t)ns + 1) * sizeof(uint64_t) + 16;
        };
        int tz = 0, ns = 0, best = 0;
        for (int t : {4, 2, 1}) {
            if ((want_tz && t != want_tz) || D % t || t * cout > 256) continue;
            for (int q : {3, 2}) {
                if ((want_ns && q != want_ns) || smem_of(t, q) > 200 * 1024) continue;
                int res = (int)((228 * 1024) / (smem_of(t, q) + 1024));  // resident CTAs: shared memory ...
                int cols = 32;
                while (cols < t * cout) cols <<= 1;
                if (res > 512 / cols) res = 512 / cols;                  // ... and tensor-memory columns
                const int score = res * 100 + t * 10 + q;
                if (score > best) {
                    best = score;
                    tz = t;
                    ns = q;
                }
            }
        }
        if (use && tz && (long long)B * D / tz <= 65535) {
            uint32_t kcols = 32;
            while ((int)kcols < tz * cout) kcols <<= 1;
            using Kern = void (*)(const uint4 *, const uint4 *, const float *, uint16_t *, int, int, int, int, int, int, int, uint32_t);
            Kern kern = tz == 4 ? (ns == 3 ? k_conv3d_kslice_umma<4, 3> : k_conv3d_kslice_umma<4, 2>)
                      : tz == 2 ? (ns == 3 ? k_conv3d_kslice_umma<2, 3> : k_conv3d_kslice_umma<2, 2>)
                                : (ns == 3 ? k_conv3d_kslice_umma<1, 3> : k_conv3d_kslice_umma<1, 2>);
            cudaError_t e = cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            if (e != cudaSuccess) return fail(std::string("conv3d: ") + cudaGetErrorString(e));
            kern<<<dim3((unsigned)(W / HT_X), (unsigned)(H / HT_Y), (unsigned)(B * D / tz)), KS_THREADS, smem_of(tz, ns),
                   (cudaStream_t)stream>>>((const uint4 *)in, (const uint4 *)wpk, bias, (uint16_t *)out, B, D, H, W, cin, cout,
                                           relu, kcols);
            e = cudaPeekAtLastError();
            if (e != cudaSuccess) return fail(std::string("conv3d launch: ") + cudaGetErrorString(e));
            return 0;
        }
    }
    if (taps == 27 && H % lfts::unet::HT_Y == 0 && W % lfts::unet::HT_X == 0) {
        // halo-staged kernel: TZ output planes per CTA, a ring of NS weight stages
        using namespace lfts::unet;
        auto hs = [&](int tz, int ns) {
            return (size_t)16 * ((size_t)(cin / 8) * ((tz + 2) * HROW + 1) + (size_t)ns * (cin / 8) * cout) +
                   (2 * (size_t)ns + 1) * sizeof(uint64_t) + 16;
        };
        // CTAs per SM that the shared memory allows (228 KB per SM, 1 KB reserved per CTA)
        auto fit = [](size_t smem) { return (int)((228 * 1024) / (smem + 1024)); };
        // the most weight stages (2..8) within 200 KB that keep the occupancy of two stages
        auto stages = [&](int tz) {
            int ns = 8;
            while (ns > 2 && (hs(tz, ns) > 200 * 1024 || fit(hs(tz, ns)) < fit(hs(tz, 2)))) ns--;
            return ns;
        };
        // two output planes per CTA when the halo of 4 planes keeps two CTAs per SM (LFTS_CONV_TZ=1|2 overrides)
        int tz = (D % 2 == 0 && 2 * cout <= 256 && hs(2, 2) <= 200 * 1024 && fit(hs(2, 2)) >= 2) ? 2 : 1;
        if (const char *env = std::getenv("LFTS_CONV_TZ")) {
            if (env[0] == '1') tz = 1;
            if (env[0] == '2' && D % 2 == 0 && 2 * cout <= 512 && hs(2, 2) <= 200 * 1024) tz = 2;
        }
        const int NS = stages(tz);
        const size_t hsmem = hs(tz, NS);
        uint32_t hcols = 32;
        while ((int)hcols < tz * cout) hcols <<= 1;
        if (hsmem <= 200 * 1024 && (long long)B * D / tz <= 65535) {
            // per device (the attribute belongs to the current device), so set on every call
            cudaError_t e = tz == 2 ? cudaFuncSetAttribute(k_conv3d_halo_umma<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)
                                    : cudaFuncSetAttribute(k_conv3d_halo_umma<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            if (e != cudaSuccess) return fail(std::string("conv3d: ") + cudaGetErrorString(e));
            const dim3 grid((unsigned)(W / HT_X), (unsigned)(H / HT_Y), (unsigned)(B * D / tz));
            if (tz == 2)
                k_conv3d_halo_umma<2><<<grid, CONV_M, hsmem, (cudaStream_t)stream>>>(
                    (const uint4 *)in, (const uint4 *)wpk, bias, (uint16_t *)out, B, D, H, W, cin, cout, relu, hcols, NS);
            else
                k_conv3d_halo_umma<1><<<grid, CONV_M, hsmem, (cudaStream_t)stream>>>(
                    (const uint4 *)in, (const uint4 *)wpk, bias, (uint16_t *)out, B, D, H, W, cin, cout, relu, hcols, NS);
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

namespace lfts {
namespace unet {

// ---------------------------------------------------------------- ReLU backward (training of the U-Net)
// g = gy where y > 0, else +0 (BF16, [npos][cpad]), and db[c] += sum_p g[p][c]
// for c < co (FP32).  Thread t of a block of cg * k threads (cg = cpad / 8
// chunks of 8 channels) keeps chunk t % cg for the whole grid-stride loop, so
// its 8 partial sums stay in registers; the block adds them up by chunk in
// shared memory and issues one atomic per channel.
__global__ void k_relu_grad_bf16(const uint4 *__restrict__ gy, const uint4 *__restrict__ y, uint4 *__restrict__ g,
                                 float *__restrict__ db, long long units, int cg, int co) {
    extern __shared__ float red[];  // [blockDim][8]
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < units; u += stride) {
        const uint4 a = gy[u], m = y[u];
        const uint32_t av[4] = {a.x, a.y, a.z, a.w}, mv[4] = {m.x, m.y, m.z, m.w};
        uint32_t ov[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            // BF16 y > 0: sign bit clear, not zero, not NaN (as torch's y > 0)
            const uint32_t lo = mv[i] & 0xFFFFu, hi = mv[i] >> 16;
            const bool plo = !(lo & 0x8000u) && (lo & 0x7FFFu) && (lo & 0x7FFFu) <= 0x7F80u;
            const bool phi = !(hi & 0x8000u) && (hi & 0x7FFFu) && (hi & 0x7FFFu) <= 0x7F80u;
            const uint32_t o = (plo ? (av[i] & 0xFFFFu) : 0u) | (phi ? (av[i] & 0xFFFF0000u) : 0u);
            ov[i] = o;
            acc[2 * i] += __uint_as_float(o << 16);
            acc[2 * i + 1] += __uint_as_float(o & 0xFFFF0000u);
        }
        g[u] = make_uint4(ov[0], ov[1], ov[2], ov[3]);
    }
#pragma unroll
    for (int i = 0; i < 8; i++) red[threadIdx.x * 8 + i] = acc[i];
    __syncthreads();
    // thread c8 < cg * 8 sums channel c8 over the block's threads of its chunk
    for (int c8 = threadIdx.x; c8 < cg * 8; c8 += blockDim.x) {
        const int chunk = c8 >> 3, i = c8 & 7;
        float s = 0.f;
        for (int t = chunk; t < (int)blockDim.x; t += cg) s += red[t * 8 + i];
        if (c8 < co) atomicAdd(db + c8, s);
    }
}
}  // namespace unet
}  // namespace lfts

extern "C" int lfts_relu_grad_bf16(void *stream, const void *gy, const void *y, void *g, float *db, long long npos, int cpad,
                                   int co) {
    if (!gy || !y || !g || !db) return fail("relu grad: null argument");
    if (npos < 0 || cpad < 8 || cpad % 8 || cpad > 256 || co < 0 || co > cpad)
        return fail("relu grad: cpad must be a multiple of 8 up to 256 and 0 <= co <= cpad");
    if (((uintptr_t)gy | (uintptr_t)y | (uintptr_t)g) & 15) return fail("relu grad: buffers must be 16-byte aligned");
    if (npos == 0) return 0;
    const int cg = cpad / 8, threads = cg * (256 / cg);
    const long long units = npos * cg;
    long long blocks = (units + threads - 1) / threads;
    if (blocks > 148 * 8) blocks = 148 * 8;
    lfts::unet::k_relu_grad_bf16<<<(unsigned)blocks, threads, (size_t)threads * 8 * sizeof(float), (cudaStream_t)stream>>>(
        (const uint4 *)gy, (const uint4 *)y, (uint4 *)g, db, units, cg, co);
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) return fail(std::string("relu grad launch: ") + cudaGetErrorString(e));
    return 0;
}
