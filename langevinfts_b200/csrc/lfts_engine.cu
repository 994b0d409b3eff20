// liblfts_b200: C-ABI implementation of the B200 chain-propagator engine.
// Declarations and the reference interfaces each entry replaces are in
// include/lfts_b200.h.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "lfts_step_fast.cuh"
#include "lfts_step_r8.cuh"
#include "lfts_step_r12.cuh"
#include "lfts_realspace.cuh"

using namespace lfts;

// ---------------------------------------------------------------- errors
static thread_local std::string g_err;

static int fail(const std::string &msg) {
    g_err = msg;
    return -1;
}
int lfts_internal_fail(const std::string &msg) { return fail(msg); }
void lfts_internal_count(lfts_ctx c, int n);
#define CK(call)                                                                                        \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return fail(std::string(#call) + ": " + cudaGetErrorString(e_) + " (" __FILE__ ":" +        \
                        std::to_string(__LINE__) + ")");                                                \
    } while (0)
#define CKLAUNCH(name) CK(cudaPeekAtLastError())

// ---------------------------------------------------------------- context
struct lfts_ctx_s {
    int device = 0, dim = 3, prec = 8;
    int nx[3] = {1, 1, 1};
    cudaStream_t stream = nullptr, own_stream = nullptr;
    GridPlan g;
    void *tables = nullptr;
    bool gen = false, nbr2 = true;
    int TJ = 16, ntiles = 1, zb = 1;
    int fastN = 0;            // cubic grid handled by the compile-time specialised kernels (0: generic)
    int r8 = 0;               // 64^3: register-resident 8x8 line transforms (lfts_step_r8.cuh)
    int fast_ok = 0, r8_ok = 0, r12_ok = 0;  // families set up at creation (lfts_set_step_impl)
    int r12 = 0;              // 96^3: register-resident 12x8 plane kernels (lfts_step_r12.cuh)
    int nsm = 0;              // streaming multiprocessors of the device
    int xcap = 0;             // CTAs per SM of the persistent x-passes (0: the kernel's own residency)
    void *stw = nullptr;
    size_t sm_pf1 = 0, sm_pf2 = 0, sm_mid = 0, sm_inv1 = 0, sm_inv2 = 0, sm_x1 = 0, sm_x2 = 0;
    double *partials = nullptr;
    size_t partials_cap = 0;
    lfts_step_job *sjobs = nullptr;
    int sjobs_cap = 0;
    lfts_step_job *sjobs_host = nullptr;
    int *status_host = nullptr;           // pinned words read by lfts_status_wait
    cudaEvent_t status_ev[LFTS_STATUS_SLOTS] = {};
    long long launches = 0;  // kernels enqueued through this context (graph replays excluded)
    // device-controlled loops inside a graph capture (lfts_graph_while_begin/end):
    // the body is captured on body_stream while the outer capture waits on outer_stream
    cudaStream_t body_stream = nullptr, outer_stream = nullptr;
};

struct lfts_graph_s {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

static void make_axis(int n, AxisPlan &ap, std::vector<short> &perm, bool &gen, std::string &err) {
    ap.n = n;
    ap.nf = 0;
    int m = n;
    auto push = [&](int r) {
        if (ap.nf >= LFTS_MAX_FACTORS) { err = "too many FFT factors"; return; }
        ap.radix[ap.nf++] = r;
    };
    while (m % 8 == 0) { push(8); m /= 8; }
    while (m % 4 == 0) { push(4); m /= 4; }
    while (m % 2 == 0) { push(2); m /= 2; }
    while (m % 3 == 0) { push(3); m /= 3; }
    while (m % 5 == 0) { push(5); m /= 5; }
    for (int p = 7; m > 1; p += 2) {
        while (m % p == 0) {
            if (p > LFTS_MAX_RADIX) { err = "grid extent " + std::to_string(n) + " has a prime factor > 64"; return; }
            gen = true;
            push(p);
            m /= p;
        }
    }
    // digit-reversal permutation, outermost radix first
    perm.assign(n, 0);
    for (int t = 0; t < n; t++) {
        int pos = 0, len = n, rem = t;
        for (int f = 0; f < ap.nf; f++) {
            const int r = ap.radix[f];
            len /= r;
            pos += (rem % r) * len;
            rem /= r;
        }
        perm[t] = (short)pos;
    }
}

template <typename T, bool GEN>
__global__ void k_xstress(GridPlan g, const lfts_step_job *__restrict__ sj, const lfts_stress_job *__restrict__ jobs,
                          const double *__restrict__ basis, int TJ, double *partials);

// The dynamic shared-memory limit is a per-kernel, process-wide attribute:
// contexts with different grids share the kernels, so every kernel gets the
// device's opt-in maximum once instead of a per-grid value (a smaller grid's
// context would otherwise lower the limit another context relies on).
// (the dynamic limit is the opt-in maximum minus the kernel's static shared memory)
template <typename K> static cudaError_t allow_smem(K kernel, int max_smem) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem - (int)fa.sharedSizeBytes);
}
template <typename T, bool GEN> static cudaError_t set_attrs_t(int max_smem) {
    cudaError_t e = cudaSuccess, r;
    if ((r = allow_smem(k_plane_forward<T, 1, GEN>, max_smem)) != cudaSuccess) e = r;
    if ((r = allow_smem(k_plane_forward<T, 2, GEN>, max_smem)) != cudaSuccess) e = r;
    if ((r = allow_smem(k_plane_mid<T, GEN>, max_smem)) != cudaSuccess) e = r;
    if ((r = allow_smem(k_plane_inverse<T, 1, EPI_SCALE, GEN>, max_smem)) != cudaSuccess) e = r;
    if ((r = allow_smem(k_plane_inverse<T, 1, EPI_RICH_ACC, GEN>, max_smem)) != cudaSuccess) e = r;
    if ((r = allow_smem(k_plane_inverse<T, 2, EPI_RICH, GEN>, max_smem)) != cudaSuccess) e = r;
    if ((r = allow_smem(k_xpass<T, 1, GEN>, max_smem)) != cudaSuccess) e = r;
    if ((r = allow_smem(k_xpass<T, 2, GEN>, max_smem)) != cudaSuccess) e = r;
    if ((r = allow_smem(k_xstress<T, GEN>, max_smem)) != cudaSuccess) e = r;
    if ((r = allow_smem(k_xpass_forward<T, GEN>, max_smem)) != cudaSuccess) e = r;
    return e;
}

// Attributes of the cubic fast kernels; 0 when their shared memory does not fit.
// Threads per CTA of the two-branch cubic plane kernels (continuous K1 and K5).
// Their shared memory holds two N x (N/2+1) spectrum planes; at 96^3 FP64
// that is 176 KB with 8 warps, so one CTA fits per SM and 512 threads double
// the warps that hide its load and shared-memory latency.
template <typename T, int N> constexpr int fast_nt2() { return (sizeof(T) == 8 && N == 96) ? 512 : NTHR; }

template <typename T, int N> static int fast_setup(int max_smem) {
    using C = typename CT<T>::type;
    constexpr int NT2 = fast_nt2<T, N>();
    const size_t f2 = fast::FSmem<C, N, 2, 1, NT2>::BYTES, f1 = fast::FSmem<C, N, 1, 1>::BYTES;
    const size_t x2 = sizeof(C) * (2 * (size_t)N * (sizeof(T) == 8 ? 16 : 32) + fast::stw_size(N) + 1);
    if (f2 > (size_t)max_smem || x2 > (size_t)max_smem) return 0;
    if (allow_smem(fast::kf_plane_forward<T, 1, N>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(fast::kf_plane_forward<T, 2, N, NT2>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(fast::kf_plane_mid<T, N>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(fast::kf_plane_inverse<T, 2, EPI_RICH, N, NT2>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(fast::kf_plane_inverse<T, 1, EPI_SCALE, N>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(fast::kf_xpass<T, 1, N>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(fast::kf_xpass<T, 2, N>, max_smem) != cudaSuccess) return 0;
    (void)f1;
    return 1;
}

template <typename T> static int r12_setup(int max_smem) {
    using C = typename CT<T>::type;
    if (r12::plane_smem<C>(r12::N) > (size_t)max_smem) return 0;
    if (allow_smem(r12::kq_plane_forward<T, FM_FAC_SQ, FM_FAC>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(r12::kq_plane_mid<T>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(r12::kq_plane_inverse<T>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(r12::kq_xpass<T, 1>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(r12::kq_xpass<T, 2>, max_smem) != cudaSuccess) return 0;
    return 1;
}

template <typename T> static int r8_setup(int max_smem) {
    using C = typename CT<T>::type;
    if (r8::plane_smem<C>() > (size_t)max_smem || r8::xpipe_smem<C>() > (size_t)max_smem) return 0;
    if (allow_smem(r8::kr_plane_forward<T, 1, FM_NONE, FM_NONE>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(r8::kr_plane_forward<T, 2, FM_FAC_SQ, FM_FAC>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(r8::kr_plane_mid<T>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(r8::kr_plane_inverse<T, 2, EPI_RICH>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(r8::kr_plane_inverse<T, 1, EPI_SCALE>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(r8::kp_xpass<T, 1>, max_smem) != cudaSuccess) return 0;
    if (allow_smem(r8::kp_xpass<T, 2>, max_smem) != cudaSuccess) return 0;
    return 1;
}

template <typename T> static int setup_plan(lfts_ctx c) {
    using C = typename CT<T>::type;
    GridPlan &g = c->g;
    const int n[3] = {g.n0, g.n1, g.n2};
    std::vector<short> perm[3];
    std::string err;
    for (int a = 0; a < 3; a++) {
        if (n[a] > LFTS_MAX_AXIS) return fail("grid extent " + std::to_string(n[a]) + " exceeds 1024");
        make_axis(n[a], g.ax[a], perm[a], c->gen, err);
        if (!err.empty()) return fail(err);
    }
    size_t bytes = 0;
    for (int a = 0; a < 3; a++) bytes += sizeof(C) * n[a] + 16 + sizeof(short) * n[a] + 16;
    CK(cudaMalloc(&c->tables, bytes));
    std::vector<unsigned char> host(bytes, 0);
    size_t off = 0;
    for (int a = 0; a < 3; a++) {
        C *tw = (C *)(host.data() + off);
        for (int j = 0; j < n[a]; j++) {
            const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)j / (long double)n[a];
            tw[j].x = (T)std::cos(ang);
            tw[j].y = (T)std::sin(ang);
        }
        g.tw[a] = (const char *)c->tables + off;
        off += (sizeof(C) * n[a] + 15) / 16 * 16;
        std::memcpy(host.data() + off, perm[a].data(), sizeof(short) * n[a]);
        g.perm[a] = (const short *)((const char *)c->tables + off);
        off += (sizeof(short) * n[a] + 15) / 16 * 16;
    }
    CK(cudaMemcpy(c->tables, host.data(), bytes, cudaMemcpyHostToDevice));

    int max_smem = 0;
    CK(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    CK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device));
    max_smem -= 64;  // headroom for static shared memory of the reduction kernels
    c->TJ = (sizeof(T) == 8) ? 16 : 32;
    c->ntiles = (int)((g.n1 * (long long)g.nzc + c->TJ - 1) / c->TJ);
    // z-lines per warp: enough lines that a radix-8 stage keeps 32 lanes busy
    c->zb = g.n2 <= 32 ? 8 : (g.n2 <= 128 ? 4 : 1);
    while (c->zb > 1 && PlaneSmem<C>::bytes(1, g.n1, g.n2, g.nzc, true, c->zb) > (size_t)max_smem) c->zb /= 2;
    c->sm_pf1 = PlaneSmem<C>::bytes(1, g.n1, g.n2, g.nzc, false, c->zb);
    c->sm_pf2 = PlaneSmem<C>::bytes(2, g.n1, g.n2, g.nzc, false, c->zb);
    c->sm_mid = PlaneSmem<C>::bytes(1, g.n1, g.n2, g.nzc, true, c->zb);
    c->sm_inv1 = c->sm_pf1;
    c->sm_inv2 = c->sm_pf2;
    c->sm_x1 = sizeof(C) * (1 * (size_t)g.n0 * c->TJ + g.n0) + sizeof(short) * g.n0;
    c->sm_x2 = sizeof(C) * (2 * (size_t)g.n0 * c->TJ + g.n0) + sizeof(short) * g.n0;
    if ((int)c->sm_mid > max_smem || (int)c->sm_x1 > max_smem)
        return fail("grid plane " + std::to_string(g.n1) + "x" + std::to_string(g.n2) +
                    " does not fit in shared memory (" + std::to_string(c->sm_mid) + " > " + std::to_string(max_smem) + " bytes)");
    c->nbr2 = (int)c->sm_pf2 <= max_smem && (int)c->sm_x2 <= max_smem;
    CK((c->gen ? set_attrs_t<T, true>(max_smem) : set_attrs_t<T, false>(max_smem)));
    g.stw = nullptr;
    if (g.n0 == g.n1 && g.n1 == g.n2 && !std::getenv("LFTS_NO_FAST")) {
        const int N = g.n0;
        int ok = 0;
        switch (N) {
            case 16: ok = fast_setup<T, 16>(max_smem); break;
            case 32: ok = fast_setup<T, 32>(max_smem); break;
            case 48: ok = fast_setup<T, 48>(max_smem); break;
            case 64: ok = fast_setup<T, 64>(max_smem); break;
            case 96: ok = fast_setup<T, 96>(max_smem); break;
            case 128: ok = fast_setup<T, 128>(max_smem); break;
            default: ok = 0;
        }
        if (ok) {
            // per-stage twiddles w_L^(j k1), stage s (innermost first) at stw_offset, [j-1][k1]
            const int nf = fast::nrad(N);
            std::vector<C> h(fast::stw_size(N) + 1);
            for (int st = 0; st < nf; st++) {
                const int R = fast::rad(N, nf - 1 - st), M = fast::span_inner(N, st), L = M * R;
                const int off = fast::stw_offset(N, st);
                for (int j = 1; j < R; j++)
                    for (int k1 = 0; k1 < M; k1++) {
                        const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)(j * k1) / (long double)L;
                        h[off + (j - 1) * M + k1].x = (T)std::cos(a);
                        h[off + (j - 1) * M + k1].y = (T)std::sin(a);
                    }
            }
            CK(cudaMalloc(&c->stw, sizeof(C) * h.size()));
            CK(cudaMemcpy(c->stw, h.data(), sizeof(C) * h.size(), cudaMemcpyHostToDevice));
            g.stw = c->stw;
            c->fastN = N;
            if (N == 64 && !std::getenv("LFTS_NO_R8")) c->r8 = r8_setup<T>(max_smem);
            if (N == 96 && !std::getenv("LFTS_NO_R12")) c->r12 = r12_setup<T>(max_smem);
            c->fast_ok = N;
            c->r8_ok = c->r8;
            c->r12_ok = c->r12;
        }
    }
    return 0;
}

extern "C" const char *lfts_last_error(void) { return g_err.c_str(); }

extern "C" int lfts_ctx_create(lfts_ctx *out, int device, int dim, const int *nx, int precision) {
    if (!out || !nx) return fail("null argument");
    if (dim < 1 || dim > 3) return fail("dim must be 1, 2 or 3");
    if (precision != 8 && precision != 4) return fail("precision must be 8 (double) or 4 (float)");
    for (int d = 0; d < dim; d++)
        if (nx[d] < 1) return fail("grid extents must be positive");
    auto *c = new lfts_ctx_s();
    c->device = device;
    c->dim = dim;
    c->prec = precision;
    int t[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) t[3 - dim + d] = nx[d];
    for (int d = 0; d < 3; d++) c->nx[d] = t[d];
    GridPlan &g = c->g;
    g.n0 = t[0];
    g.n1 = t[1];
    g.n2 = t[2];
    g.nzc = g.n2 / 2 + 1;
    g.M = (long long)g.n0 * g.n1 * g.n2;
    g.Mc = (long long)g.n0 * g.n1 * g.nzc;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { delete c; return fail(std::string("cudaSetDevice: ") + cudaGetErrorString(e)); }
    e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete c; return fail(std::string("cudaStreamCreate: ") + cudaGetErrorString(e)); }
    c->stream = c->own_stream;
    int rc = (precision == 8) ? setup_plan<double>(c) : setup_plan<float>(c);
    if (rc != 0) { lfts_ctx_destroy(c); return rc; }
    c->partials_cap = 1 << 20;
    c->sjobs_cap = 2048;
    if (cudaMalloc(&c->partials, sizeof(double) * c->partials_cap) != cudaSuccess ||
        cudaMalloc(&c->sjobs, sizeof(lfts_step_job) * c->sjobs_cap) != cudaSuccess ||
        cudaMallocHost(&c->sjobs_host, sizeof(lfts_step_job) * c->sjobs_cap) != cudaSuccess ||
        cudaMallocHost(&c->status_host, sizeof(int) * LFTS_STATUS_SLOTS) != cudaSuccess) {
        lfts_ctx_destroy(c);
        return fail("workspace allocation failed");
    }
    for (int i = 0; i < LFTS_STATUS_SLOTS; i++)
        if (cudaEventCreateWithFlags(&c->status_ev[i], cudaEventDisableTiming) != cudaSuccess) {
            lfts_ctx_destroy(c);
            return fail("event creation failed");
        }
    *out = c;
    return 0;
}

extern "C" int lfts_ctx_destroy(lfts_ctx c) {
    if (!c) return 0;
    cudaSetDevice(c->device);
    if (c->tables) cudaFree(c->tables);
    if (c->stw) cudaFree(c->stw);
    if (c->partials) cudaFree(c->partials);
    if (c->sjobs) cudaFree(c->sjobs);
    if (c->sjobs_host) cudaFreeHost(c->sjobs_host);
    if (c->status_host) cudaFreeHost(c->status_host);
    for (int i = 0; i < LFTS_STATUS_SLOTS; i++)
        if (c->status_ev[i]) cudaEventDestroy(c->status_ev[i]);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    if (c->body_stream) cudaStreamDestroy(c->body_stream);
    delete c;
    return 0;
}

extern "C" int lfts_ctx_set_stream(lfts_ctx c, void *stream) {
    if (!c) return fail("null context");
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return 0;
}
extern "C" void *lfts_ctx_stream(lfts_ctx c) { return c ? (void *)c->stream : nullptr; }
extern "C" int lfts_ctx_info(lfts_ctx c, long long *M, long long *Mc, int *prec) {
    if (!c) return fail("null context");
    if (M) *M = c->g.M;
    if (Mc) *Mc = c->g.Mc;
    if (prec) *prec = c->prec;
    return 0;
}

extern "C" int lfts_malloc(lfts_ctx c, void **ptr, size_t bytes) {
    if (!c || !ptr) return fail("null argument");
    CK(cudaSetDevice(c->device));
    CK(cudaMalloc(ptr, bytes ? bytes : 16));
    return 0;
}
extern "C" int lfts_free(lfts_ctx c, void *ptr) {
    if (!c) return fail("null context");
    if (ptr) CK(cudaFree(ptr));
    return 0;
}
extern "C" int lfts_malloc_host(lfts_ctx c, void **ptr, size_t bytes) {
    if (!c || !ptr) return fail("null argument");
    CK(cudaSetDevice(c->device));
    void *h = nullptr, *d = nullptr;
    CK(cudaHostAlloc(&h, bytes ? bytes : 16, cudaHostAllocMapped | cudaHostAllocPortable));
    const cudaError_t e = cudaHostGetDevicePointer(&d, h, 0);
    if (e != cudaSuccess || d != h) {
        cudaFreeHost(h);
        return fail("lfts_malloc_host: the pinned allocation has no device address equal to its host address");
    }
    *ptr = h;
    return 0;
}
extern "C" int lfts_free_host(lfts_ctx c, void *ptr) {
    if (!c) return fail("null context");
    if (ptr) CK(cudaFreeHost(ptr));
    return 0;
}
extern "C" int lfts_memset_async(lfts_ctx c, void *ptr, int v, size_t bytes) {
    CK(cudaMemsetAsync(ptr, v, bytes, c->stream));
    return 0;
}
extern "C" int lfts_memcpy_h2d(lfts_ctx c, void *dst, const void *src, size_t bytes) {
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c->stream));  // dst may be mapped host memory
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}
// Read and clear the device error word that kernels set instead of spinning
// forever or touching a misaligned copy (called after a stream synchronisation).
static int check_kernel_errors() {
    unsigned int e = 0;
    CK(cudaMemcpyFromSymbol(&e, g_kerr, sizeof e));
    if (!e) return 0;
    const unsigned int z = 0;
    CK(cudaMemcpyToSymbol(g_kerr, &z, sizeof z));
    std::string what;
    if (e & KERR_WAIT_TIMEOUT) what += " a kernel's wait for its bulk copies timed out;";
    if (e & KERR_MISALIGNED) what += " a spectrum buffer is not 16-byte aligned;";
    return fail("device error word " + std::to_string(e) + ":" + what + " results of the affected launch are invalid");
}

extern "C" int lfts_memcpy_d2h(lfts_ctx c, void *dst, const void *src, size_t bytes) {
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return check_kernel_errors();
}
extern "C" int lfts_memcpy_d2d_async(lfts_ctx c, void *dst, const void *src, size_t bytes) {
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c->stream));  // either side may be mapped host memory
    return 0;
}
extern "C" int lfts_status_post(lfts_ctx c, const int *d_word, int slot) {
    if (!c || !d_word) return fail("null argument");
    if (slot < 0 || slot >= LFTS_STATUS_SLOTS) return fail("status slot out of range");
    CK(cudaMemcpyAsync(c->status_host + slot, d_word, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaEventRecord(c->status_ev[slot], c->stream));
    return 0;
}
extern "C" int lfts_status_wait(lfts_ctx c, int slot, int *value) {
    if (!c || !value) return fail("null argument");
    if (slot < 0 || slot >= LFTS_STATUS_SLOTS) return fail("status slot out of range");
    CK(cudaEventSynchronize(c->status_ev[slot]));
    *value = c->status_host[slot];
    return check_kernel_errors();
}
extern "C" int lfts_synchronize(lfts_ctx c) {
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaGetLastError());
    return check_kernel_errors();
}

extern "C" int lfts_graph_begin(lfts_ctx c) {
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    return 0;
}
extern "C" int lfts_graph_end(lfts_ctx c, lfts_graph *out) {
    auto *gr = new lfts_graph_s();
    cudaError_t e = cudaStreamEndCapture(c->stream, &gr->graph);
    if (e != cudaSuccess) { delete gr; return fail(std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e)); }
    e = cudaGraphInstantiate(&gr->exec, gr->graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(gr->graph);
        delete gr;
        return fail(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }
    *out = gr;
    return 0;
}
// A conditional WHILE node after the work captured so far on the context
// stream; the context stream then points at a private stream that captures
// into the node's body graph until lfts_graph_while_end.  The handle starts at
// 1 on every launch of the graph (cudaGraphCondAssignDefault), so the body
// runs at least once; device code in the body sets it (lfts_saddle_next).
extern "C" int lfts_graph_while_begin(lfts_ctx c, unsigned long long *handle) {
    if (!c || !handle) return fail("null argument");
    if (c->outer_stream) return fail("lfts_graph_while_begin: loops do not nest");
    cudaStreamCaptureStatus status;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    CK(cudaStreamGetCaptureInfo(c->stream, &status, nullptr, &g, &deps, &ndeps));
    if (status != cudaStreamCaptureStatusActive || !g) return fail("lfts_graph_while_begin: the context stream is not capturing");
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};  // the rest zero-initialised
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, ndeps, &np));
    CK(cudaStreamUpdateCaptureDependencies(c->stream, &node, 1, cudaStreamSetCaptureDependencies));
    if (!c->body_stream) CK(cudaStreamCreateWithFlags(&c->body_stream, cudaStreamNonBlocking));
    CK(cudaStreamBeginCaptureToGraph(c->body_stream, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    c->outer_stream = c->stream;
    c->stream = c->body_stream;
    *handle = (unsigned long long)h;
    return 0;
}
extern "C" int lfts_graph_while_end(lfts_ctx c) {
    if (!c) return fail("null context");
    if (!c->outer_stream) return fail("lfts_graph_while_end without lfts_graph_while_begin");
    cudaGraph_t body = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->body_stream, &body);
    c->stream = c->outer_stream;
    c->outer_stream = nullptr;
    if (e != cudaSuccess) return fail(std::string("lfts_graph_while_end: cudaStreamEndCapture: ") + cudaGetErrorString(e));
    return 0;
}
extern "C" int lfts_graph_launch(lfts_ctx c, lfts_graph g) {
    CK(cudaGraphLaunch(g->exec, c->stream));
    return 0;
}
extern "C" int lfts_graph_destroy(lfts_graph g) {
    if (!g) return 0;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return 0;
}

// ---------------------------------------------------------------- tables
// Boltzmann bond factor, same arithmetic as the reference's Pseudo.cpp:17-82
// (xfactor from nx*dx, integer wave numbers folded at n/2), then / M.
template <typename T>
static int bond_tables_t(lfts_ctx c, double b2, double ds, const double *lx, void *b_out, void *bh_out) {
    const GridPlan &g = c->g;
    const int tn[3] = {g.n0, g.n1, g.n2};
    double tdx[3] = {1.0, 1.0, 1.0};
    for (int d = 0; d < c->dim; d++) tdx[3 - c->dim + d] = lx[d] / c->nx[3 - c->dim + d];
    const double PI = 3.14159265358979323846;
    std::vector<T> hb(g.Mc), hh(g.Mc);
    double xf[3], xh[3];
    for (int d = 0; d < 3; d++) {
        xf[d] = -b2 * std::pow(2 * PI / (tn[d] * tdx[d]), 2) * ds / 6.0;
        xh[d] = -(b2 / 2) * std::pow(2 * PI / (tn[d] * tdx[d]), 2) * ds / 6.0;
    }
    const double invM = 1.0 / (double)g.M;
    for (int i = 0; i < tn[0]; i++) {
        const int it = i > tn[0] / 2 ? tn[0] - i : i;
        for (int j = 0; j < tn[1]; j++) {
            const int jt = j > tn[1] / 2 ? tn[1] - j : j;
            for (int k = 0; k < g.nzc; k++) {
                const long long idx = ((long long)i * tn[1] + j) * g.nzc + k;
                hb[idx] = (T)(std::exp(it * it * xf[0] + jt * jt * xf[1] + k * k * xf[2]) * invM);
                hh[idx] = (T)(std::exp(it * it * xh[0] + jt * jt * xh[1] + k * k * xh[2]) * invM);
            }
        }
    }
    CK(cudaMemcpyAsync(b_out, hb.data(), sizeof(T) * g.Mc, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(bh_out, hh.data(), sizeof(T) * g.Mc, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}
extern "C" int lfts_bond_tables(lfts_ctx c, double b2, double ds, const double *lx, void *b_out, void *bh_out) {
    if (!c || !lx || !b_out || !bh_out) return fail("null argument");
    return c->prec == 8 ? bond_tables_t<double>(c, b2, ds, lx, b_out, bh_out)
                        : bond_tables_t<float>(c, b2, ds, lx, b_out, bh_out);
}

// Pseudo.cpp:84-153: k_d^2 (2 pi / L_d)^2, doubled for 0 < kz < n2/2
extern "C" int lfts_fourier_basis(lfts_ctx c, const double *lx, double *basis_out) {
    if (!c || !lx || !basis_out) return fail("null argument");
    const GridPlan &g = c->g;
    const int tn[3] = {g.n0, g.n1, g.n2};
    double tdx[3] = {1.0, 1.0, 1.0};
    for (int d = 0; d < c->dim; d++) tdx[3 - c->dim + d] = lx[d] / c->nx[3 - c->dim + d];
    const double PI = 3.14159265358979323846;
    double xf[3];
    for (int d = 0; d < 3; d++) xf[d] = std::pow(2 * PI / (tn[d] * tdx[d]), 2);
    std::vector<double> h(3 * g.Mc);
    for (int i = 0; i < tn[0]; i++) {
        const int it = i > tn[0] / 2 ? tn[0] - i : i;
        for (int j = 0; j < tn[1]; j++) {
            const int jt = j > tn[1] / 2 ? tn[1] - j : j;
            for (int k = 0; k < g.nzc; k++) {
                const long long idx = ((long long)i * tn[1] + j) * g.nzc + k;
                double bx = it * it * xf[0], by = jt * jt * xf[1], bz = k * k * xf[2];
                if (k != 0 && 2 * k != tn[2]) { bx *= 2; by *= 2; bz *= 2; }
                h[idx] = bx;
                h[g.Mc + idx] = by;
                h[2 * g.Mc + idx] = bz;
            }
        }
    }
    CK(cudaMemcpyAsync(basis_out, h.data(), sizeof(double) * 3 * g.Mc, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

template <typename T>
__global__ void k_field_factors(const double *__restrict__ w, double coef, T *__restrict__ fac, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        fac[i] = (T)exp(coef * w[i]);
}
static int grid_for(long long n) {
    long long b = (n + NTHR - 1) / NTHR;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b < 1 ? 1 : b);
}
extern "C" int lfts_field_factors(lfts_ctx c, const double *w, double coef, void *fac_out) {
    if (!c || !w || !fac_out) return fail("null argument");
    if (c->prec == 8)
        k_field_factors<double><<<grid_for(c->g.M), NTHR, 0, c->stream>>>(w, coef, (double *)fac_out, c->g.M);
    else
        k_field_factors<float><<<grid_for(c->g.M), NTHR, 0, c->stream>>>(w, coef, (float *)fac_out, c->g.M);
    c->launches += 1;
    CKLAUNCH();
    return 0;
}

// ---------------------------------------------------------------- steps
template <typename T, int N>
static int step_cont_fast(lfts_ctx c, const lfts_step_job *jobs, int nj, int s) {
    using C = typename CT<T>::type;
    const GridPlan &g = c->g;
    cudaStream_t st = c->stream;
    constexpr int TJ = sizeof(T) == 8 ? 16 : 32;
    const dim3 gp(N, nj), gx((unsigned)(((long long)N * (N / 2 + 1) + TJ - 1) / TJ), nj);
    constexpr int NT2 = fast_nt2<T, N>();
    const size_t f2 = fast::FSmem<C, N, 2, 1, NT2>::BYTES, f1 = fast::FSmem<C, N, 1, 1>::BYTES;
    const size_t x2 = sizeof(C) * (2 * (size_t)N * TJ + fast::stw_size(N) + 1);
    const size_t x1 = sizeof(C) * ((size_t)N * TJ + fast::stw_size(N) + 1);
    if constexpr (N == r8::N) {
        if (c->r8) {
            const dim3 rp(N, nj);
            const size_t ps = r8::plane_smem<C>();
            const long long it2 = (long long)nj * 2 * r8::xpipe_tiles<C>(), it1 = (long long)nj * r8::xpipe_tiles<C>(), cap = (long long)(c->xcap ? c->xcap : 3) * c->nsm;
            const dim3 px2((unsigned)(it2 < cap ? it2 : cap)), px1((unsigned)(it1 < cap ? it1 : cap));
            r8::kr_plane_forward<T, 2, FM_FAC_SQ, FM_FAC><<<rp, NTHR, ps, st>>>(g, jobs, s, 0);
            r8::kp_xpass<T, 2><<<px2, NTHR, r8::xpipe_smem<C>(), st>>>(g, jobs, nj, 0, 0, 1);
            r8::kr_plane_mid<T><<<rp, NTHR, ps, st>>>(g, jobs, 1);
            r8::kp_xpass<T, 1><<<px1, NTHR, r8::xpipe_smem<C>(), st>>>(g, jobs, nj, 1, 1, 1);
            r8::kr_plane_inverse<T, 2, EPI_RICH><<<rp, NTHR, ps, st>>>(g, jobs, s, 0, 0);
            CKLAUNCH();
            return 0;
        }
    }
    if constexpr (N == r12::N) {
        if (c->r12) {
            const size_t p2 = r12::plane_smem<C>(N), p1 = r12::plane_smem<C>(N / 2), xs = r12::xpipe_smem<C>();
            const long long it2 = (long long)nj * 2 * r12::XTILES, it1 = (long long)nj * r12::XTILES;
            const long long cap = (long long)(c->xcap ? c->xcap : r12::minb_xpass<T>()) * c->nsm;
            r12::kq_plane_forward<T, FM_FAC_SQ, FM_FAC><<<gp, r12::NT, p2, st>>>(g, jobs, s, 0);
            r12::kq_xpass<T, 2><<<(unsigned)(it2 < cap ? it2 : cap), NTHR, xs, st>>>(g, jobs, nj, 0, 0, 1);
            r12::kq_plane_mid<T><<<gp, r12::NT, p1, st>>>(g, jobs, 1);
            r12::kq_xpass<T, 1><<<(unsigned)(it1 < cap ? it1 : cap), NTHR, xs, st>>>(g, jobs, nj, 1, 1, 1);
            r12::kq_plane_inverse<T><<<gp, r12::NT, p2, st>>>(g, jobs, s, 0);
            CKLAUNCH();
            return 0;
        }
    }
    fast::kf_plane_forward<T, 2, N, NT2><<<gp, NT2, f2, st>>>(g, jobs, s, FM_FAC_SQ, FM_FAC, 0);
    fast::kf_xpass<T, 2, N><<<gx, NTHR, x2, st>>>(g, jobs, 0, 0, 1);
    fast::kf_plane_mid<T, N><<<gp, NTHR, f1, st>>>(g, jobs, 1);
    fast::kf_xpass<T, 1, N><<<gx, NTHR, x1, st>>>(g, jobs, 1, 1, 1);
    fast::kf_plane_inverse<T, 2, EPI_RICH, N, NT2><<<gp, NT2, f2, st>>>(g, jobs, s, 0, 0);
    CKLAUNCH();
    return 0;
}
template <typename T, int N>
static int step_disc_fast(lfts_ctx c, const lfts_step_job *jobs, int nj, int s, int half, int with_fac) {
    using C = typename CT<T>::type;
    const GridPlan &g = c->g;
    cudaStream_t st = c->stream;
    constexpr int TJ = sizeof(T) == 8 ? 16 : 32;
    const dim3 gp(N, nj), gx((unsigned)(((long long)N * (N / 2 + 1) + TJ - 1) / TJ), nj);
    const size_t f1 = fast::FSmem<C, N, 1, 1>::BYTES;
    const size_t x1 = sizeof(C) * ((size_t)N * TJ + fast::stw_size(N) + 1);
    if constexpr (N == r8::N) {
        if (c->r8) {
            const dim3 rp(N, nj);
            const size_t ps = r8::plane_smem<C>();
            r8::kr_plane_forward<T, 1, FM_NONE, FM_NONE><<<rp, NTHR, ps, st>>>(g, jobs, s, 0);
            const long long it1 = (long long)nj * r8::xpipe_tiles<C>(), cap = (long long)(c->xcap ? c->xcap : 3) * c->nsm;
            r8::kp_xpass<T, 1><<<(unsigned)(it1 < cap ? it1 : cap), NTHR, r8::xpipe_smem<C>(), st>>>(g, jobs, nj, 0, half, half);
            r8::kr_plane_inverse<T, 1, EPI_SCALE><<<rp, NTHR, ps, st>>>(g, jobs, s, 0, with_fac ? FM_FAC : FM_NONE);
            CKLAUNCH();
            return 0;
        }
    }
    fast::kf_plane_forward<T, 1, N><<<gp, NTHR, f1, st>>>(g, jobs, s, FM_NONE, 0, 0);
    fast::kf_xpass<T, 1, N><<<gx, NTHR, x1, st>>>(g, jobs, 0, half, half);
    fast::kf_plane_inverse<T, 1, EPI_SCALE, N><<<gp, NTHR, f1, st>>>(g, jobs, s, 0, with_fac ? FM_FAC : FM_NONE);
    CKLAUNCH();
    return 0;
}
template <typename T>
static int step_fast_dispatch(lfts_ctx c, const lfts_step_job *jobs, int nj, int s, int disc, int half, int wf) {
    switch (c->fastN) {
        case 16: return disc ? step_disc_fast<T, 16>(c, jobs, nj, s, half, wf) : step_cont_fast<T, 16>(c, jobs, nj, s);
        case 32: return disc ? step_disc_fast<T, 32>(c, jobs, nj, s, half, wf) : step_cont_fast<T, 32>(c, jobs, nj, s);
        case 48: return disc ? step_disc_fast<T, 48>(c, jobs, nj, s, half, wf) : step_cont_fast<T, 48>(c, jobs, nj, s);
        case 64: return disc ? step_disc_fast<T, 64>(c, jobs, nj, s, half, wf) : step_cont_fast<T, 64>(c, jobs, nj, s);
        case 96: return disc ? step_disc_fast<T, 96>(c, jobs, nj, s, half, wf) : step_cont_fast<T, 96>(c, jobs, nj, s);
        case 128: return disc ? step_disc_fast<T, 128>(c, jobs, nj, s, half, wf) : step_cont_fast<T, 128>(c, jobs, nj, s);
    }
    return fail("no specialised kernels for this grid");
}

template <typename T, bool GEN>
static int step_cont_t(lfts_ctx c, const lfts_step_job *jobs, int nj, int s) {
    const GridPlan &g = c->g;
    cudaStream_t st = c->stream;
    const dim3 gp(g.n0, nj), gx(c->ntiles, nj);
    if (c->nbr2) {
        k_plane_forward<T, 2, GEN><<<gp, NTHR, c->sm_pf2, st>>>(g, jobs, s, FM_FAC_SQ, FM_FAC, 0, c->zb);
        k_xpass<T, 2, GEN><<<gx, NTHR, c->sm_x2, st>>>(g, jobs, 0, 0, 1, c->TJ);
    } else {
        k_plane_forward<T, 1, GEN><<<gp, NTHR, c->sm_pf1, st>>>(g, jobs, s, FM_FAC_SQ, 0, 0, c->zb);
        k_plane_forward<T, 1, GEN><<<gp, NTHR, c->sm_pf1, st>>>(g, jobs, s, FM_FAC, 0, 1, c->zb);
        k_xpass<T, 1, GEN><<<gx, NTHR, c->sm_x1, st>>>(g, jobs, 0, 0, 0, c->TJ);
        k_xpass<T, 1, GEN><<<gx, NTHR, c->sm_x1, st>>>(g, jobs, 1, 1, 1, c->TJ);
    }
    k_plane_mid<T, GEN><<<gp, NTHR, c->sm_mid, st>>>(g, jobs, 1, c->zb);
    k_xpass<T, 1, GEN><<<gx, NTHR, c->sm_x1, st>>>(g, jobs, 1, 1, 1, c->TJ);
    if (c->nbr2) {
        k_plane_inverse<T, 2, EPI_RICH, GEN><<<gp, NTHR, c->sm_inv2, st>>>(g, jobs, s, 0, 0, c->zb);
    } else {
        k_plane_inverse<T, 1, EPI_SCALE, GEN><<<gp, NTHR, c->sm_inv1, st>>>(g, jobs, s, 0, FM_FAC_SQ, c->zb);
        k_plane_inverse<T, 1, EPI_RICH_ACC, GEN><<<gp, NTHR, c->sm_inv1, st>>>(g, jobs, s, 1, 0, c->zb);
    }
    CKLAUNCH();
    return 0;
}
extern "C" int lfts_step_continuous(lfts_ctx c, const lfts_step_job *jobs, int nj, int s) {
    if (!c || !jobs) return fail("null argument");
    if (nj <= 0) return 0;
    if (nj > 65535) return fail("too many jobs in one launch (max 65535)");
    if (c->fastN) {
        c->launches += 5;
        return c->prec == 8 ? step_fast_dispatch<double>(c, jobs, nj, s, 0, 0, 0) : step_fast_dispatch<float>(c, jobs, nj, s, 0, 0, 0);
    }
    c->launches += c->nbr2 ? 5 : 8;
    if (c->prec == 8) return c->gen ? step_cont_t<double, true>(c, jobs, nj, s) : step_cont_t<double, false>(c, jobs, nj, s);
    return c->gen ? step_cont_t<float, true>(c, jobs, nj, s) : step_cont_t<float, false>(c, jobs, nj, s);
}

template <typename T, bool GEN>
static int step_disc_t(lfts_ctx c, const lfts_step_job *jobs, int nj, int s, int half, int with_fac) {
    const GridPlan &g = c->g;
    cudaStream_t st = c->stream;
    const dim3 gp(g.n0, nj), gx(c->ntiles, nj);
    k_plane_forward<T, 1, GEN><<<gp, NTHR, c->sm_pf1, st>>>(g, jobs, s, FM_NONE, 0, 0, c->zb);
    k_xpass<T, 1, GEN><<<gx, NTHR, c->sm_x1, st>>>(g, jobs, 0, half, half, c->TJ);
    k_plane_inverse<T, 1, EPI_SCALE, GEN><<<gp, NTHR, c->sm_inv1, st>>>(g, jobs, s, 0, with_fac ? FM_FAC : FM_NONE, c->zb);
    CKLAUNCH();
    return 0;
}
extern "C" int lfts_step_discrete(lfts_ctx c, const lfts_step_job *jobs, int nj, int s, int half, int with_fac) {
    if (!c || !jobs) return fail("null argument");
    if (nj <= 0) return 0;
    if (nj > 65535) return fail("too many jobs in one launch (max 65535)");
    half = half ? 1 : 0;
    c->launches += 3;
    if (c->fastN)
        return c->prec == 8 ? step_fast_dispatch<double>(c, jobs, nj, s, 1, half, with_fac)
                            : step_fast_dispatch<float>(c, jobs, nj, s, 1, half, with_fac);
    if (c->prec == 8)
        return c->gen ? step_disc_t<double, true>(c, jobs, nj, s, half, with_fac) : step_disc_t<double, false>(c, jobs, nj, s, half, with_fac);
    return c->gen ? step_disc_t<float, true>(c, jobs, nj, s, half, with_fac) : step_disc_t<float, false>(c, jobs, nj, s, half, with_fac);
}

// ---------------------------------------------------------------- junctions
template <typename T>
__global__ void k_junctions(const lfts_junction_job *__restrict__ jobs, const void *const *__restrict__ deps,
                            const double *__restrict__ wts, long long M) {
    const lfts_junction_job jb = jobs[blockIdx.y];
    T *out = (T *)jb.out;
    const T *fac = (const T *)jb.fac;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M; i += (long long)gridDim.x * blockDim.x) {
        T v;
        if (jb.ndeps == 0) {
            v = (T)1;
        } else if (jb.mode == 0) {
            v = (T)1;
            for (int d = 0; d < jb.ndeps; d++) v *= ((const T *)deps[jb.dep_offset + d])[i];
        } else {
            v = (T)0;
            for (int d = 0; d < jb.ndeps; d++) v += ((const T *)deps[jb.dep_offset + d])[i] * (T)wts[jb.dep_offset + d];
        }
        if (fac) v *= fac[i];
        out[i] = v;
    }
}
extern "C" int lfts_junctions(lfts_ctx c, const lfts_junction_job *jobs, int nj, const void *const *dep_ptrs,
                              const double *dep_weights) {
    if (!c || !jobs) return fail("null argument");
    if (nj <= 0) return 0;
    long long b = (c->g.M + NTHR - 1) / NTHR;
    if (b > 1024) b = 1024;
    const dim3 grid((unsigned)b, nj);
    if (c->prec == 8) k_junctions<double><<<grid, NTHR, 0, c->stream>>>(jobs, dep_ptrs, dep_weights, c->g.M);
    else k_junctions<float><<<grid, NTHR, 0, c->stream>>>(jobs, dep_ptrs, dep_weights, c->g.M);
    c->launches += 1;
    CKLAUNCH();
    return 0;
}

// ---------------------------------------------------------------- reductions
// warp + block sum of a double (block of NTHR threads); result valid in thread 0
__device__ __forceinline__ double block_sum(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    v = 0;
    if (w == 0) {
        v = lane < NWARP ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

// Compensated (error-free transform) summation for the FP32 propagator form:
// sums of FP32 products are accumulated in FP64 as a pair (s, c) where s is
// the running sum and c the running sum of the rounding errors of every
// addition (Knuth's two-sum; Neumaier's improvement of Kahan's method), and
// reduced across threads with the same transform.  The FP64 form keeps the
// plain FP64 sums.
__device__ __forceinline__ void comp_add(double &s, double &c, double x) {
    const double t = s + x;
    const double bp = t - s;
    c += (s - (t - bp)) + (x - bp);
    s = t;
}
// block sum of compensated pairs (block of NTHR threads, sh holds 2 * NWARP
// doubles); s + c of the block is valid in thread 0
__device__ __forceinline__ double block_sum_comp(double s, double c, double *sh) {
    for (int o = 16; o > 0; o >>= 1) {
        const double so = __shfl_down_sync(0xffffffffu, s, o), co = __shfl_down_sync(0xffffffffu, c, o);
        comp_add(s, c, so);
        c += co;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) { sh[w] = s; sh[NWARP + w] = c; }
    __syncthreads();
    s = 0.0;
    c = 0.0;
    if (w == 0) {
        s = lane < NWARP ? sh[lane] : 0.0;
        c = lane < NWARP ? sh[NWARP + lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            const double so = __shfl_down_sync(0xffffffffu, s, o), co = __shfl_down_sync(0xffffffffu, c, o);
            comp_add(s, c, so);
            c += co;
        }
    }
    return s + c;
}
template <typename T>
struct Acc {  // plain FP64 sum for T = double, compensated FP64 sum for T = float
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x) {
        if (sizeof(T) == 4) comp_add(s, c, x);
        else s += x;
    }
    __device__ __forceinline__ double value() const { return s + c; }
    __device__ __forceinline__ double block(double *sh) const {
        return sizeof(T) == 4 ? block_sum_comp(s, c, sh) : block_sum(s, sh);
    }
};

constexpr int DOT_CHUNKS = 128;

template <typename T>
__global__ void __launch_bounds__(NTHR) k_dots(const lfts_dot_job *__restrict__ jobs, long long M, double *partials) {
    __shared__ double sh[2 * NWARP];
    const lfts_dot_job jb = jobs[blockIdx.y];
    const T *a = (const T *)jb.a, *b = (const T *)jb.b, *w = (const T *)jb.w;
    Acc<T> acc;
    for (long long i = blockIdx.x * (long long)NTHR + threadIdx.x; i < M; i += (long long)gridDim.x * NTHR) {
        double v = (double)a[i] * (double)b[i];  // exact for FP32 operands
        if (w) v /= (double)w[i];
        acc.add(v);
    }
    const double v = acc.block(sh);
    if (threadIdx.x == 0) partials[(long long)blockIdx.y * gridDim.x + blockIdx.x] = v;
}
// T selects the summation of the partials as in Acc<T> (compensated for float)
template <typename T = double>
__global__ void __launch_bounds__(NTHR) k_finish(const double *__restrict__ partials, int nparts, const double *scale_src,
                                                 int scale_stride, double mult, double *out, int out_stride, int ncomp) {
    // job = blockIdx.x; component = blockIdx.y; partials[(job*nparts + p)*ncomp + comp]
    __shared__ double sh[2 * NWARP];
    const int j = blockIdx.x, d = blockIdx.y;
    Acc<T> a;
    for (int p = threadIdx.x; p < nparts; p += NTHR) a.add(partials[((long long)j * nparts + p) * ncomp + d]);
    const double acc = a.block(sh);
    if (threadIdx.x == 0) {
        const double sc = scale_src ? *(const double *)((const char *)scale_src + (long long)j * scale_stride) : 1.0;
        out[(long long)j * out_stride + d] = acc * sc * mult;
    }
}
extern "C" int lfts_dots(lfts_ctx c, const lfts_dot_job *jobs, int nj, double *out) {
    if (!c || !jobs || !out) return fail("null argument");
    for (int j0 = 0; j0 < nj; j0 += 4096) {
        const int n = nj - j0 < 4096 ? nj - j0 : 4096;
        const dim3 grid(DOT_CHUNKS, n);
        if (c->prec == 8) {
            k_dots<double><<<grid, NTHR, 0, c->stream>>>(jobs + j0, c->g.M, c->partials);
            k_finish<double><<<dim3(n, 1), NTHR, 0, c->stream>>>(c->partials, DOT_CHUNKS, (const double *)&jobs[j0].scale,
                                                                (int)sizeof(lfts_dot_job), 1.0, out + j0, 1, 1);
        } else {
            k_dots<float><<<grid, NTHR, 0, c->stream>>>(jobs + j0, c->g.M, c->partials);
            k_finish<float><<<dim3(n, 1), NTHR, 0, c->stream>>>(c->partials, DOT_CHUNKS, (const double *)&jobs[j0].scale,
                                                               (int)sizeof(lfts_dot_job), 1.0, out + j0, 1, 1);
        }
        c->launches += 2;
    }
    CKLAUNCH();
    return 0;
}

// block concentrations
template <typename T, int MODEL>
__global__ void __launch_bounds__(NTHR) k_phi(const lfts_phi_job *__restrict__ jobs, const double *__restrict__ coefs,
                                              long long M) {
    const lfts_phi_job jb = jobs[blockIdx.y];
    const T *ql = (const T *)jb.q_left, *qr = (const T *)jb.q_right;
    const double norm = jb.q_div ? jb.norm / *jb.q_div : jb.norm;
    for (long long i = blockIdx.x * (long long)NTHR + threadIdx.x; i < M; i += (long long)gridDim.x * NTHR) {
        Acc<T> a;
        double acc;
        if (MODEL == 0) {
            for (int n = 0; n <= jb.n_right; n++)
                a.add(coefs[jb.coef_offset + n] * (double)ql[(long long)(jb.n_left - n) * M + i] * (double)qr[(long long)n * M + i]);
            acc = a.value();
        } else {
            for (int n = 1; n <= jb.n_right; n++)
                a.add((double)ql[(long long)(jb.n_left - n + 1) * M + i] * (double)qr[(long long)n * M + i]);
            acc = a.value() / (double)((const T *)jb.fac)[i];
        }
        jb.phi[i] = acc * norm;
    }
}
extern "C" int lfts_phi_blocks(lfts_ctx c, int model, const lfts_phi_job *jobs, int nj, const double *coefs) {
    if (!c || !jobs) return fail("null argument");
    if (nj <= 0) return 0;
    long long b = (c->g.M + NTHR - 1) / NTHR;
    if (b > 2048) b = 2048;
    const dim3 grid((unsigned)b, nj);
    if (c->prec == 8) {
        if (model == 0) k_phi<double, 0><<<grid, NTHR, 0, c->stream>>>(jobs, coefs, c->g.M);
        else k_phi<double, 1><<<grid, NTHR, 0, c->stream>>>(jobs, coefs, c->g.M);
    } else {
        if (model == 0) k_phi<float, 0><<<grid, NTHR, 0, c->stream>>>(jobs, coefs, c->g.M);
        else k_phi<float, 1><<<grid, NTHR, 0, c->stream>>>(jobs, coefs, c->g.M);
    }
    c->launches += 1;
    CKLAUNCH();
    return 0;
}

// stress: x-transform of both zy spectra of a job, then the weighted k-sum
template <typename T, bool GEN>
__global__ void __launch_bounds__(NTHR) k_xstress(GridPlan g, const lfts_step_job *__restrict__ sj,
                                                  const lfts_stress_job *__restrict__ jobs, const double *__restrict__ basis,
                                                  int TJ, double *partials) {
    using C = typename CT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sh[2 * NWARP];
    const int n0 = g.n0;
    C *tile = (C *)smem_raw;
    C *twx = tile + 2 * n0 * TJ;
    short *px = (short *)(twx + n0);
    const int job = blockIdx.y;
    const lfts_step_job jb = sj[2 * job];
    const T *bond = (const T *)jobs[job].bond;
    const int tid = threadIdx.x;
    for (int i = tid; i < n0; i += NTHR) { twx[i] = ((const C *)g.tw[0])[i]; px[i] = g.perm[0][i]; }
    __syncthreads();
    const long long plane = (long long)g.n1 * g.nzc;
    const long long j0 = (long long)blockIdx.x * TJ;
    const int tot = 2 * n0 * TJ;
    const C *spec = (const C *)jb.spec;  // two consecutive Mc slots: F_zy[q1], F_zy[q2]
    for (int i = tid; i < tot; i += NTHR) {
        const int jj = i % TJ, x = (i / TJ) % n0, b = i / (TJ * n0);
        C v = cmk<C>(0, 0);
        if (j0 + jj < plane) v = spec[(size_t)b * g.Mc + x * plane + j0 + jj];
        tile[(b * n0 + px[x]) * TJ + jj] = v;
    }
    __syncthreads();
    const LineMap lmx = {2 * TJ, TJ, n0 * TJ, TJ};
    dit_lines<C, true, GEN>(tile, lmx, g.ax[0], twx, -1, tid, NTHR);
    Acc<T> acc[3];
    for (int i = tid; i < n0 * TJ; i += NTHR) {
        const int jj = i % TJ, x = i / TJ;
        if (j0 + jj < plane) {
            const long long k = x * plane + j0 + jj;
            const C A = tile[x * TJ + jj], B = tile[(n0 + x) * TJ + jj];
            double co = (double)A.x * (double)B.x + (double)A.y * (double)B.y;
            if (bond) co *= (double)bond[k] * (double)g.M;  // tables carry 1/M
            acc[0].add(co * basis[k]);
            acc[1].add(co * basis[g.Mc + k]);
            acc[2].add(co * basis[2 * g.Mc + k]);
        }
    }
    for (int d = 0; d < 3; d++) {
        const double v = acc[d].block(sh);
        if (tid == 0) partials[((long long)job * gridDim.x + blockIdx.x) * 3 + d] = v;
    }
}

template <typename T>
__global__ void k_stress_prep(const lfts_stress_job *__restrict__ jobs, int nj, void *spec, long long Mc,
                              lfts_step_job *sj) {
    using C = typename CT<T>::type;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nj; j += gridDim.x * blockDim.x) {
        C *sp = (C *)spec + (size_t)2 * j * Mc;
        lfts_step_job a = {jobs[j].q1, 0, nullptr, 0, nullptr, nullptr, nullptr, sp, nullptr, 0, 0};
        lfts_step_job b = {jobs[j].q2, 0, nullptr, 0, nullptr, nullptr, nullptr, sp + Mc, nullptr, 0, 0};
        sj[2 * j] = a;
        sj[2 * j + 1] = b;
    }
}

template <typename T, bool GEN>
static int stress_t(lfts_ctx c, const lfts_stress_job *jobs, int nj, const double *basis, void *spec, int max_chunk,
                    double *out) {
    const GridPlan &g = c->g;
    cudaStream_t st = c->stream;
    const size_t smx = sizeof(typename CT<T>::type) * (2 * (size_t)g.n0 * c->TJ + g.n0) + sizeof(short) * g.n0;
    for (int j0 = 0; j0 < nj; j0 += max_chunk) {
        const int n = nj - j0 < max_chunk ? nj - j0 : max_chunk;
        if (2 * n > c->sjobs_cap) return fail("stress chunk too large");
        if ((size_t)n * c->ntiles * 3 > c->partials_cap) return fail("stress chunk exceeds the partial-sum workspace");
        k_stress_prep<T><<<(n + 127) / 128, 128, 0, st>>>(jobs + j0, n, spec, g.Mc, c->sjobs);
        k_plane_forward<T, 1, GEN><<<dim3(g.n0, 2 * n), NTHR, c->sm_pf1, st>>>(g, c->sjobs, 0, FM_NONE, 0, 0, c->zb);
        k_xstress<T, GEN><<<dim3(c->ntiles, n), NTHR, smx, st>>>(g, c->sjobs, jobs + j0, basis, c->TJ, c->partials);
        k_finish<T><<<dim3(n, 3), NTHR, 0, st>>>(c->partials, c->ntiles, (const double *)&jobs[j0].weight,
                                                (int)sizeof(lfts_stress_job), 1.0, out + 3 * (long long)j0, 3, 3);
    }
    CKLAUNCH();
    return 0;
}
extern "C" int lfts_stress(lfts_ctx c, const lfts_stress_job *jobs, int nj, const double *basis, void *spec,
                           int max_chunk, double *out) {
    if (!c || !jobs || !basis || !spec || !out) return fail("null argument");
    if (nj <= 0) return 0;
    if (max_chunk <= 0) return fail("max_chunk must be positive");
    if (c->prec == 8) return c->gen ? stress_t<double, true>(c, jobs, nj, basis, spec, max_chunk, out)
                                    : stress_t<double, false>(c, jobs, nj, basis, spec, max_chunk, out);
    return c->gen ? stress_t<float, true>(c, jobs, nj, basis, spec, max_chunk, out)
                  : stress_t<float, false>(c, jobs, nj, basis, spec, max_chunk, out);
}

// ---------------------------------------------------------------- Anderson mixing
__device__ __forceinline__ long long ring_slot(int i, int head, int len) { return (long long)(((head - i) % len + len) % len); }

__global__ void __launch_bounds__(NTHR) k_am_dots(const double *__restrict__ d, const double *__restrict__ hist,
                                                  long long stride, long long n, double *partials, int head, int len) {
    __shared__ double sh[NWARP];
    const double *h = hist + ring_slot(blockIdx.y, head, len) * stride;
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)NTHR + threadIdx.x; i < n; i += (long long)gridDim.x * NTHR) acc += d[i] * h[i];
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) partials[(long long)blockIdx.y * gridDim.x + blockIdx.x] = acc;
}
extern "C" int lfts_am_dots(lfts_ctx c, const double *d, const double *hist, long long stride, int nhist, long long n,
                            double *dots, int head, int ring_len) {
    if (!c || !d || !hist || !dots) return fail("null argument");
    if (nhist <= 0) return 0;
    if (ring_len <= 0 || nhist > ring_len) return fail("invalid history ring");
    if ((size_t)nhist * DOT_CHUNKS > c->partials_cap) return fail("too many history vectors");
    k_am_dots<<<dim3(DOT_CHUNKS, nhist), NTHR, 0, c->stream>>>(d, hist, stride, n, c->partials, head, ring_len);
    k_finish<<<dim3(nhist, 1), NTHR, 0, c->stream>>>(c->partials, DOT_CHUNKS, nullptr, 0, 1.0, dots, 1, 1);
    CKLAUNCH();
    return 0;
}
__global__ void k_am_update(double *__restrict__ wn, const double *__restrict__ wh, const double *__restrict__ dh,
                            long long stride, int nh, const double *__restrict__ a, long long n, int head, int len) {
    const long long s0 = ring_slot(0, head, len) * stride;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double w1 = wh[s0 + i], d1 = dh[s0 + i];
        double acc = w1 + d1;
        for (int h = 0; h < nh; h++) {
            const long long sh = ring_slot(h + 1, head, len) * stride;
            acc += a[h] * (wh[sh + i] + dh[sh + i] - w1 - d1);
        }
        wn[i] = acc;
    }
}
extern "C" int lfts_am_update(lfts_ctx c, double *w_new, const double *w_hist, const double *d_hist, long long stride,
                              int nh, const double *a, long long n, int head, int ring_len) {
    if (!c || !w_new || !w_hist || !d_hist) return fail("null argument");
    if (ring_len <= 0 || nh + 1 > ring_len) return fail("invalid history ring");
    k_am_update<<<grid_for(n), NTHR, 0, c->stream>>>(w_new, w_hist, d_hist, stride, nh, a, n, head, ring_len);
    CKLAUNCH();
    return 0;
}
__global__ void k_am_simple(double *__restrict__ wn, const double *__restrict__ w, const double *__restrict__ d,
                            double mix, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        wn[i] = w[i] + mix * d[i];
}
extern "C" int lfts_am_simple(lfts_ctx c, double *w_new, const double *w, const double *d, double mix, long long n) {
    if (!c || !w_new || !w || !d) return fail("null argument");
    k_am_simple<<<grid_for(n), NTHR, 0, c->stream>>>(w_new, w, d, mix, n);
    CKLAUNCH();
    return 0;
}

// ---------------------------------------------------------------- helpers
constexpr int LINCOMB_MAX = 16;
struct LincombArgs {
    const double *src[LINCOMB_MAX];
    double coef[LINCOMB_MAX];
    int n;
    int accumulate;
};
__global__ void k_lincomb(double *__restrict__ out, LincombArgs a, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double v = a.accumulate ? out[i] : 0.0;
        for (int k = 0; k < a.n; k++) v += a.coef[k] * a.src[k][i];
        out[i] = v;
    }
}
extern "C" int lfts_lincomb(lfts_ctx c, double *out, int nsrc, const double *const *srcs, const double *coefs, long long n) {
    if (!c || !out) return fail("null argument");
    if (nsrc < 0) return fail("negative source count");
    int k0 = 0;
    do {
        LincombArgs a;
        a.n = nsrc - k0 < LINCOMB_MAX ? nsrc - k0 : LINCOMB_MAX;
        a.accumulate = k0 > 0;
        for (int k = 0; k < a.n; k++) { a.src[k] = srcs[k0 + k]; a.coef[k] = coefs ? coefs[k0 + k] : 1.0; }
        k_lincomb<<<grid_for(n), NTHR, 0, c->stream>>>(out, a, n);
        c->launches += 1;
        k0 += a.n;
    } while (k0 < nsrc);
    CKLAUNCH();
    return 0;
}

template <typename T>
__global__ void __launch_bounds__(NTHR) k_pow_sum(const T *__restrict__ fac, int power, long long M, double *partials) {
    __shared__ double sh[2 * NWARP];
    Acc<T> acc;
    for (long long i = blockIdx.x * (long long)NTHR + threadIdx.x; i < M; i += (long long)gridDim.x * NTHR) {
        double f = (double)fac[i], v = f;
        for (int p = 1; p < power; p++) v *= f;
        acc.add(v);
    }
    const double v = acc.block(sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = v;
}
template <typename T>
__global__ void k_solvent_phi(const T *__restrict__ fac, int power, double vf, const double *__restrict__ Q,
                              double *__restrict__ phi, long long M) {
    const double q = *Q;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M; i += (long long)gridDim.x * blockDim.x) {
        double f = (double)fac[i], v = f;
        for (int p = 1; p < power; p++) v *= f;
        phi[i] = vf * v / q;
    }
}
extern "C" int lfts_solvent(lfts_ctx c, const void *fac, int power, double vf, double dv_over_V, double *phi_out,
                            double *Q_out) {
    if (!c || !fac || !phi_out || !Q_out) return fail("null argument");
    if (power < 1) return fail("power must be >= 1");
    const long long M = c->g.M;
    if (c->prec == 8) k_pow_sum<double><<<DOT_CHUNKS, NTHR, 0, c->stream>>>((const double *)fac, power, M, c->partials);
    else k_pow_sum<float><<<DOT_CHUNKS, NTHR, 0, c->stream>>>((const float *)fac, power, M, c->partials);
    if (c->prec == 8) k_finish<double><<<dim3(1, 1), NTHR, 0, c->stream>>>(c->partials, DOT_CHUNKS, nullptr, 0, dv_over_V, Q_out, 1, 1);
    else k_finish<float><<<dim3(1, 1), NTHR, 0, c->stream>>>(c->partials, DOT_CHUNKS, nullptr, 0, dv_over_V, Q_out, 1, 1);
    if (c->prec == 8) k_solvent_phi<double><<<grid_for(M), NTHR, 0, c->stream>>>((const double *)fac, power, vf, Q_out, phi_out, M);
    else k_solvent_phi<float><<<grid_for(M), NTHR, 0, c->stream>>>((const float *)fac, power, vf, Q_out, phi_out, M);
    CKLAUNCH();
    return 0;
}

void lfts_internal_count(lfts_ctx c, int n) {
    if (c) c->launches += n;
}
extern "C" long long lfts_ctx_launches(lfts_ctx c) { return c ? c->launches : 0; }

extern "C" int lfts_field_factors_batch(lfts_ctx c, const double *w, double coef, void *fac_out, int count) {
    if (!c || !w || !fac_out) return fail("null argument");
    const long long n = c->g.M * (long long)count;
    if (c->prec == 8)
        k_field_factors<double><<<grid_for(n), NTHR, 0, c->stream>>>(w, coef, (double *)fac_out, n);
    else
        k_field_factors<float><<<grid_for(n), NTHR, 0, c->stream>>>(w, coef, (float *)fac_out, n);
    c->launches += 1;
    CKLAUNCH();
    return 0;
}

// ---------------------------------------------------------------- Adam field update
// m = b1 m + (1 - b1) d; v = b2 v + (1 - b2) d^2; w_new = w + lr (m / bc1) / (sqrt(v / bc2) + eps)
__global__ void __launch_bounds__(NTHR) k_adam(double *__restrict__ w_new, const double *__restrict__ w,
                                               const double *__restrict__ d, double *__restrict__ m, double *__restrict__ v,
                                               long long n, double lr, double b1, double b2, double eps, double bc1, double bc2) {
    for (long long i = blockIdx.x * (long long)NTHR + threadIdx.x; i < n; i += (long long)gridDim.x * NTHR) {
        const double di = d[i];
        const double mi = b1 * m[i] + (1.0 - b1) * di;
        const double vi = b2 * v[i] + (1.0 - b2) * (di * di);
        m[i] = mi;
        v[i] = vi;
        w_new[i] = w[i] + lr * (mi / bc1) / (sqrt(vi / bc2) + eps);
    }
}

extern "C" int lfts_adam_update(lfts_ctx c, double *w_new, const double *w, const double *d, double *m, double *v,
                                long long n, double lr, double b1, double b2, double eps, int count) {
    if (!c || !w_new || !w || !d || !m || !v) return fail("null argument");
    if (count < 1) return fail("the Adam step count starts at 1");
    const double bc1 = 1.0 - std::pow(b1, (double)count), bc2 = 1.0 - std::pow(b2, (double)count);
    k_adam<<<grid_for(n), NTHR, 0, c->stream>>>(w_new, w, d, m, v, n, lr, b1, b2, eps, bc1, bc2);
    c->launches += 1;
    CKLAUNCH();
    return 0;
}

// ---------------------------------------------------------------- forward FFT and structure function
extern "C" int lfts_fft_forward(lfts_ctx c, const lfts_step_job *jobs, int nj) {
    if (!c || !jobs) return fail("null argument");
    if (c->prec != 8) return fail("lfts_fft_forward needs a double-precision context");
    if (nj <= 0) return 0;
    if (nj > 65535) return fail("too many jobs in one launch (max 65535)");
    const GridPlan &g = c->g;
    const dim3 gp(g.n0, nj), gx(c->ntiles, nj);
    if (c->gen) {
        k_plane_forward<double, 1, true><<<gp, NTHR, c->sm_pf1, c->stream>>>(g, jobs, 0, FM_NONE, 0, 0, c->zb);
        k_xpass_forward<double, true><<<gx, NTHR, c->sm_x1, c->stream>>>(g, jobs, 0, c->TJ);
    } else {
        k_plane_forward<double, 1, false><<<gp, NTHR, c->sm_pf1, c->stream>>>(g, jobs, 0, FM_NONE, 0, 0, c->zb);
        k_xpass_forward<double, false><<<gx, NTHR, c->sm_x1, c->stream>>>(g, jobs, 0, c->TJ);
    }
    c->launches += 2;
    CKLAUNCH();
    return 0;
}

// sf[r][p][k] += mu_a(k) conj(phi_b(k) inv_m),  mu_a = sum_q spec[r][S+q][k] coef[q][a]
__global__ void __launch_bounds__(NTHR) k_sf_accumulate(int R, int S, int I, long long Mc, const double2 *__restrict__ spec,
                                                        const double *__restrict__ coef, double inv_m, int npairs,
                                                        const int *__restrict__ pairs, double2 *__restrict__ sf) {
    const long long n = (long long)R * Mc;
    for (long long idx = blockIdx.x * (long long)NTHR + threadIdx.x; idx < n; idx += (long long)gridDim.x * NTHR) {
        const int r = (int)(idx / Mc);
        const long long k = idx - (long long)r * Mc;
        const double2 *sr = spec + (size_t)r * (S + I) * Mc + k;
        double2 mu[LFTS_MAX_MONOMERS];
#pragma unroll
        for (int a = 0; a < LFTS_MAX_MONOMERS; a++) mu[a] = make_double2(0.0, 0.0);
        for (int q = 0; q < I; q++) {
            const double2 w = sr[(size_t)(S + q) * Mc];
#pragma unroll
            for (int a = 0; a < LFTS_MAX_MONOMERS; a++) {
                if (a < S) {
                    const double cf = coef[q * S + a];
                    mu[a].x += w.x * cf;
                    mu[a].y += w.y * cf;
                }
            }
        }
        double2 *o = sf + (size_t)r * npairs * Mc + k;
        for (int p = 0; p < npairs; p++) {
            const int a = pairs[2 * p], b = pairs[2 * p + 1];
            double2 ph = sr[(size_t)b * Mc];
            ph.x *= inv_m;
            ph.y *= inv_m;
            double2 m = make_double2(0.0, 0.0);
#pragma unroll
            for (int t = 0; t < LFTS_MAX_MONOMERS; t++)
                if (t == a) m = mu[t];
            double2 acc = o[(size_t)p * Mc];
            acc.x += m.x * ph.x + m.y * ph.y;
            acc.y += m.y * ph.x - m.x * ph.y;
            o[(size_t)p * Mc] = acc;
        }
    }
}

extern "C" int lfts_sf_accumulate(lfts_ctx c, int R, int S, int I, const void *spec, const double *coef, double inv_m,
                                  int npairs, const int *pairs, void *sf) {
    if (!c || !spec || !coef || !pairs || !sf) return fail("null argument");
    if (R <= 0 || S <= 0 || I < 0 || npairs <= 0) return fail("R, S and npairs must be positive, I non-negative");
    if (S > LFTS_MAX_MONOMERS) return fail("at most " + std::to_string(LFTS_MAX_MONOMERS) + " monomer types");
    const long long n = (long long)R * c->g.Mc;
    k_sf_accumulate<<<grid_for(n), NTHR, 0, c->stream>>>(R, S, I, c->g.Mc, (const double2 *)spec, coef, inv_m, npairs, pairs,
                                                        (double2 *)sf);
    c->launches += 1;
    CKLAUNCH();
    return 0;
}

// ---------------------------------------------------------------- allocation-free inner products
// The same two kernels as lfts_dots, with their partial sums in a file-scope
// device array instead of context-owned memory.  Every call on a device shares
// the array; k_dots writes all nj * DOT_CHUNKS entries that k_finish reads, so
// no entry has to start at zero.
static __device__ __align__(256) double g_dots_static_scratch[LFTS_DOTS_STATIC_MAX_JOBS * DOT_CHUNKS];
constexpr int DOTS_STATIC_MAX_DEVICES = 64;
static std::mutex g_dots_static_mu;
static double *g_dots_static_ptr[DOTS_STATIC_MAX_DEVICES];

// The current context's unique id (cuCtxGetId, never reused within a
// process), through the driver entry points the runtime exposes, so the
// library needs no link to the driver library.  0 when no context is current.
typedef CUresult (*lfts_pfn_ctx_get_current)(CUcontext *);
typedef CUresult (*lfts_pfn_ctx_get_id)(CUcontext, unsigned long long *);
static int current_context_id(unsigned long long *id) {
    static lfts_pfn_ctx_get_current get_current = nullptr;
    static lfts_pfn_ctx_get_id get_id = nullptr;
    if (!get_current || !get_id) {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        CK(cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa));
        CK(cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb));
        if (!a || !b || qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess)
            return fail("lfts_dots_static: the driver offers no cuCtxGetCurrent / cuCtxGetId");
        get_current = (lfts_pfn_ctx_get_current)a;
        get_id = (lfts_pfn_ctx_get_id)b;
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS) return fail("lfts_dots_static: cuCtxGetCurrent failed");
    *id = 0;
    if (ctx && get_id(ctx, id) != CUDA_SUCCESS) return fail("lfts_dots_static: cuCtxGetId failed");
    return 0;
}

// Address of the scratch array in the current device's context, looked up
// (with that device current) the first time a context is seen and cached with
// the context's id: a new context on the device (after cudaDeviceReset, which
// reloads the module, possibly at another address) gets a new lookup.
static unsigned long long g_dots_static_ctx[DOTS_STATIC_MAX_DEVICES];
static int dots_static_scratch(double **out) {
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= DOTS_STATIC_MAX_DEVICES)
        return fail("lfts_dots_static: device ordinal " + std::to_string(dev) + " out of range");
    std::lock_guard<std::mutex> lock(g_dots_static_mu);
    unsigned long long id = 0;
    if (current_context_id(&id)) return -1;
    if (!g_dots_static_ptr[dev] || id == 0 || id != g_dots_static_ctx[dev]) {
        double *p = nullptr;
        CK(cudaGetSymbolAddress((void **)&p, g_dots_static_scratch));  // makes the primary context current if none is
        if (!p) return fail("lfts_dots_static: cudaGetSymbolAddress returned a null address");
        if (current_context_id(&id)) return -1;
        g_dots_static_ptr[dev] = p;
        g_dots_static_ctx[dev] = id;
    }
    *out = g_dots_static_ptr[dev];
    return 0;
}

extern "C" int lfts_dots_static(int precision, long long M, const lfts_dot_job *jobs, int nj, double *out, void *stream) {
    if (!jobs || !out) return fail("lfts_dots_static: null argument");
    if (precision != 4 && precision != 8) return fail("lfts_dots_static: precision must be 4 or 8");
    if (M <= 0) return fail("lfts_dots_static: M must be positive");
    if (nj < 0 || nj > LFTS_DOTS_STATIC_MAX_JOBS)
        return fail("lfts_dots_static: njobs = " + std::to_string(nj) + " is outside [0, " +
                    std::to_string(LFTS_DOTS_STATIC_MAX_JOBS) + "], the size of the static scratch array");
    if (nj == 0) return 0;
    double *scratch = nullptr;
    if (dots_static_scratch(&scratch)) return -1;
    cudaStream_t st = (cudaStream_t)stream;
    const dim3 grid(DOT_CHUNKS, nj);
    if (precision == 8) {
        k_dots<double><<<grid, NTHR, 0, st>>>(jobs, M, scratch);
        k_finish<double><<<dim3(nj, 1), NTHR, 0, st>>>(scratch, DOT_CHUNKS, (const double *)&jobs[0].scale,
                                                       (int)sizeof(lfts_dot_job), 1.0, out, 1, 1);
    } else {
        k_dots<float><<<grid, NTHR, 0, st>>>(jobs, M, scratch);
        k_finish<float><<<dim3(nj, 1), NTHR, 0, st>>>(scratch, DOT_CHUNKS, (const double *)&jobs[0].scale,
                                                      (int)sizeof(lfts_dot_job), 1.0, out, 1, 1);
    }
    CKLAUNCH();
    return 0;
}

// ---------------------------------------------------------------- autotuner
// Times lfts_step_continuous for every step family the grid supports, and the
// persistent x-pass residency of the register families, on njobs synthetic
// jobs (q = 1, fac = 1, bond tables of a box of edge n), and keeps the fastest.
// The most specialised family (register-resident, then cubic, then generic) is
// the default; another one is taken only when it is more than 5 % faster, so
// the choice (and with it the last bits of the results) is stable.
namespace {
struct TuneCand {
    int fastN, r8, r12, xcap;
    const char *name;
};
}  // namespace

extern "C" int lfts_autotune(lfts_ctx c, int njobs, int reps, char *report, size_t report_cap) {
    if (!c) return fail("null context");
    if (njobs < 1 || njobs > 65535) return fail("autotune: njobs must be 1..65535");
    if (reps < 1) reps = 5;
    const int fastN = c->fastN, r8v = c->r8, r12v = c->r12, xcap0 = c->xcap;
    std::vector<TuneCand> cands;
    if (r8v) {
        cands.push_back({fastN, 1, 0, 0, "register-64"});
        cands.push_back({fastN, 1, 0, 2, "register-64 xcap2"});
    }
    if (r12v) {
        cands.push_back({fastN, 0, 1, 0, "register-96"});
        cands.push_back({fastN, 0, 1, 1, "register-96 xcap1"});
    }
    if (fastN) cands.push_back({fastN, 0, 0, 0, "cubic"});
    cands.push_back({0, 0, 0, 0, "generic"});
    const size_t sb = (size_t)c->prec, M = (size_t)c->g.M, Mc = (size_t)c->g.Mc;
    void *q = nullptr, *fac = nullptr, *bond = nullptr, *spec = nullptr, *w = nullptr;
    lfts_step_job *djobs = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::string rep;
    int best = 0, rc = 0;
    auto cleanup = [&]() {
        if (q) cudaFree(q);
        if (fac) cudaFree(fac);
        if (bond) cudaFree(bond);
        if (spec) cudaFree(spec);
        if (w) cudaFree(w);
        if (djobs) cudaFree(djobs);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    };
    CK(cudaSetDevice(c->device));
    if (cudaMalloc(&q, (size_t)njobs * 2 * M * sb) != cudaSuccess || cudaMalloc(&fac, M * sb) != cudaSuccess ||
        cudaMalloc(&bond, 2 * Mc * sb) != cudaSuccess || cudaMalloc(&spec, (size_t)njobs * 2 * Mc * 2 * sb) != cudaSuccess ||
        cudaMalloc(&w, M * sizeof(double)) != cudaSuccess || cudaMalloc(&djobs, sizeof(lfts_step_job) * njobs) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cleanup();
        return fail("autotune: allocation of the synthetic jobs failed");
    }
    {
        // q = 1 everywhere (bit pattern of 1.0 in the ctx precision), fac = exp(0) = 1
        std::vector<unsigned char> one(sb);
        if (sb == 8) { const double v = 1.0; std::memcpy(one.data(), &v, 8); }
        else { const float v = 1.0f; std::memcpy(one.data(), &v, 4); }
        std::vector<unsigned char> row(M * sb);
        for (size_t i = 0; i < M; i++) std::memcpy(row.data() + i * sb, one.data(), sb);
        for (int jb = 0; jb < njobs; jb++)
            CK(cudaMemcpy((char *)q + (size_t)jb * 2 * M * sb, row.data(), M * sb, cudaMemcpyHostToDevice));
        CK(cudaMemset(w, 0, M * sizeof(double)));
        if ((rc = lfts_field_factors(c, (const double *)w, 0.0, fac)) != 0) { cleanup(); return rc; }
        const double lx[3] = {(double)c->nx[0], (double)c->nx[1], (double)c->nx[2]};
        if ((rc = lfts_bond_tables(c, 1.0, 0.01, lx, bond, (char *)bond + Mc * sb)) != 0) { cleanup(); return rc; }
        std::vector<lfts_step_job> hj(njobs);
        for (int jb = 0; jb < njobs; jb++) {
            lfts_step_job &j = hj[jb];
            std::memset(&j, 0, sizeof j);
            j.in = (char *)q + (size_t)jb * 2 * M * sb;
            j.out = (char *)q + ((size_t)jb * 2 + 1) * M * sb;
            j.fac = fac;
            j.bond = bond;
            j.bond_half = (char *)bond + Mc * sb;
            j.spec = (char *)spec + (size_t)jb * 2 * Mc * 2 * sb;
        }
        CK(cudaMemcpy(djobs, hj.data(), sizeof(lfts_step_job) * njobs, cudaMemcpyHostToDevice));
    }
    std::vector<float> ms(cands.size(), 0.f);
    for (size_t k = 0; k < cands.size() && rc == 0; k++) {
        c->fastN = cands[k].fastN;
        c->r8 = cands[k].r8;
        c->r12 = cands[k].r12;
        c->xcap = cands[k].xcap;
        for (int i = 0; i < 2 && rc == 0; i++) rc = lfts_step_continuous(c, djobs, njobs, 0);
        if (rc) break;
        CK(cudaEventRecord(e0, c->stream));
        for (int i = 0; i < reps && rc == 0; i++) rc = lfts_step_continuous(c, djobs, njobs, 0);
        CK(cudaEventRecord(e1, c->stream));
        CK(cudaEventSynchronize(e1));
        CK(cudaEventElapsedTime(&ms[k], e0, e1));
        ms[k] /= (float)reps;
    }
    if (rc == 0) rc = check_kernel_errors();
    if (rc == 0) {
        for (size_t k = 1; k < cands.size(); k++)
            if (ms[k] < 0.95f * ms[best]) best = (int)k;
        c->fastN = cands[best].fastN;
        c->r8 = cands[best].r8;
        c->r12 = cands[best].r12;
        c->xcap = cands[best].xcap;
        char buf[96];
        for (size_t k = 0; k < cands.size(); k++) {
            std::snprintf(buf, sizeof buf, "%s%s %.4f ms", k ? "; " : "", cands[k].name, (double)ms[k]);
            rep += buf;
        }
        std::snprintf(buf, sizeof buf, " -> %s (%d jobs)", cands[best].name, njobs);
        rep += buf;
    } else {
        c->fastN = fastN;
        c->r8 = r8v;
        c->r12 = r12v;
        c->xcap = xcap0;
    }
    cleanup();
    if (report && report_cap) {
        std::strncpy(report, rep.c_str(), report_cap - 1);
        report[report_cap - 1] = 0;
    }
    return rc;
}

extern "C" int lfts_set_step_impl(lfts_ctx c, const char *name) {
    if (!c || !name) return fail("null argument");
    const std::string n(name);
    const int fastN = c->fast_ok;
    auto set = [&](int f, int r8, int r12) {
        c->fastN = f;
        c->r8 = r8;
        c->r12 = r12;
        c->xcap = 0;
        return 0;
    };
    if (n == "register-64" && c->r8_ok) return set(fastN, 1, 0);
    if (n == "register-96" && c->r12_ok) return set(fastN, 0, 1);
    if (n == "cubic" && fastN) return set(fastN, 0, 0);
    if (n == "generic") return set(0, 0, 0);
    return fail("step implementation \"" + n + "\" is not available for this context");
}

extern "C" int lfts_step_impl(lfts_ctx c, char *name, size_t cap) {
    if (!c || !name || cap == 0) return fail("null argument");
    std::string n = c->r8 ? (c->xcap ? "register-64 xcap" + std::to_string(c->xcap) : std::string("register-64"))
                  : c->r12 ? (c->xcap ? "register-96 xcap" + std::to_string(c->xcap) : std::string("register-96"))
                  : c->fastN ? std::string("cubic") : std::string("generic");
    std::strncpy(name, n.c_str(), cap - 1);
    name[cap - 1] = 0;
    return 0;
}

// ---------------------------------------------------------------- real-space solver
extern "C" long long lfts_realspace_table_size(lfts_ctx c) {
    if (!c) return 0;
    return (long long)rs::ROWS * (c->g.n0 + c->g.n1 + c->g.n2) + 6;
}

// Tridiagonal rows of the Crank-Nicolson step along one axis
// (src/common/FiniteDifference.cpp:20-99), then the pivots of the reference's
// line solves (CpuSolverReal.cpp:480-549) for that matrix, in its order.
static void realspace_axis(double b2, double ds, double dx, int n, int bc_lo, int bc_hi, double *t, double &denom,
                           double &periodic) {
    double *l = t, *d = t + n, *h = t + 2 * n, *p = t + 3 * n, *c = t + 4 * n, *v = t + 5 * n, *rp = t + 6 * n;
    const double xf = b2 * ds / (std::pow(dx, 2) * 6.0);
    for (int i = 0; i < n; i++) {
        l[i] = -0.5 * xf;
        d[i] = 1.0 + xf;
        h[i] = -0.5 * xf;
        c[i] = 0.0;
        v[i] = 0.0;
    }
    if (bc_lo == 1) {  // reflecting
        d[0] += l[0];
        l[0] = 0.0;
    } else if (bc_lo == 2) {  // absorbing
        l[0] = 0.0;
    }
    if (bc_hi == 1) {
        d[n - 1] += h[n - 1];
        h[n - 1] = 0.0;
    } else if (bc_hi == 2) {
        h[n - 1] = 0.0;
    }
    periodic = bc_lo == 0 ? 1.0 : 0.0;
    denom = 1.0;
    if (bc_lo != 0) {
        p[0] = d[0];
        for (int i = 1; i < n; i++) {
            c[i - 1] = h[i - 1] / p[i - 1];
            p[i] = d[i] - l[i] * c[i - 1];
        }
    } else {
        p[0] = d[0] - 1.0;
        v[0] = 1.0 / p[0];
        for (int i = 1; i < n - 1; i++) {
            c[i - 1] = h[i - 1] / p[i - 1];
            p[i] = d[i] - l[i] * c[i - 1];
            v[i] = (-l[i] * v[i - 1]) / p[i];
        }
        c[n - 2] = h[n - 2] / p[n - 2];
        p[n - 1] = d[n - 1] - h[n - 1] * l[0] - l[n - 1] * c[n - 2];
        v[n - 1] = (h[n - 1] - l[n - 1] * v[n - 2]) / p[n - 1];
        for (int i = n - 2; i >= 0; i--) v[i] = v[i] - c[i] * v[i + 1];
        denom = 1.0 + v[0] + l[0] * v[n - 1];
    }
    for (int i = 0; i < n; i++) rp[i] = 1.0 / p[i];
}

extern "C" int lfts_realspace_tables(lfts_ctx c, double b2, double ds, int dim, const double *dx, const int *bc,
                                     double *out) {
    if (!c || !dx || !bc || !out) return fail("null argument");
    if (dim < 1 || dim > 3 || dim != c->dim) return fail("realspace tables: dim must be the context's dimension");
    const int n[3] = {c->g.n0, c->g.n1, c->g.n2};
    const long long tail = (long long)rs::ROWS * (n[0] + n[1] + n[2]);
    for (int d = 0; d < dim; d++) {
        if (bc[2 * d] < 0 || bc[2 * d] > 2 || bc[2 * d + 1] < 0 || bc[2 * d + 1] > 2)
            return fail("realspace tables: boundary codes are 0 (periodic), 1 (reflecting), 2 (absorbing)");
        if ((bc[2 * d] == 0) != (bc[2 * d + 1] == 0))
            return fail("realspace tables: a periodic side needs a periodic opposite side");
        if (n[3 - dim + d] < 2) return fail("realspace tables: every axis of the box needs at least 2 points");
    }
    long long off = 0;
    for (int a = 0; a < 3; a++) {
        const int d = a - (3 - dim);
        if (d < 0) {  // padding axis (extent 1): never solved
            for (int r = 0; r < rs::ROWS; r++) out[off + (long long)r * n[a]] = r == 1 || r == 3 || r == 6 ? 1.0 : 0.0;
            out[tail + a] = 1.0;
            out[tail + 3 + a] = 0.0;
        } else {
            realspace_axis(b2, ds, dx[d], n[a], bc[2 * d], bc[2 * d + 1], out + off, out[tail + a], out[tail + 3 + a]);
        }
        off += (long long)rs::ROWS * n[a];
    }
    return 0;
}

extern "C" int lfts_step_realspace(lfts_ctx c, const lfts_step_job *jobs, int nj, int s, int dim) {
    if (!c || !jobs) return fail("null argument");
    if (c->prec != 8) return fail("the real-space step runs in FP64 contexts only");
    if (dim < 1 || dim > 3 || dim != c->dim) return fail("real-space step: dim must be the context's dimension");
    if (nj <= 0) return 0;
    if (nj > 65535) return fail("real-space step: at most 65535 jobs per call");
    const GridPlan &g = c->g;
    cudaStream_t st = c->stream;
    auto blocks = [&](long long n_axis) { return (unsigned)((g.M / n_axis + NTHR - 1) / NTHR); };
    // the last-axis sweep through a shared-memory tile of ZL lines
    // (a tile of long lines that does not fit shared memory walks the lines in global memory)
    const size_t zsm = sizeof(double) * 2 * rs::ZL * (size_t)(g.n2 + 1);
    const unsigned zblocks = (unsigned)((g.M / g.n2 + rs::ZL - 1) / rs::ZL);
    const bool tiled = zsm <= 200 * 1024;
    if (tiled && zsm > 48 * 1024)
        CK(cudaFuncSetAttribute(rs::k_rs_last_axis<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsm));
    auto last_axis = [&](int src_half) {
        if (tiled) rs::k_rs_last_axis<true><<<dim3(zblocks, nj), rs::ZL, zsm, st>>>(g, jobs, s, src_half);
        else rs::k_rs_next<2, true><<<dim3(blocks(g.n2), nj), NTHR, 0, st>>>(g, jobs, s, src_half);
    };
    if (dim == 3) {
        rs::k_rs_first<3><<<dim3(blocks(g.n0), nj), NTHR, 0, st>>>(g, jobs, s);
        rs::k_rs_next<1, false><<<dim3(blocks(g.n1), nj), NTHR, 0, st>>>(g, jobs, s, 0);
        last_axis(1);
        c->launches += 3;
    } else if (dim == 2) {
        rs::k_rs_first<2><<<dim3(blocks(g.n1), nj), NTHR, 0, st>>>(g, jobs, s);
        last_axis(0);
        c->launches += 2;
    } else {
        rs::k_rs_first<1><<<dim3(blocks(g.n2), nj), NTHR, 0, st>>>(g, jobs, s);
        c->launches += 1;
    }
    CKLAUNCH();
    return 0;
}

// ---------------------------------------------------------------- U-Net convolution (tcgen05)
#include "lfts_unet.cuh"
