// api.cu -- C host layer behind the C ABI (include/mela.h).
//
// Host entry points mirror the reference MEX gateways' semantics (input
// validation order, logical/double reading, MATLAB column-major layout) and
// run every computation on the GPU: host arrays are copied in, packed,
// processed and unpacked by kernels, and copied out.  Device entry points
// are stream-ordered and never synchronise.
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "mela_common.cuh"
#include "mela_internal.h"
#include "mela_host.h"

namespace mela {

// ---------------------------------------------------------------- errors
static thread_local char t_err[512] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_err, sizeof t_err, fmt, ap);
    va_end(ap);
}

mela_status cuda_status(cudaError_t e, const char *what)
{
    set_error("%s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return MELA_ERR_NOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return MELA_ERR_NO_DEVICE;
    return MELA_ERR_CUDA;
}

__device__ u32 g_device_error;

static constexpr int kMaxDevices = 64;
static std::mutex g_dev_mu;
static u32 *g_err_addr[kMaxDevices];
static int g_sms[kMaxDevices];

static int current_device()
{
    int d = 0;
    cudaGetDevice(&d);
    return (d >= 0 && d < kMaxDevices) ? d : 0;
}

u32 *device_error_word()
{
    int d = current_device();
    std::lock_guard<std::mutex> g(g_dev_mu);
    if (!g_err_addr[d]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_device_error) == cudaSuccess) g_err_addr[d] = (u32 *)p;
    }
    return g_err_addr[d];
}

int sm_count()
{
    int d = current_device();
    std::lock_guard<std::mutex> g(g_dev_mu);
    if (!g_sms[d]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
        g_sms[d] = v > 0 ? v : 1;
    }
    return g_sms[d];
}

// ---------------------------------------------------------------- per-thread context
// One non-blocking stream per host thread and device for the host entry
// points; device buffers come from the stream-ordered pool (cached between
// calls, so repeated gateway calls do not pay cudaMalloc).
struct HostCtx {
    cudaStream_t stream[kMaxDevices] = {};
    cudaStream_t copy_in[kMaxDevices] = {};   // pipelined host products: uploads
    cudaStream_t copy_out[kMaxDevices] = {};  //   and downloads
    cudaStream_t side[kMaxDevices] = {};      // work forked off a caller's stream
    cudaStream_t capture[kMaxDevices] = {};   // origin of graph captures
    cudaStream_t aux[kMaxDevices] = {};       // a second fork off a caller's stream
};
static thread_local HostCtx t_ctx;

mela_status host_stream(cudaStream_t *s)
{
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        set_error("no CUDA device visible");
        return MELA_ERR_NO_DEVICE;
    }
    int d = current_device();
    if (!t_ctx.stream[d]) {
        MELA_CUDA_TRY(cudaStreamCreateWithFlags(&t_ctx.stream[d], cudaStreamNonBlocking));
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, d) == cudaSuccess) {
            unsigned long long thr = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    *s = t_ctx.stream[d];
    return MELA_OK;
}

// The calling thread's upload and download streams (created on first use).
static mela_status copy_streams(cudaStream_t *in, cudaStream_t *out)
{
    const int d = current_device();
    if (!t_ctx.copy_in[d]) MELA_CUDA_TRY(cudaStreamCreateWithFlags(&t_ctx.copy_in[d], cudaStreamNonBlocking));
    if (!t_ctx.copy_out[d]) MELA_CUDA_TRY(cudaStreamCreateWithFlags(&t_ctx.copy_out[d], cudaStreamNonBlocking));
    *in = t_ctx.copy_in[d];
    *out = t_ctx.copy_out[d];
    return MELA_OK;
}

mela_status side_stream(cudaStream_t *s)
{
    const int d = current_device();
    if (!t_ctx.side[d]) MELA_CUDA_TRY(cudaStreamCreateWithFlags(&t_ctx.side[d], cudaStreamNonBlocking));
    *s = t_ctx.side[d];
    return MELA_OK;
}

mela_status aux_stream(cudaStream_t *s)
{
    const int d = current_device();
    if (!t_ctx.aux[d]) MELA_CUDA_TRY(cudaStreamCreateWithFlags(&t_ctx.aux[d], cudaStreamNonBlocking));
    *s = t_ctx.aux[d];
    return MELA_OK;
}

mela_status capture_stream(cudaStream_t *s)
{
    const int d = current_device();
    if (!t_ctx.capture[d]) MELA_CUDA_TRY(cudaStreamCreateWithFlags(&t_ctx.capture[d], cudaStreamNonBlocking));
    *s = t_ctx.capture[d];
    return MELA_OK;
}

DevBuf::~DevBuf()
{
    if (p) cudaFreeAsync(p, s);
}

mela_status DevBuf::alloc(size_t bytes, cudaStream_t st)
{
    s = st;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMallocAsync(&p, bytes, st);
    if (e != cudaSuccess) {
        p = nullptr;
        return cuda_status(e, "cudaMallocAsync");
    }
    return MELA_OK;
}

mela_status finish(cudaStream_t s)
{
    MELA_CUDA_TRY(cudaStreamSynchronize(s));
    u32 flags = 0;
    if (mela_device_error_flags(&flags, 1) == MELA_OK && (flags & kErrWaitTimeout)) {
        set_error("a bounded device-side wait timed out");
        return MELA_ERR_TIMEOUT;
    }
    return MELA_OK;
}

// ---------------------------------------------------------------- products
i64 even_words(i64 bits)
{
    i64 w = words_of(bits);
    return (w + 1) & ~1LL;
}

static i64 round_up(i64 x, i64 a) { return (x + a - 1) / a * a; }

// workspace layout for each variant
struct GemmPlan {
    int variant;          // base variant
    int tc_tile;          // tile choice: tensor cores 1 single CTAs / 2 CTA pairs; M4RI 1 = 8 warps
    i64 ldbt;             // packed Bt row pitch (words)
    size_t bt_bytes;      // packed Bt
    i64 mp, np, kp;       // padded byte-operand shape (tensor cores)
    size_t a8_bytes, b8_bytes;
    size_t total;
};

// Workspace layout of a concrete variant argument (AUTO already resolved).
static GemmPlan plan_gemm(int32_t variant, i64 m, i64 k, i64 n)
{
    GemmPlan p{};
    Tuning t{};
    if (!decode_gemm_variant(variant, &t) || t.base == MELA_GEMM_AUTO) t.base = MELA_GEMM_PLAIN;
    p.variant = t.base;
    p.tc_tile = t.tc_tile;
    p.ldbt = even_words(k);
    if (p.variant == MELA_GEMM_PLAIN) p.bt_bytes = (size_t)n * p.ldbt * 8;
    if (p.variant == MELA_GEMM_TC) {
        p.mp = round_up(m, 256);  // 256-row tiles for CTA pairs
        p.np = round_up(n, 256);
        p.kp = round_up(k, 128);  // bytes = values
        p.a8_bytes = (size_t)p.mp * p.kp;
        p.b8_bytes = (size_t)p.np * p.kp;
    }
    if (p.variant == MELA_GEMM_TC_FP4) {
        p.mp = round_up(m, 256);
        p.np = round_up(n, 256);
        p.kp = round_up(k, 256) / 2;  // bytes, two values each
        p.a8_bytes = (size_t)p.mp * p.kp;
        p.b8_bytes = (size_t)p.np * p.kp;
    }
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    p.total = al(p.bt_bytes) + al(p.a8_bytes) + al(p.b8_bytes);
    return p;
}

struct GemmBufs {
    u64 *Bt;
    unsigned char *A8, *B8;
};

static GemmBufs carve(const GemmPlan &p, void *ws)
{
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    unsigned char *w = (unsigned char *)ws;
    GemmBufs b;
    b.Bt = (u64 *)w;
    b.A8 = w + al(p.bt_bytes);
    b.B8 = b.A8 + al(p.a8_bytes);
    return b;
}

static mela_status check_ws(const GemmPlan &p, void *ws, size_t ws_bytes)
{
    if (ws_bytes < p.total || (p.total && !ws)) {
        set_error("mela_dev_matmul: workspace of %zu bytes needed, %zu given", p.total, ws_bytes);
        return MELA_ERR_INVALID;
    }
    return MELA_OK;
}

// Operand preparation: B transposed (plain and tensor-core forms) and the
// 0/1 byte expansion of A and Bt (tensor-core form).
mela_status gemm_prepare(int variant, const u64 *A, i64 lda, const u64 *B, i64 ldb, i64 m, i64 k,
                         i64 n, void *ws, size_t ws_bytes, cudaStream_t s)
{
    if (m == 0 || n == 0 || k == 0) return MELA_OK;
    variant = resolve_gemm_variant(variant, A, lda, m, k, n, s);
    GemmPlan p = plan_gemm(variant, m, k, n);
    mela_status st = check_ws(p, ws, ws_bytes);
    if (st != MELA_OK) return st;
    GemmBufs b = carve(p, ws);
    if (p.variant == MELA_GEMM_TC_FP4 && k >= (1LL << 23)) {
        set_error("fp4 tensor-core product needs k < 2^23 (exact f32 sums)");
        return MELA_ERR_UNSUPPORTED;
    }
    if (p.variant == MELA_GEMM_PLAIN) {
        if ((st = launch_transpose(B, ldb, k, n, b.Bt, p.ldbt, s)) != MELA_OK) return st;
        if (p.ldbt > words_of(k)) {
            // the pad word of each Bt row must read as zero
            MELA_CUDA_TRY(cudaMemset2DAsync(b.Bt + words_of(k), (size_t)p.ldbt * 8, 0, 8, (size_t)n, s));
        }
    }
    if (p.variant == MELA_GEMM_TC) {
        if ((st = launch_expand_u8(A, lda, m, k, p.mp, p.kp, b.A8, s)) != MELA_OK) return st;
        if ((st = launch_expand_t(B, ldb, k, n, p.np, p.kp, b.B8, false, s)) != MELA_OK) return st;
    }
    if (p.variant == MELA_GEMM_TC_FP4) {
        if ((st = launch_expand_f4(A, lda, m, k, p.mp, p.kp, b.A8, s)) != MELA_OK) return st;
        if ((st = launch_expand_t(B, ldb, k, n, p.np, p.kp, b.B8, true, s)) != MELA_OK) return st;
    }
    return MELA_OK;
}

// The product kernel itself on prepared operands.
mela_status gemm_run(int variant, const u64 *A, i64 lda, const u64 *B, i64 ldb, u64 *C, i64 ldc,
                     i64 m, i64 k, i64 n, void *ws, size_t ws_bytes, cudaStream_t s)
{
    if (m == 0 || n == 0) return MELA_OK;
    if (k == 0) {
        MELA_CUDA_TRY(cudaMemset2DAsync(C, (size_t)ldc * 8, 0, (size_t)words_of(n) * 8, (size_t)m, s));
        return MELA_OK;
    }
    variant = resolve_gemm_variant(variant, A, lda, m, k, n, s);
    GemmPlan p = plan_gemm(variant, m, k, n);
    mela_status st = check_ws(p, ws, ws_bytes);
    if (st != MELA_OK) return st;
    GemmBufs b = carve(p, ws);
    switch (p.variant) {
    case MELA_GEMM_PLAIN: return launch_gemm_plain(A, lda, b.Bt, p.ldbt, C, ldc, m, k, n, s);
    case MELA_GEMM_TC: return launch_gemm_tc(b.A8, b.B8, p.mp, p.np, p.kp, C, ldc, m, n, s, false, p.tc_tile);
    case MELA_GEMM_TC_FP4:
        if (k >= (1LL << 23)) {
            set_error("fp4 tensor-core product needs k < 2^23 (exact f32 sums)");
            return MELA_ERR_UNSUPPORTED;
        }
        return launch_gemm_tc(b.A8, b.B8, p.mp, p.np, p.kp, C, ldc, m, n, s, true, p.tc_tile);
    case MELA_GEMM_M4RI: return launch_gemm_m4ri(A, lda, B, ldb, C, ldc, m, k, n, s, p.tc_tile);
    default:
        set_error("unknown product variant %d", p.variant);
        return MELA_ERR_INVALID;
    }
}

mela_status gemm_device(int variant, const u64 *A, i64 lda, const u64 *B, i64 ldb, u64 *C, i64 ldc,
                        i64 m, i64 k, i64 n, void *ws, size_t ws_bytes, cudaStream_t s)
{
    if (m > 0 && n > 0 && k > 0) variant = resolve_gemm_variant(variant, A, lda, m, k, n, s);
    mela_status st = gemm_prepare(variant, A, lda, B, ldb, m, k, n, ws, ws_bytes, s);
    if (st != MELA_OK) return st;
    return gemm_run(variant, A, lda, B, ldb, C, ldc, m, k, n, ws, ws_bytes, s);
}

size_t gemm_workspace(int variant, i64 m, i64 k, i64 n)
{
    if (m <= 0 || n <= 0 || k <= 0) return 0;
    if (MELA_VARIANT_BASE(variant) != MELA_GEMM_AUTO) return plan_gemm(variant, m, k, n).total;
    // AUTO decides on the data: room for any configuration it may pick
    size_t most = plan_gemm(fixed_gemm_variant(m, k, n), m, k, n).total;
    for (int c = 0; c < config_count(MELA_OP_MATMUL); ++c) {
        const size_t t = plan_gemm(config_variant(MELA_OP_MATMUL, c), m, k, n).total;
        if (t > most) most = t;
    }
    return most;
}

// ---------------------------------------------------------------- host-matrix helpers
namespace {
// Host threads that copy a caller's (pageable) array into page-locked
// staging memory in parallel: one copy thread saturates neither the host's
// memory system nor the PCIe link.  Created on first use, never torn down.
class CopyPool {
public:
    static CopyPool &get()
    {
        static CopyPool *p = new CopyPool();
        return *p;
    }
    // dst[0, bytes) = src[0, bytes), split over the pool and the caller.
    void copy(void *dst, const void *src, size_t bytes)
    {
        const int parts = (int)workers_.size() + 1;
        if (bytes < ((size_t)1 << 20) || parts == 1) {
            std::memcpy(dst, src, bytes);
            return;
        }
        std::lock_guard<std::mutex> one_job(call_mu_);  // callers on other threads queue here
        std::unique_lock<std::mutex> lk(mu_);
        job_dst_ = (char *)dst;
        job_src_ = (const char *)src;
        job_bytes_ = bytes;
        job_parts_ = parts;
        pending_ = parts - 1;
        ++gen_;
        lk.unlock();
        cv_.notify_all();
        run_part(0);
        lk.lock();
        done_.wait(lk, [&] { return pending_ == 0; });
    }

private:
    CopyPool()
    {
        unsigned hw = std::thread::hardware_concurrency();
        int n = hw >= 4 ? (int)(hw / 2) : 1;
        if (n > 8) n = 8;
        for (int i = 1; i < n; ++i) workers_.emplace_back([this, i] { loop(i); });
        for (auto &t : workers_) t.detach();
    }
    void run_part(int i)
    {
        const size_t per = (job_bytes_ / job_parts_ + 63) & ~(size_t)63;
        const size_t a = per * (size_t)i, b = a + per < job_bytes_ ? a + per : job_bytes_;
        if (a < b) std::memcpy(job_dst_ + a, job_src_ + a, b - a);
    }
    void loop(int i)
    {
        unsigned long long seen = 0;
        for (;;) {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return gen_ != seen; });
            seen = gen_;
            lk.unlock();
            run_part(i);
            lk.lock();
            if (--pending_ == 0) done_.notify_one();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex call_mu_, mu_;
    std::condition_variable cv_, done_;
    unsigned long long gen_ = 0;
    int pending_ = 0, job_parts_ = 1;
    char *job_dst_ = nullptr;
    const char *job_src_ = nullptr;
    size_t job_bytes_ = 0;
};

// Page-locked staging slots of the calling thread (per device), reused
// across calls: a slot is refilled once the upload that read it has
// completed.
constexpr int kStageSlots = 3;
constexpr size_t kStageBytes = (size_t)8 << 20;
struct Staging {
    void *slot[kStageSlots] = {};
    cudaEvent_t read[kStageSlots] = {};  // the upload from the slot is done
    cudaEvent_t fence = nullptr;         // the device staging buffer is allocated
    bool ready = false;
    bool failed = false;
};
// one set per device: events belong to the device they were created on
thread_local Staging t_stage[kMaxDevices];
thread_local mela_upload_stats t_upload_stats;

double now_us()
{
    return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool staging_ready()
{
    Staging &S = t_stage[current_device()];
    if (S.ready) return true;
    if (S.failed) return false;
    for (int i = 0; i < kStageSlots; ++i) {
        if (cudaHostAlloc(&S.slot[i], kStageBytes, cudaHostAllocPortable) != cudaSuccess ||
            cudaEventCreateWithFlags(&S.read[i], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            S.failed = true;
            return false;
        }
    }
    if (cudaEventCreateWithFlags(&S.fence, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        S.failed = true;
        return false;
    }
    S.ready = true;
    return true;
}
}  // namespace

// Column blocks of the MATLAB array go through the page-locked slots: the
// host copy of block b+1 (parallel memcpy) overlaps the upload of block b on
// the upload stream, and each block is packed on s as soon as it has landed
// (blocks are whole packed words: multiples of 64 columns).
static mela_status upload_and_pack_blocks(const mela_host_matrix *M, u64 *dP, i64 ld, cudaStream_t s,
                                          DevBuf &staging, i64 cols_per_block)
{
    const i64 m = M->rows, n = M->cols;
    const size_t esz = M->kind == MELA_KIND_DOUBLE ? 8 : 1;
    mela_status st = staging.alloc((size_t)m * (size_t)n * esz, s);
    if (st != MELA_OK) return st;
    cudaStream_t sin = nullptr, sout = nullptr;
    if ((st = copy_streams(&sin, &sout)) != MELA_OK) return st;
    Staging &S = t_stage[current_device()];
    // the device staging buffer comes from s's pool: uploads wait for it
    MELA_CUDA_TRY(cudaEventRecord(S.fence, s));
    MELA_CUDA_TRY(cudaStreamWaitEvent(sin, S.fence, 0));
    const char *src = (const char *)M->data;
    char *dst = (char *)staging.p;
    int slot = 0;
    for (i64 j0 = 0; j0 < n; j0 += cols_per_block) {
        const i64 nc = n - j0 < cols_per_block ? n - j0 : cols_per_block;
        const size_t off = (size_t)j0 * (size_t)m * esz, bytes = (size_t)nc * (size_t)m * esz;
        const double t0 = now_us();
        MELA_CUDA_TRY(cudaEventSynchronize(S.read[slot]));  // the slot's previous upload is done
        const double t1 = now_us();
        CopyPool::get().copy(S.slot[slot], src + off, bytes);
        t_upload_stats.slot_wait_us += t1 - t0;
        t_upload_stats.host_copy_us += now_us() - t1;
        t_upload_stats.blocked_bytes += (int64_t)bytes;
        t_upload_stats.blocks += 1;
        MELA_CUDA_TRY(cudaMemcpyAsync(dst + off, S.slot[slot], bytes, cudaMemcpyHostToDevice, sin));
        MELA_CUDA_TRY(cudaEventRecord(S.read[slot], sin));
        MELA_CUDA_TRY(cudaStreamWaitEvent(s, S.read[slot], 0));
        // the last block also writes the row padding words
        const i64 words = j0 + nc >= n ? ld - j0 / 64 : words_of(nc);
        if ((st = launch_pack_words(M->kind, m, nc, dst + off, dP + j0 / 64, ld, words, s)) != MELA_OK)
            return st;
        slot = (slot + 1) % kStageSlots;
    }
    return MELA_OK;
}

mela_status upload_and_pack(const mela_host_matrix *M, u64 *dP, i64 ld, cudaStream_t s,
                            DevBuf &staging)
{
    const i64 m = M->rows, n = M->cols;
    if (m == 0 || n == 0) {
        if (m > 0) MELA_CUDA_TRY(cudaMemsetAsync(dP, 0, (size_t)m * ld * 8, s));
        return MELA_OK;
    }
    const size_t esz = M->kind == MELA_KIND_DOUBLE ? 8 : 1;
    const size_t bytes = (size_t)m * (size_t)n * esz;
    // blocks of whole packed words that fit a staging slot
    const i64 cols_per_block = (i64)(kStageBytes / ((size_t)m * esz)) / 64 * 64;
    if (bytes >= ((size_t)2 << 20) && cols_per_block >= 64 && staging_ready())
        return upload_and_pack_blocks(M, dP, ld, s, staging, cols_per_block);
    mela_status st = staging.alloc(bytes, s);
    if (st != MELA_OK) return st;
    MELA_CUDA_TRY(cudaMemcpyAsync(staging.p, M->data, bytes, cudaMemcpyHostToDevice, s));
    t_upload_stats.direct_bytes += (int64_t)bytes;
    return launch_pack(M->kind, m, n, staging.p, dP, ld, s);
}

}  // namespace mela

// ---------------------------------------------------------------- C ABI
using namespace mela;

extern "C" int mela_version(void) { return 10000; }

extern "C" void mela_upload_stats_get(mela_upload_stats *out, int reset)
{
    if (out) *out = t_upload_stats;
    if (reset) t_upload_stats = mela_upload_stats{};
}

extern "C" const char *mela_status_string(mela_status s)
{
    switch (s) {
    case MELA_OK: return "ok";
    case MELA_ERR_INVALID: return "invalid argument";
    case MELA_ERR_SPARSE: return "sparse input not supported";
    case MELA_ERR_DIM: return "inner dimensions must agree";
    case MELA_ERR_TYPE: return "input must be logical or double";
    case MELA_ERR_NOMEM: return "out of memory";
    case MELA_ERR_CUDA: return "CUDA error";
    case MELA_ERR_TIMEOUT: return "device wait timed out";
    case MELA_ERR_UNSUPPORTED: return "unsupported";
    case MELA_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

extern "C" const char *mela_last_error(void) { return t_err; }

extern "C" mela_status mela_device_error_flags(uint32_t *flags, int clear)
{
    u32 *p = device_error_word();
    if (!p) {
        set_error("device error word unavailable");
        return MELA_ERR_CUDA;
    }
    u32 v = 0;
    MELA_CUDA_TRY(cudaMemcpy(&v, p, 4, cudaMemcpyDeviceToHost));
    if (clear && v) MELA_CUDA_TRY(cudaMemset(p, 0, 4));
    if (flags) *flags = v;
    return MELA_OK;
}

extern "C" size_t mela_matmul_workspace_size(int32_t variant, int64_t m, int64_t k, int64_t n)
{
    Tuning t;
    if (!decode_gemm_variant(variant, &t)) return 0;
    return gemm_workspace(variant, m, k, n);
}

extern "C" mela_status mela_dev_matmul(int32_t variant, const uint64_t *dA, int64_t lda,
                                       const uint64_t *dB, int64_t ldb, uint64_t *dC, int64_t ldc,
                                       int64_t m, int64_t k, int64_t n, void *workspace,
                                       size_t workspace_bytes, void *stream)
{
    Tuning tn;
    if (m < 0 || k < 0 || n < 0 || !decode_gemm_variant(variant, &tn) ||
        lda < words_of(k) || ldb < words_of(n) || ldc < words_of(n)) {
        set_error("mela_dev_matmul: bad shape, leading dimension or variant");
        return MELA_ERR_INVALID;
    }
    if (m > 0 && n > 0 && (!dC || (k > 0 && (!dA || !dB)))) {
        set_error("mela_dev_matmul: null operand");
        return MELA_ERR_INVALID;
    }
    return gemm_device(variant, (const u64 *)dA, lda, (const u64 *)dB, ldb, (u64 *)dC, ldc, m, k,
                       n, workspace, workspace_bytes, (cudaStream_t)stream);
}

static mela_status check_dev_matmul_args(int32_t variant, const uint64_t *dA, int64_t lda,
                                         const uint64_t *dB, int64_t ldb, int64_t ldc, int64_t m,
                                         int64_t k, int64_t n)
{
    Tuning tn;
    if (m < 0 || k < 0 || n < 0 || !decode_gemm_variant(variant, &tn) ||
        lda < words_of(k) || ldb < words_of(n) || ldc < words_of(n)) {
        set_error("bad shape, leading dimension or variant");
        return MELA_ERR_INVALID;
    }
    if (m > 0 && n > 0 && k > 0 && (!dA || !dB)) {
        set_error("null operand");
        return MELA_ERR_INVALID;
    }
    return MELA_OK;
}

extern "C" mela_status mela_dev_matmul_prepare(int32_t variant, const uint64_t *dA, int64_t lda,
                                               const uint64_t *dB, int64_t ldb, int64_t m,
                                               int64_t k, int64_t n, void *workspace,
                                               size_t workspace_bytes, void *stream)
{
    mela_status st = check_dev_matmul_args(variant, dA, lda, dB, ldb, words_of(n), m, k, n);
    if (st != MELA_OK) return st;
    return gemm_prepare(variant, (const u64 *)dA, lda, (const u64 *)dB, ldb, m, k, n, workspace,
                        workspace_bytes, (cudaStream_t)stream);
}

extern "C" mela_status mela_dev_matmul_run(int32_t variant, const uint64_t *dA, int64_t lda,
                                           const uint64_t *dB, int64_t ldb, uint64_t *dC,
                                           int64_t ldc, int64_t m, int64_t k, int64_t n,
                                           void *workspace, size_t workspace_bytes, void *stream)
{
    mela_status st = check_dev_matmul_args(variant, dA, lda, dB, ldb, ldc, m, k, n);
    if (st != MELA_OK) return st;
    if (m > 0 && n > 0 && !dC) {
        set_error("null output");
        return MELA_ERR_INVALID;
    }
    return gemm_run(variant, (const u64 *)dA, lda, (const u64 *)dB, ldb, (u64 *)dC, ldc, m, k, n,
                    workspace, workspace_bytes, (cudaStream_t)stream);
}

// Tensor-core product of host matrices with the transfers overlapped.  A is
// cut into row blocks A_i and B into column blocks B_j (up to 4 x 4); the
// upload stream sends A_0, B_0, A_1, B_1, ...; the compute stream prepares
// each block as it lands (A_i expanded; B_j transposed and expanded) and runs
// the product C_ij = A_i B_j as soon as both of its blocks are in, in the
// order (i, j <= i) after A_i and (i <= j, j) after B_j; the download stream
// sends each C_ij back while the next one is computed.  The first product thus
// starts after two blocks have landed rather than after all of B.  (With
// page-locked host buffers the three streams run concurrently; pageable
// buffers still give the right result, with less overlap.)
static constexpr i64 kPipeMin = 8192;  // pipelined when m and n both reach this

static mela_status matmul_packed_host_pipelined(const uint64_t *A, int64_t lda, const uint64_t *B, int64_t ldb,
                                                uint64_t *C, int64_t ldc, i64 m, i64 k, i64 n, int variant,
                                                cudaStream_t s)
{
    cudaStream_t sin = nullptr, sout = nullptr;
    mela_status st = copy_streams(&sin, &sout);
    if (st != MELA_OK) return st;
    const bool fp4 = MELA_VARIANT_BASE(variant) == MELA_GEMM_TC_FP4;
    if (fp4 && k >= (1LL << 23)) {
        set_error("fp4 tensor-core product needs k < 2^23 (exact f32 sums)");
        return MELA_ERR_UNSUPPORTED;
    }
    const GemmPlan p = plan_gemm(variant, m, k, n);
    const i64 wk = words_of(k), wn = words_of(n);
    // blocks: a multiple of 256 rows (columns), at most 4 per operand
    const i64 mb = round_up((m + 3) / 4, 256), nb = round_up((n + 3) / 4, 256);
    const int bm = (int)((m + mb - 1) / mb), bn = (int)((n + nb - 1) / nb);
    DevBuf dA, dB, dC, ws;
    if ((st = dA.alloc((size_t)m * wk * 8, s)) != MELA_OK) return st;
    if ((st = dB.alloc((size_t)k * wn * 8, s)) != MELA_OK) return st;
    if ((st = dC.alloc((size_t)m * wn * 8, s)) != MELA_OK) return st;
    if ((st = ws.alloc(p.total, s)) != MELA_OK) return st;
    const GemmBufs b = carve(p, ws.p);
    u64 *a = (u64 *)dA.p, *bb = (u64 *)dB.p, *c = (u64 *)dC.p;

    // events: buffers allocated; A_i uploaded; B_j uploaded; C_ij computed; copy streams done
    constexpr int kMaxEv = 1 + 4 + 4 + 16 + 2;
    cudaEvent_t evs[kMaxEv];
    const int nev = 1 + bm + bn + bm * bn + 2;
    int made = 0;
    auto cleanup = [&]() {
        for (int i = 0; i < made; ++i) cudaEventDestroy(evs[i]);
    };
    for (; made < nev; ++made) {
        if (cudaEventCreateWithFlags(&evs[made], cudaEventDisableTiming) != cudaSuccess) {
            cleanup();
            set_error("cudaEventCreate failed");
            return MELA_ERR_CUDA;
        }
    }
    cudaEvent_t ev_alloc = evs[0], ev_done_in = evs[nev - 2], ev_done_out = evs[nev - 1];
    auto ev_a = [&](int i) { return evs[1 + i]; };
    auto ev_b = [&](int j) { return evs[1 + bm + j]; };
    auto ev_c = [&](int i, int j) { return evs[1 + bm + bn + i * bn + j]; };
    auto rows_of = [&](int i) { return (m - i * mb) < mb ? (m - i * mb) : mb; };
    auto cols_of = [&](int j) { return (n - j * nb) < nb ? (n - j * nb) : nb; };

    auto product = [&](int i, int j) -> mela_status {
        const i64 r0 = i * mb, c0 = j * nb, rows = rows_of(i), cols = cols_of(j);
        mela_status e = launch_gemm_tc(b.A8 + (size_t)r0 * p.kp, b.B8 + (size_t)c0 * p.kp, round_up(rows, 256),
                                       round_up(cols, 256), p.kp, c + r0 * wn + c0 / 64, wn, rows, cols, s, fp4,
                                       p.tc_tile);
        if (e != MELA_OK) return e;
        MELA_CUDA_TRY(cudaEventRecord(ev_c(i, j), s));
        MELA_CUDA_TRY(cudaStreamWaitEvent(sout, ev_c(i, j), 0));
        MELA_CUDA_TRY(cudaMemcpy2DAsync(C + r0 * ldc + c0 / 64, (size_t)ldc * 8, c + r0 * wn + c0 / 64,
                                        (size_t)wn * 8, (size_t)words_of(cols) * 8, (size_t)rows,
                                        cudaMemcpyDeviceToHost, sout));
        return MELA_OK;
    };
    auto run = [&]() -> mela_status {
        MELA_CUDA_TRY(cudaEventRecord(ev_alloc, s));
        MELA_CUDA_TRY(cudaStreamWaitEvent(sin, ev_alloc, 0));
        MELA_CUDA_TRY(cudaStreamWaitEvent(sout, ev_alloc, 0));
        for (int r = 0; r < (bm > bn ? bm : bn); ++r) {
            if (r < bm) {
                const i64 r0 = r * mb;
                MELA_CUDA_TRY(cudaMemcpy2DAsync(a + r0 * wk, (size_t)wk * 8, A + r0 * lda, (size_t)lda * 8,
                                                (size_t)wk * 8, (size_t)rows_of(r), cudaMemcpyHostToDevice, sin));
                MELA_CUDA_TRY(cudaEventRecord(ev_a(r), sin));
            }
            if (r < bn) {
                const i64 w0 = r * nb / 64;
                MELA_CUDA_TRY(cudaMemcpy2DAsync(bb + w0, (size_t)wn * 8, B + w0, (size_t)ldb * 8,
                                                (size_t)words_of(cols_of(r)) * 8, (size_t)k,
                                                cudaMemcpyHostToDevice, sin));
                MELA_CUDA_TRY(cudaEventRecord(ev_b(r), sin));
            }
        }
        mela_status e;
        for (int r = 0; r < (bm > bn ? bm : bn); ++r) {
            if (r < bm) {
                const i64 r0 = r * mb, rows = rows_of(r);
                MELA_CUDA_TRY(cudaStreamWaitEvent(s, ev_a(r), 0));
                e = fp4 ? launch_expand_f4(a + r0 * wk, wk, rows, k, round_up(rows, 256), p.kp,
                                           b.A8 + (size_t)r0 * p.kp, s)
                        : launch_expand_u8(a + r0 * wk, wk, rows, k, round_up(rows, 256), p.kp,
                                           b.A8 + (size_t)r0 * p.kp, s);
                if (e != MELA_OK) return e;
                for (int j = 0; j < r && j < bn; ++j)
                    if ((e = product(r, j)) != MELA_OK) return e;
            }
            if (r < bn) {
                const i64 c0 = r * nb, cols = cols_of(r);
                MELA_CUDA_TRY(cudaStreamWaitEvent(s, ev_b(r), 0));
                e = launch_expand_t(bb + c0 / 64, wn, k, cols, round_up(cols, 256), p.kp, b.B8 + (size_t)c0 * p.kp,
                                    fp4, s);
                if (e != MELA_OK) return e;
                for (int i = 0; i <= r && i < bm; ++i)
                    if ((e = product(i, r)) != MELA_OK) return e;
            }
        }
        return MELA_OK;
    };
    st = run();
    // the buffers are released on s: it waits for both copy streams first
    if (cudaEventRecord(ev_done_in, sin) == cudaSuccess) cudaStreamWaitEvent(s, ev_done_in, 0);
    if (cudaEventRecord(ev_done_out, sout) == cudaSuccess) cudaStreamWaitEvent(s, ev_done_out, 0);
    const mela_status fin = finish(s);
    cleanup();
    return st != MELA_OK ? st : fin;
}

extern "C" mela_status mela_matmul_packed_host(const uint64_t *A, int64_t lda, const uint64_t *B,
                                               int64_t ldb, uint64_t *C, int64_t ldc, int64_t m,
                                               int64_t k, int64_t n, int32_t variant)
{
    Tuning tn;
    if (m < 0 || k < 0 || n < 0 || lda < words_of(k) || ldb < words_of(n) || ldc < words_of(n) ||
        !decode_gemm_variant(variant, &tn)) {
        set_error("mela_matmul_packed_host: bad shape or variant");
        return MELA_ERR_INVALID;
    }
    if (m == 0 || n == 0) return MELA_OK;
    cudaStream_t s;
    mela_status st = host_stream(&s);
    if (st != MELA_OK) return st;
    {
        // The transfers are pipelined for an explicit tensor-core variant, and
        // for AUTO under the fixed rule; AUTO with a cost model installed
        // uploads first, since the model's choice depends on the data.
        int32_t v = variant;
        if (tn.base == MELA_GEMM_AUTO && !costmodel_loaded()) v = fixed_gemm_variant(m, k, n);
        const int b = MELA_VARIANT_BASE(v);
        if ((b == MELA_GEMM_TC || b == MELA_GEMM_TC_FP4) && k > 0 && m >= kPipeMin && n >= kPipeMin)
            return matmul_packed_host_pipelined(A, lda, B, ldb, C, ldc, m, k, n, v, s);
    }
    const i64 wk = words_of(k), wn = words_of(n);
    DevBuf dA, dB, dC, ws;
    if ((st = dA.alloc((size_t)m * (wk ? wk : 1) * 8, s)) != MELA_OK) return st;
    if ((st = dB.alloc((size_t)(k ? k : 1) * wn * 8, s)) != MELA_OK) return st;
    if ((st = dC.alloc((size_t)m * wn * 8, s)) != MELA_OK) return st;
    size_t wsb = gemm_workspace(variant, m, k, n);
    if ((st = ws.alloc(wsb, s)) != MELA_OK) return st;
    if (k > 0) {
        MELA_CUDA_TRY(cudaMemcpy2DAsync(dA.p, (size_t)wk * 8, A, (size_t)lda * 8, (size_t)wk * 8,
                                        (size_t)m, cudaMemcpyHostToDevice, s));
        MELA_CUDA_TRY(cudaMemcpy2DAsync(dB.p, (size_t)wn * 8, B, (size_t)ldb * 8, (size_t)wn * 8,
                                        (size_t)k, cudaMemcpyHostToDevice, s));
    }
    st = gemm_device(variant, (const u64 *)dA.p, wk, (const u64 *)dB.p, wn, (u64 *)dC.p, wn, m, k, n,
                     ws.p, wsb, s);
    if (st != MELA_OK) return st;
    MELA_CUDA_TRY(cudaMemcpy2DAsync(C, (size_t)ldc * 8, dC.p, (size_t)wn * 8, (size_t)wn * 8,
                                    (size_t)m, cudaMemcpyDeviceToHost, s));
    return finish(s);
}

// Shared body of the two product gateways (reference validation order:
// src/mela_matmul_gf2.c:75-88).
static mela_status matmul_host(const mela_host_matrix *A, const mela_host_matrix *B, uint8_t *C,
                               int variant)
{
    if (!A || !B) {
        set_error("null argument");
        return MELA_ERR_INVALID;
    }
    if (A->sparse || B->sparse) return MELA_ERR_SPARSE;
    if (A->cols != B->rows) return MELA_ERR_DIM;
    auto ok_kind = [](int k) { return k == MELA_KIND_LOGICAL || k == MELA_KIND_DOUBLE; };
    if (!ok_kind(A->kind) || !ok_kind(B->kind)) return MELA_ERR_TYPE;
    const i64 m = A->rows, k = A->cols, n = B->cols;
    if (m < 0 || k < 0 || n < 0) return MELA_ERR_INVALID;
    if (m == 0 || n == 0) return MELA_OK;
    if (!C || (k > 0 && (!A->data || !B->data))) {
        set_error("null data pointer");
        return MELA_ERR_INVALID;
    }
    cudaStream_t s;
    mela_status st = host_stream(&s);
    if (st != MELA_OK) return st;
    const i64 lda = even_words(k), ldb = even_words(n), ldc = even_words(n);
    DevBuf pA, pB, pC, sA, sB, ws, outb;
    if ((st = pA.alloc((size_t)m * lda * 8, s)) != MELA_OK) return st;
    if ((st = pB.alloc((size_t)(k ? k : 1) * ldb * 8, s)) != MELA_OK) return st;
    if ((st = pC.alloc((size_t)m * ldc * 8, s)) != MELA_OK) return st;
    if ((st = upload_and_pack(A, (u64 *)pA.p, lda, s, sA)) != MELA_OK) return st;
    if ((st = upload_and_pack(B, (u64 *)pB.p, ldb, s, sB)) != MELA_OK) return st;
    size_t wsb = gemm_workspace(variant, m, k, n);
    if ((st = ws.alloc(wsb, s)) != MELA_OK) return st;
    st = gemm_device(variant, (const u64 *)pA.p, lda, (const u64 *)pB.p, ldb, (u64 *)pC.p, ldc, m,
                     k, n, ws.p, wsb, s);
    if (st != MELA_OK) return st;
    if ((st = outb.alloc((size_t)m * n, s)) != MELA_OK) return st;
    if ((st = launch_unpack((const u64 *)pC.p, ldc, m, n, (unsigned char *)outb.p, s)) != MELA_OK)
        return st;
    MELA_CUDA_TRY(cudaMemcpyAsync(C, outb.p, (size_t)m * n, cudaMemcpyDeviceToHost, s));
    return finish(s);
}

extern "C" mela_status mela_matmul_gf2(const mela_host_matrix *A, const mela_host_matrix *B,
                                       uint8_t *C)
{
    return matmul_host(A, B, C, MELA_GEMM_AUTO);
}

extern "C" mela_status mela_matmul_m4ri(const mela_host_matrix *A, const mela_host_matrix *B,
                                        uint8_t *C)
{
    return matmul_host(A, B, C, MELA_GEMM_M4RI);
}
