// noalloc.cu -- a GF(2) product entry point that allocates no device memory.
//
// Who needs it: code that is handed device buffers but may not allocate any
// itself -- for example a plugin inside a host application that owns the
// GPU's memory through its own allocator and has fixed the budget up front,
// or a latency-critical loop that cannot afford cudaMalloc's implicit device
// synchronisation.  mela_dev_matmul asks such callers for a workspace they
// cannot provide; this entry point needs none.
//
// How: the plain AND+popcount product needs one scratch buffer, the
// transposed right operand (n rows of ceil(k/64) words, rounded up to an even
// count).  Here that buffer is a file-scope __device__ array of fixed size,
// kMaxScratchBytes (16 MiB), which every GPU that loads the library holds
// until the process exits.  Larger products are rejected with
// MELA_ERR_UNSUPPORTED before any device work.
//
// Host code cannot use the array's name as a device address (on the host it
// names a host-side shadow), so the first call on each device looks the
// address up with cudaGetSymbolAddress, with that device current, and caches
// it.  That first call should therefore come before any stream capture.  The
// cache is keyed on the device's current CUDA context: after a device reset
// (a new primary context, where the module may load at another address) the
// next call looks the address up again.
//
// All calls share the one array and it keeps whatever the last call left in
// it.  Nothing in it needs to start at zero: the transpose kernel writes
// every word the product kernel later reads.  Calls whose work overlaps on
// the GPU (different streams, or different host threads, on the same device)
// race on the array; serialise them.
#include <mutex>

#include <cuda.h>

#include "mela_common.cuh"
#include "mela_internal.h"
#include "mela_host.h"

namespace mela {

static constexpr size_t kMaxScratchBytes = (size_t)16 << 20;

static __device__ __align__(256) unsigned char g_static_scratch[kMaxScratchBytes];

namespace {
constexpr int kMaxDev = 64;
std::mutex g_mu;
void *g_scratch_addr[kMaxDev];
unsigned long long g_scratch_ctx[kMaxDev];  // id of the context the address belongs to

// Unique id of the calling thread's current context (0 when there is none).
// The driver functions are looked up through the runtime, so the library
// loads on machines without the driver.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);
unsigned long long current_context_id()
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        void *p = nullptr, *q = nullptr;
        cudaDriverEntryPointQueryResult r1, r2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &r1) != cudaSuccess ||
            r1 != cudaDriverEntryPointSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &q, cudaEnableDefault, &r2) != cudaSuccess ||
            r2 != cudaDriverEntryPointSuccess)
            return 0;
        get_current = (CtxGetCurrentFn)p;
        get_id = (CtxGetIdFn)q;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}
}  // namespace

// Device address of g_static_scratch on the current device, looked up once
// per device and context.
static mela_status static_scratch(void **out)
{
    int d = 0;
    MELA_CUDA_TRY(cudaGetDevice(&d));
    if (d < 0 || d >= kMaxDev) {
        set_error("device ordinal %d beyond the library's limit", d);
        return MELA_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> g(g_mu);
    const unsigned long long ctx = current_context_id();
    if (!g_scratch_addr[d] || ctx == 0 || ctx != g_scratch_ctx[d]) {
        // the lookup also makes the device's primary context current
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p) return cuda_status(e, "cudaGetSymbolAddress(g_static_scratch)");
        g_scratch_addr[d] = p;
        g_scratch_ctx[d] = current_context_id();
    }
    *out = g_scratch_addr[d];
    return MELA_OK;
}

}  // namespace mela

using namespace mela;

extern "C" size_t mela_static_scratch_bytes(void) { return kMaxScratchBytes; }

extern "C" mela_status mela_dev_matmul_plain_static(const uint64_t *dA, int64_t lda,
                                                    const uint64_t *dB, int64_t ldb, uint64_t *dC,
                                                    int64_t ldc, int64_t m, int64_t k, int64_t n,
                                                    void *stream)
{
    if (m < 0 || k < 0 || n < 0 || lda < words_of(k) || ldb < words_of(n) || ldc < words_of(n)) {
        set_error("mela_dev_matmul_plain_static: bad shape or leading dimension");
        return MELA_ERR_INVALID;
    }
    if (m == 0 || n == 0) return MELA_OK;
    if (!dC || (k > 0 && (!dA || !dB))) {
        set_error("mela_dev_matmul_plain_static: null operand");
        return MELA_ERR_INVALID;
    }
    const i64 ldbt = even_words(k);
    const double need = (double)n * (double)ldbt * 8.0;
    if (need > (double)kMaxScratchBytes) {
        set_error("mela_dev_matmul_plain_static: transposed operand needs %.0f bytes, the static "
                  "scratch holds %zu (n * ceil(k/64 rounded to even) * 8 must fit)",
                  need, kMaxScratchBytes);
        return MELA_ERR_UNSUPPORTED;
    }
    // launch shapes of the transpose (k / 256 row blocks) and of the product
    // (m / 128 row tiles) are checked before any device work
    if (mela_status st = check_grid_yz((k + 255) / 256, (m + 127) / 128, "mela_dev_matmul_plain_static");
        st != MELA_OK)
        return st;
    cudaStream_t s = (cudaStream_t)stream;
    if (k == 0) {
        MELA_CUDA_TRY(cudaMemset2DAsync(dC, (size_t)ldc * 8, 0, (size_t)words_of(n) * 8, (size_t)m, s));
        return MELA_OK;
    }
    void *scratch = nullptr;
    mela_status st = static_scratch(&scratch);
    if (st != MELA_OK) return st;
    u64 *Bt = (u64 *)scratch;
    if ((st = launch_transpose((const u64 *)dB, ldb, k, n, Bt, ldbt, s)) != MELA_OK) return st;
    return launch_gemm_plain((const u64 *)dA, lda, Bt, ldbt, (u64 *)dC, ldc, m, k, n, s);
}
