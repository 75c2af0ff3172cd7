// dispatch.cu -- how each request is computed: variant arguments with their
// tuning fields, the configurations the cost model prices, the density it is
// fed, and the fixed rule it is compared against.
//
// A variant argument is a base variant (bits 0-7) with optional tuning
// fields (MELA_TUNE_K, MELA_TUNE_TILE in include/mela.h).  The AUTO
// variants ask the installed cost model for a configuration -- measuring
// the input's density on the device first -- or, without a model, apply
// the fixed rule.  Nothing here changes a result.
#include <cmath>

#include "mela_common.cuh"
#include "mela_internal.h"
#include "mela_host.h"

namespace mela {

// ---------------------------------------------------------------- variant arguments
bool decode_elim_variant(int32_t v, Tuning *t)
{
    if (v & ~0xffff) return false;
    const int base = v & 0xff, k = (v >> 8) & 0xf, tile = (v >> 12) & 0xf;
    if (base < MELA_ELIM_AUTO || base > MELA_ELIM_TC) return false;
    Tuning r{};
    r.base = base;
    r.k = 0;
    r.row_tile = 1024;
    r.tc_tile = 0;
    if (base == MELA_ELIM_M4RI || base == MELA_ELIM_M4RI_K4) {
        const int dflt = base == MELA_ELIM_M4RI ? 8 : 4;
        r.k = k ? k : dflt;
        if (base == MELA_ELIM_M4RI_K4 && r.k != 4) return false;
        if (r.k != 4 && (r.k < 6 || r.k > 10)) return false;
        static const int tiles[4] = {1024, 256, 1024, 4096};
        if (tile > 3) return false;
        r.row_tile = tiles[tile];
    } else if (k || tile) {
        return false;
    }
    *t = r;
    return true;
}

bool decode_gemm_variant(int32_t v, Tuning *t)
{
    if (v & ~0xffff) return false;
    const int base = v & 0xff, k = (v >> 8) & 0xf, tile = (v >> 12) & 0xf;
    if (base < MELA_GEMM_AUTO || base > MELA_GEMM_TC_FP4) return false;
    Tuning r{};
    r.base = base;
    r.row_tile = 0;
    r.k = 0;
    r.tc_tile = 0;
    if (base == MELA_GEMM_M4RI) {
        if (k && k != 8) return false;
        r.k = 8;
        if (tile > 2) return false;
        r.tc_tile = tile;  // 1: 8 warps of 64 rows; 0 / 2: 16 warps of 32 rows
    } else if (base == MELA_GEMM_TC || base == MELA_GEMM_TC_FP4) {
        if (k || tile > 2) return false;
        r.tc_tile = tile;
    } else if (k || tile) {
        return false;
    }
    *t = r;
    return true;
}

// ---------------------------------------------------------------- configurations
// Model output order per op.  Elimination: the plain form, the blocked form
// over M4RI k = 4, 6, 7, 8 (with 1024-row update tiles), k = 8 with 256-row
// tiles (more CTAs for short matrices), k = 9 and 10 with 4096-row tiles
// (their larger tables pay off over more rows), the single-CTA form and the
// tensor-core windows.  Products: plain, Four-Russians (16 warps of 32 rows
// or 8 of 64), and each tensor-core form on CTA pairs and on single CTAs.  Batches: the engine per matrix.
static const int32_t kElimConfigs[] = {
    MELA_ELIM_PLAIN,
    MELA_ELIM_M4RI_K4,
    MELA_ELIM_M4RI | MELA_TUNE_K(6),
    MELA_ELIM_M4RI | MELA_TUNE_K(7),
    MELA_ELIM_M4RI | MELA_TUNE_K(8),
    MELA_ELIM_M4RI | MELA_TUNE_K(8) | MELA_TUNE_TILE(1),
    MELA_ELIM_M4RI | MELA_TUNE_K(9) | MELA_TUNE_TILE(3),
    MELA_ELIM_M4RI | MELA_TUNE_K(10) | MELA_TUNE_TILE(3),
    MELA_ELIM_FUSED,
    MELA_ELIM_TC,
};
static const int32_t kGemmConfigs[] = {
    MELA_GEMM_PLAIN,
    MELA_GEMM_M4RI,
    MELA_GEMM_M4RI | MELA_TUNE_TILE(1),
    MELA_GEMM_TC | MELA_TUNE_TILE(2),
    MELA_GEMM_TC | MELA_TUNE_TILE(1),
    MELA_GEMM_TC_FP4 | MELA_TUNE_TILE(2),
    MELA_GEMM_TC_FP4 | MELA_TUNE_TILE(1),
};
static const int32_t kBatchConfigs[] = {0, 1, 2};
static_assert(sizeof kElimConfigs / sizeof kElimConfigs[0] <= MELA_MLP_OUT, "model outputs");
static_assert(sizeof kGemmConfigs / sizeof kGemmConfigs[0] <= MELA_MLP_OUT, "model outputs");

int config_count(int op)
{
    switch (op) {
    case MELA_OP_RANK:
    case MELA_OP_NULL: return (int)(sizeof kElimConfigs / sizeof kElimConfigs[0]);
    case MELA_OP_MATMUL: return (int)(sizeof kGemmConfigs / sizeof kGemmConfigs[0]);
    case MELA_OP_BATCH: return (int)(sizeof kBatchConfigs / sizeof kBatchConfigs[0]);
    default: return 0;
    }
}

int32_t config_variant(int op, int index)
{
    if (index < 0 || index >= config_count(op)) return -1;
    switch (op) {
    case MELA_OP_RANK:
    case MELA_OP_NULL: return kElimConfigs[index];
    case MELA_OP_MATMUL: return kGemmConfigs[index];
    default: return kBatchConfigs[index];
    }
}

// ---------------------------------------------------------------- density
namespace {
__global__ void popcount_kernel(const u64 *__restrict__ M, i64 ld, i64 m, i64 wc, u64 last_mask,
                                unsigned long long *count)
{
    unsigned long long c = 0;
    const i64 total = m * wc;
    for (i64 e = blockIdx.x * (i64)blockDim.x + threadIdx.x; e < total; e += (i64)gridDim.x * blockDim.x) {
        const i64 i = e / wc, w = e - i * wc;
        u64 v = M[i * ld + w];
        if (w == wc - 1) v &= last_mask;
        c += __popcll(v);
    }
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ unsigned long long part[8];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += part[q];
        atomicAdd(count, t);
    }
}
}  // namespace

mela_status launch_popcount(const u64 *M, i64 ld, i64 m, i64 n, long long *d_count, cudaStream_t s)
{
    MELA_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(long long), s));
    if (m <= 0 || n <= 0) return MELA_OK;
    const i64 wc = words_of(n);
    const u64 last_mask = (n & 63) ? ((1ull << (n & 63)) - 1) : ~0ull;
    i64 blocks = (m * wc + 255) / 256;
    const i64 cap = (i64)sm_count() * 8;
    if (blocks > cap) blocks = cap;
    popcount_kernel<<<(unsigned)blocks, 256, 0, s>>>(M, ld, m, wc, last_mask, (unsigned long long *)d_count);
    MELA_LAUNCH_CHECK("popcount_kernel");
    return MELA_OK;
}

// The calling thread's counter for density read-backs: one device word and
// one page-locked host word per device, allocated on first use.
namespace {
struct DensitySlot {
    long long *d = nullptr;
    long long *h = nullptr;
    bool failed = false;
};
thread_local DensitySlot t_density[64];
}  // namespace

double measure_density(const u64 *M, i64 ld, i64 m, i64 n, cudaStream_t s)
{
    if (m <= 0 || n <= 0 || !M) return 0.5;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return 0.5;  // no read-back while a graph is being captured
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0.5;
    DensitySlot &S = t_density[dev];
    if (!S.d && !S.failed) {
        if (cudaMalloc((void **)&S.d, sizeof(long long)) != cudaSuccess ||
            cudaMallocHost((void **)&S.h, sizeof(long long)) != cudaSuccess) {
            cudaGetLastError();
            S.failed = true;
        }
    }
    if (S.failed) return 0.5;
    if (launch_popcount(M, ld, m, n, S.d, s) != MELA_OK ||
        cudaMemcpyAsync(S.h, S.d, sizeof(long long), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return 0.5;
    }
    return (double)*S.h / ((double)m * (double)n);
}

// The calling thread's last AUTO resolution (mela_dispatch_last).
namespace {
thread_local int32_t t_last_variant = -1;
thread_local double t_last_density = -1.0;
}  // namespace

static int32_t remember(int32_t v, double density)
{
    t_last_variant = v;
    t_last_density = density;
    return v;
}

// The model's choice for a request whose density is not known yet.  The
// model is evaluated at densities spanning its range first.  The density is
// measured on the device (a popcount and a read-back that waits for the
// stream, about 15 us) only when that can pay: when no single configuration
// is predicted within kMeasureCostUs of the best at every probed density.
// Otherwise that configuration (the one whose worst predicted loss is
// smallest) is taken as it is.
constexpr double kMeasureCostUs = 15.0;

// Without the density: the configuration whose worst predicted loss over
// the probed densities is smallest (index), and whether that loss exceeds
// what measuring costs.  -1 without a model.
static int choose_unmeasured(int op, double m, double n, double p, double cells, bool *measure)
{
    static const double probe[kCostProbes] = {0.001, 0.01, 0.1, 0.5};
    const double lc = std::log2(cells > 1 ? cells : 1);
    const int nc = config_count(op);
    float y[kCostProbes][MELA_MLP_OUT];
    double best[kCostProbes];
    if (nc <= 0 || !costmodel_predict_densities(op, m, n, p, probe, 1, lc, y)) return -1;
    for (int d = 0; d < kCostProbes; ++d) {
        best[d] = 1e300;
        for (int c = 0; c < nc; ++c) best[d] = std::fmin(best[d], std::exp2((double)y[d][c]));
    }
    int pick = 0;
    double pick_loss = 1e300;
    for (int c = 0; c < nc; ++c) {
        double loss = 0;
        for (int d = 0; d < kCostProbes; ++d) loss = std::fmax(loss, std::exp2((double)y[d][c]) - best[d]);
        if (loss < pick_loss) {
            pick_loss = loss;
            pick = c;
        }
    }
    *measure = pick_loss > kMeasureCostUs;
    return pick;
}

// The calling thread's recent pre-data decisions, by (op, shape) and model
// generation: repeated shapes skip the model evaluation.
namespace {
struct PlanEntry {
    unsigned gen;
    int op, pick;
    bool measure;
    double m, n, p;
};
constexpr int kPlanCache = 256;
thread_local PlanEntry t_plans[kPlanCache];
}  // namespace

static int choose_unmeasured_cached(int op, double m, double n, double p, double cells, bool *measure)
{
    const unsigned gen = costmodel_generation();
    const unsigned long long h = ((unsigned long long)op * 0x9E3779B97F4A7C15ull) ^
                                 ((unsigned long long)m * 0xBF58476D1CE4E5B9ull) ^
                                 ((unsigned long long)n * 0x94D049BB133111EBull) ^ (unsigned long long)p;
    PlanEntry &e = t_plans[(h ^ (h >> 29)) % kPlanCache];
    if (e.gen == gen && e.op == op && e.m == m && e.n == n && e.p == p) {
        *measure = e.measure;
        return e.pick;
    }
    const int pick = choose_unmeasured(op, m, n, p, cells, measure);
    if (pick >= 0) e = PlanEntry{gen, op, pick, *measure, m, n, p};
    return pick;
}

static int choose_measuring(int op, double m, double n, double p, double cells,
                            const u64 *M, i64 ld, i64 rows, i64 cols, cudaStream_t s)
{
    bool measure = false;
    const int pick = choose_unmeasured_cached(op, m, n, p, cells, &measure);
    t_last_density = -1.0;
    if (pick < 0 || !measure) return pick;
    const double d = measure_density(M, ld, rows, cols, s);
    t_last_density = d;
    return costmodel_choose(op, m, n, p, d, 1, std::log2(cells > 1 ? cells : 1));
}

// ---------------------------------------------------------------- choices
int32_t resolve_gemm_variant(int32_t variant, const u64 *A, i64 lda, i64 m, i64 k, i64 n, cudaStream_t s)
{
    if (MELA_VARIANT_BASE(variant) != MELA_GEMM_AUTO) return variant;
    if (costmodel_loaded() && m > 0 && n > 0 && k > 0) {
        const int c = choose_measuring(MELA_OP_MATMUL, (double)m, (double)k, (double)n, (double)m * (double)k,
                                       A, lda, m, k, s);
        if (c >= 0) {
            int32_t v = config_variant(MELA_OP_MATMUL, c);
            // the FP4 form's f32 sums are exact below 2^24: past 2^23 terms use INT8
            if (MELA_VARIANT_BASE(v) == MELA_GEMM_TC_FP4 && k >= (1LL << 23))
                v = MELA_GEMM_TC | (v & ~0xff);
            return remember(v, t_last_density);
        }
    }
    return remember(fixed_gemm_variant(m, k, n), -1.0);
}

int32_t fixed_gemm_variant(i64 m, i64 k, i64 n)
{
    // tensor cores pay off once every dimension spans a few tiles (below
    // that the expansion of the operands dominates); the FP4 form runs at
    // twice the INT8 rate while its f32 sums stay exact
    if (m >= 1024 && n >= 1024 && k >= 1024) return k < (1LL << 23) ? MELA_GEMM_TC_FP4 : MELA_GEMM_TC;
    return MELA_GEMM_PLAIN;
}

int32_t resolve_elim_variant(int32_t variant, const u64 *M, i64 ld, i64 m, i64 n, int rref, cudaStream_t s)
{
    if (MELA_VARIANT_BASE(variant) != MELA_ELIM_AUTO) return variant;
    if (costmodel_loaded() && m > 0 && n > 0) {
        const int c = choose_measuring(rref ? MELA_OP_NULL : MELA_OP_RANK, (double)m, (double)n, 0.0,
                                       (double)m * (double)n, M, ld, m, n, s);
        if (c >= 0) return remember(config_variant(MELA_OP_RANK, c), t_last_density);
    }
    return remember(fixed_elim_variant(m, n), -1.0);
}

int32_t fixed_elim_variant(i64 m, i64 n)
{
    // one CTA for small matrices, tensor-core windows otherwise
    return (double)m * (double)n < 8192.0 ? MELA_ELIM_FUSED : MELA_ELIM_TC;
}

}  // namespace mela

using namespace mela;

extern "C" int32_t mela_costmodel_config_count(int32_t op) { return config_count(op); }

extern "C" int32_t mela_costmodel_plan(int32_t op, int64_t m, int64_t n, int64_t p, int32_t *measure)
{
    if (op != MELA_OP_RANK && op != MELA_OP_NULL && op != MELA_OP_MATMUL) return -1;
    bool ms = false;
    // products: m x n times n x p, the density is A's (m x n)
    const int c = choose_unmeasured(op, (double)m, (double)n, (double)p, (double)m * (double)n, &ms);
    if (measure) *measure = ms ? 1 : 0;
    return c;
}

extern "C" int32_t mela_dispatch_last(double *density)
{
    if (density) *density = t_last_density;
    return t_last_variant;
}

extern "C" int32_t mela_costmodel_config(int32_t op, int32_t index) { return config_variant(op, index); }

extern "C" mela_status mela_dev_popcount(const uint64_t *dM, int64_t ld, int64_t m, int64_t n, int64_t *d_count,
                                         void *stream)
{
    if (m < 0 || n < 0 || !d_count || (m > 0 && n > 0 && (!dM || ld < words_of(n)))) {
        set_error("mela_dev_popcount: bad shape, leading dimension or pointer");
        return MELA_ERR_INVALID;
    }
    return launch_popcount((const u64 *)dM, ld, m, n, (long long *)d_count, (cudaStream_t)stream);
}
