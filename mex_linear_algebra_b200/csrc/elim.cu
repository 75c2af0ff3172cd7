// elim.cu -- Gaussian elimination over GF(2) on packed device matrices:
// rank (forward elimination) and reduced row echelon form, in two forms.
//
// Results are those of the reference's algorithms: the rank of
// bitrank_packed / rank_m4ri (src/mela_rank_gf2.c:27-121,
// src/mela_rank_m4ri.c:94-279), and the pivot columns and RREF rows of
// gf2_rref_standard (src/mela_null_gf2.c:88-131).  Both are properties of
// the row space (greedy pivot columns, unique RREF), so any elimination
// order that keeps the pivots greedy reproduces them bit for bit.
//
// Rows never move in memory.  Each row is "active" (not yet a pivot) or a
// pivot; pivot t of the result lives in physical row prow[t] and has its
// leading one in column piv[t].  RREF row t is therefore M[prow[t]].
//
// Blocked form (the Four-Russians / PLE form), one 64-column panel (one
// word column w) at a time:
//   panel_select  one CTA.  Each warp inserts its rows' panel words into a
//                 warp-local XOR basis (lowest set bit leading, warp ballots
//                 resolve who inserts next); the 32 warp bases are merged by
//                 re-inserting their ORIGINAL words, so the final basis is
//                 spanned by p original active rows S.  Its leading bits are
//                 the panel's greedy pivot columns.  A warp Gauss-Jordan on
//                 Q = S restricted to the pivot columns gives, for each
//                 pivot k, the combination coef[k] of S rows whose panel part
//                 is the unit vector of that pivot column.
//   panel_rows    R_k = XOR of the S rows in coef[k] (full width from word
//                 w on), written to a panel buffer and over the S rows.
//   panel_update  every other row j (active rows for rank; all rows for
//                 RREF) XORs sum_k bit(c_k of row j) * R_k, looked up 8 pivot
//                 bits at a time in shared-memory tables of the 256
//                 combinations of 8 R rows (built level by level).
// Plain form: one cooperative persistent kernel, one grid barrier per
// column: every CTA searches its rows for the first active row holding the
// column's bit (atomicMin over the grid), then every CTA XORs that pivot row
// into its rows holding the bit.
#include <climits>
#include <cstring>

#include "mela_common.cuh"
#include "mela_internal.h"
#include "mela_host.h"
#include "elim.h"
#include "basis.cuh"

namespace mela {

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ int ctz64(u64 x) { return ctz64_(x); }

// Panel bookkeeping shared by the three blocked kernels (device memory).
struct PanelState {
    long long rank;  // pivots found so far
    int p;           // pivots in the current panel
    int pad;
    u64 pivmask;     // pivot bit positions of the current panel
    int srow[64];    // physical row that receives R_k
    int sel[64];     // original S rows (index i of coef)
    u64 coef[64];    // R_k = XOR_{i in coef[k]} row sel[i]
};

// ---------------------------------------------------------------- panel_select
namespace {
constexpr int SEL_WARPS = 32;
struct SelSmem {
    WarpBasis wb[SEL_WARPS];
    u64 have[SEL_WARPS];
    int bits[64];
};
}  // namespace

__global__ void __launch_bounds__(1024, 1)
panel_select_kernel(const u64 *__restrict__ M, i64 ld, i64 m, i64 w, unsigned char *state,
                    int *stamp, int panel, PanelState *ps, long long *piv, long long *prow,
                    u64 *__restrict__ ysnap)
{
    extern __shared__ __align__(16) unsigned char sel_raw[];
    SelSmem &sm = *reinterpret_cast<SelSmem *>(sel_raw);
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    u64 have = 0;
    for (i64 chunk = wi; chunk * 32 < m; chunk += SEL_WARPS) {
        const i64 j = chunk * 32 + lane;
        u64 x = 0;
        if (j < m) {
            // the update kernel reads every row's panel word from this snapshot,
            // because the CTA owning word w rewrites it while the others read it
            const u64 word = M[j * ld + w];
            ysnap[j] = word;
            if (state[j]) x = word;
        }
        warp_basis_insert(sm.wb[wi], x, x, (int)j, have);
    }
    if (lane == 0) sm.have[wi] = have;
    for (int step = 1; step < SEL_WARPS; step <<= 1) {
        __syncthreads();
        if ((wi % (2 * step)) == 0 && wi + step < SEL_WARPS) {
            warp_basis_merge(sm.wb[wi], have, sm.wb[wi + step], sm.have[wi + step]);
            if (lane == 0) sm.have[wi] = have;
        }
    }
    __syncthreads();
    if (wi != 0) return;

    const u64 pm = have;
    const long long r0 = ps->rank;
    const int p = warp_panel_gauss_jordan(sm.wb[0], pm, sm.bits, ps->coef, ps->srow, ps->sel);
    for (int t = lane; t < p; t += 32) {
        const int rs = ps->srow[t];
        piv[r0 + t] = 64 * w + sm.bits[t];
        prow[r0 + t] = rs;
        state[rs] = 0;
        stamp[rs] = panel;
    }
    if (lane == 0) {
        ps->p = p;
        ps->pivmask = pm;
        ps->rank = r0 + p;
    }
}

// ---------------------------------------------------------------- panel_rows
// Block: 32 words x all p rows.  Loads S rows' words into shared memory,
// forms R_k, writes R_k to the panel buffer and over row srow[k].
__global__ void __launch_bounds__(256)
panel_rows_kernel(u64 *__restrict__ M, i64 ld, i64 wc, i64 w, const PanelState *ps,
                  u64 *__restrict__ Rbuf)
{
    __shared__ u64 S[64][33];
    __shared__ u64 coef[64];
    __shared__ int srow[64];
    const int p = ps->p;
    if (p == 0) return;
    const i64 w0 = w + (i64)blockIdx.x * 32;
    const int tid = threadIdx.x;
    for (int e = tid; e < p * 32; e += 256) {
        const int i = e >> 5, t = e & 31;
        const i64 word = w0 + t;
        S[i][t] = word < wc ? M[(i64)ps->sel[i] * ld + word] : 0ull;
    }
    if (tid < p) {
        coef[tid] = ps->coef[tid];
        srow[tid] = ps->srow[tid];
    }
    __syncthreads();
    u64 out[8];
    int cnt = 0;
    for (int e = tid; e < p * 32; e += 256) {
        const int k = e >> 5, t = e & 31;
        u64 c = coef[k], v = 0;
        while (c) {
            const int i = ctz64(c);
            c &= c - 1;
            v ^= S[i][t];
        }
        out[cnt++] = v;
    }
    __syncthreads();  // every S row is read before any is overwritten
    cnt = 0;
    for (int e = tid; e < p * 32; e += 256) {
        const int k = e >> 5, t = e & 31;
        const i64 word = w0 + t;
        const u64 v = out[cnt++];
        if (word < wc) {
            M[(i64)srow[k] * ld + word] = v;
            Rbuf[(i64)k * wc + word] = v;
        }
    }
}

// ---------------------------------------------------------------- panel_update
// Four-Russians update with tables of K pivot bits (M4RI k = K).  The panel's
// 64 bit positions are cut into G = ceil(64/K) groups of consecutive
// positions (the last one shorter when K does not divide 64); group g's table
// holds the 2^bits(g) XOR combinations of the reduced rows R of its positions
// (zero rows where a position holds no pivot), built level by level: entry v
// = entry (v - 2^h) ^ entry 2^h for v in (2^h, 2^(h+1)).  Every other row j
// (active rows for the rank; all rows for the RREF) then XORs, per word,
// one entry per group, indexed by its panel bits at the pivot positions.
// Each CTA covers TW words (columns) and `rt` rows; the table build is paid
// once per CTA, so a larger K (fewer lookups per row) pays off with more
// rows per CTA.  Shared memory: (G-1)*2^K + 2^bits(G-1) entries of TW words.
template <int K>
struct M4riGroups {
    static constexpr int G = (64 + K - 1) / K;
    static constexpr int last_bits = 64 - (G - 1) * K;
    static constexpr int entries = (G - 1) * (1 << K) + (1 << last_bits);
    __host__ __device__ static constexpr int bits(int g) { return g == G - 1 ? last_bits : K; }
};

template <int K, int TW>
__global__ void __launch_bounds__(256)
panel_update_kernel(u64 *__restrict__ M, i64 ld, i64 m, i64 wc, i64 w, const PanelState *ps,
                    const u64 *__restrict__ Rbuf, const unsigned char *state, const int *stamp,
                    int panel, int rref, const u64 *__restrict__ ysnap, int rt)
{
    using Gr = M4riGroups<K>;
    extern __shared__ __align__(16) unsigned char upd_raw[];
    u64 *T = reinterpret_cast<u64 *>(upd_raw);  // entry e of group g: T[((g << K) + e) * TW + t]
    const int p = ps->p;
    if (p == 0) return;
    const u64 pm = ps->pivmask;
    const i64 w0 = w + (i64)blockIdx.x * TW;
    const int tid = threadIdx.x;

    // level 0: entry 0 of every group is zero, entry 2^h of group g is R'(gK + h)
    for (int e = tid; e < Gr::G * TW; e += 256) T[(((e / TW) << K)) * TW + e % TW] = 0;
    for (int e = tid; e < 64 * TW; e += 256) {
        const int t = e % TW, b = e / TW, g = b / K, h = b - g * K;
        const i64 word = w0 + t;
        u64 v = 0;
        if (((pm >> b) & 1) && word < wc) {
            const int k = __popcll(pm & ((1ull << b) - 1));
            v = Rbuf[(i64)k * wc + word];
        }
        T[((g << K) + (1 << h)) * TW + t] = v;
    }
    __syncthreads();
#pragma unroll 1
    for (int h = 1; h < K; ++h) {
        const int cnt = (1 << h) - 1;
        for (int e = tid; e < Gr::G * cnt * TW; e += 256) {
            const int t = e % TW, rest = e / TW, g = rest / cnt, v = (1 << h) + 1 + rest % cnt;
            if (h < Gr::bits(g)) {
                u64 *Tg = T + ((size_t)g << K) * TW;
                Tg[v * TW + t] = Tg[(v - (1 << h)) * TW + t] ^ Tg[(1 << h) * TW + t];
            }
        }
        __syncthreads();
    }

    const i64 row0 = (i64)blockIdx.y * rt;
    const int t = tid % TW;
    const i64 word = w0 + t;
    for (int rr = tid / TW; rr < rt; rr += 256 / TW) {
        const i64 j = row0 + rr;
        if (j >= m) break;
        if (rref ? (stamp[j] == panel) : (state[j] == 0)) continue;
        const u64 y = ysnap[j] & pm;
        if (!y || word >= wc) continue;
        u64 acc = 0;
#pragma unroll
        for (int g = 0; g < Gr::G; ++g)
            acc ^= T[((g << K) + (int)((y >> (g * K)) & ((1ull << Gr::bits(g)) - 1))) * TW + t];
        M[j * ld + word] ^= acc;
    }
}

// The (K, TW) pairs the blocked form runs with: TW (words per CTA) shrinks as
// the tables grow, keeping them within 100 KB of shared memory.
template <int K>
struct M4riTile;
template <> struct M4riTile<4> { static constexpr int TW = 8; };
template <> struct M4riTile<6> { static constexpr int TW = 8; };
template <> struct M4riTile<7> { static constexpr int TW = 4; };
template <> struct M4riTile<8> { static constexpr int TW = 4; };
template <> struct M4riTile<9> { static constexpr int TW = 2; };
template <> struct M4riTile<10> { static constexpr int TW = 2; };

template <int K>
static mela_status launch_panel_update(u64 *M, i64 ld, i64 m, i64 wc, i64 w, const PanelState *ps,
                                       const u64 *Rbuf, const unsigned char *state, const int *stamp,
                                       int panel, int rref, const u64 *ysnap, int rt, cudaStream_t s,
                                       bool configure)
{
    constexpr int TW = M4riTile<K>::TW;
    constexpr size_t smem = (size_t)M4riGroups<K>::entries * TW * 8;
    if (configure) {
        MELA_CUDA_TRY(cudaFuncSetAttribute(panel_update_kernel<K, TW>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        return MELA_OK;
    }
    const i64 rem = wc - w;
    const i64 rtiles = (m + rt - 1) / rt;
    panel_update_kernel<K, TW><<<dim3((unsigned)((rem + TW - 1) / TW), (unsigned)rtiles), 256, smem, s>>>(
        M, ld, m, wc, w, ps, Rbuf, state, stamp, panel, rref, ysnap, rt);
    return MELA_OK;
}

using PanelUpdateFn = mela_status (*)(u64 *, i64, i64, i64, i64, const PanelState *, const u64 *,
                                      const unsigned char *, const int *, int, int, const u64 *, int,
                                      cudaStream_t, bool);

static PanelUpdateFn panel_update_for(int k)
{
    switch (k) {
    case 4: return launch_panel_update<4>;
    case 6: return launch_panel_update<6>;
    case 7: return launch_panel_update<7>;
    case 8: return launch_panel_update<8>;
    case 9: return launch_panel_update<9>;
    case 10: return launch_panel_update<10>;
    default: return nullptr;
    }
}

// ---------------------------------------------------------------- plain form
struct GridBar {
    unsigned count;
    unsigned gen;
    int abort;
};

__device__ bool grid_sync(GridBar *gb, unsigned nblocks, u32 *err)
{
    __syncthreads();
    __shared__ int s_abort;
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = &gb->gen;
        const unsigned g = *vgen;
        __threadfence();
        if (atomicAdd(&gb->count, 1u) == nblocks - 1) {
            gb->count = 0;
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            int spins = 0;
            while (*vgen == g) {
                if (((++spins) & 255) == 0) {
                    if (*((volatile int *)&gb->abort)) break;
                    if (global_ns() - t0 > kWaitLimitNs) {
                        atomicOr(err, kErrWaitTimeout);
                        atomicExch(&gb->abort, 1);
                        break;
                    }
                }
            }
        }
        __threadfence();
        s_abort = *((volatile int *)&gb->abort);
    }
    __syncthreads();
    return s_abort == 0;
}

__global__ void __launch_bounds__(512)
ge_plain_kernel(u64 *__restrict__ M, i64 ld, i64 m, i64 n, int rref, unsigned char *state,
                long long *piv, long long *prow, long long *rank_out, int *cand, GridBar *gb,
                u32 *err)
{
    extern __shared__ u64 prow_buf[];
    __shared__ int s_min;
    const i64 wc = words_of(n);
    const i64 per = (m + gridDim.x - 1) / gridDim.x;
    const i64 r0 = (i64)blockIdx.x * per;
    const i64 r1 = (r0 + per < m) ? r0 + per : m;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;

    auto search = [&](i64 c) {
        // first active row of this CTA holding bit c -> atomicMin(cand[c % 3])
        if (tid == 0) s_min = INT_MAX;
        __syncthreads();
        if (c < n) {
            const i64 cw = c >> 6;
            const u64 bit = 1ull << (c & 63);
            for (i64 j = r0 + tid; j < r1; j += blockDim.x) {
                if (state[j] && (M[j * ld + cw] & bit)) {
                    atomicMin(&s_min, (int)j);
                    break;
                }
            }
        }
        __syncthreads();
        if (tid == 0 && s_min != INT_MAX) atomicMin(&cand[c % 3], s_min);
    };

    long long r = 0;
    search(0);
    for (i64 c = 0; c < n; ++c) {
        if (!grid_sync(gb, gridDim.x, err)) break;
        const int p = *((volatile int *)&cand[c % 3]);
        if (blockIdx.x == 0 && tid == 0) cand[(c + 2) % 3] = INT_MAX;
        if (p == INT_MAX) {
            search(c + 1);
            continue;
        }
        if (blockIdx.x == 0 && tid == 0) {
            piv[r] = c;
            prow[r] = p;
        }
        ++r;
        if (p >= r0 && p < r1 && tid == 0) state[p] = 0;
        const i64 cw = c >> 6;
        const u64 bit = 1ull << (c & 63);
        for (i64 t = cw + tid; t < wc; t += blockDim.x) prow_buf[t] = M[(i64)p * ld + t];
        __syncthreads();
        // warp per row, lanes over words
        for (i64 j = r0 + warp; j < r1; j += nwarps) {
            if (j == p) continue;
            if (!rref && !state[j]) continue;
            if (!(M[j * ld + cw] & bit)) continue;
            for (i64 t = cw + lane; t < wc; t += 32) M[j * ld + t] ^= prow_buf[t];
        }
        __syncthreads();
        search(c + 1);
        if (r >= m) break;  // every row is a pivot: no later column can hold one
    }
    if (blockIdx.x == 0 && tid == 0 && rank_out) *rank_out = r;
}

// ---------------------------------------------------------------- null basis
// Pivot-column bitmap and per-word pivot counts.
__global__ void pivmask_kernel(const long long *piv, long long r, u64 *pm)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r;
         t += (long long)gridDim.x * blockDim.x)
        atomicOr(&pm[piv[t] >> 6], 1ull << (piv[t] & 63));
}

// One CTA: exclusive scans of pivot and free counts per word; free column list.
__global__ void __launch_bounds__(1024)
free_cols_kernel(const u64 *pm, i64 wc, i64 n, long long *pbase, long long *free_cols)
{
    __shared__ long long s_pc[1024], s_fc[1024];
    __shared__ long long carry_p, carry_f;
    if (threadIdx.x == 0) carry_p = carry_f = 0;
    __syncthreads();
    for (i64 base = 0; base < wc; base += 1024) {
        const i64 W = base + threadIdx.x;
        u64 pmw = 0, fm = 0;
        if (W < wc) {
            pmw = pm[W];
            const i64 valid = n - 64 * W;
            const u64 vm = valid >= 64 ? ~0ull : ((1ull << valid) - 1);
            fm = ~pmw & vm;
        }
        s_pc[threadIdx.x] = __popcll(pmw);
        s_fc[threadIdx.x] = __popcll(fm);
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            long long vp = 0, vf = 0;
            if ((int)threadIdx.x >= off) {
                vp = s_pc[threadIdx.x - off];
                vf = s_fc[threadIdx.x - off];
            }
            __syncthreads();
            s_pc[threadIdx.x] += vp;
            s_fc[threadIdx.x] += vf;
            __syncthreads();
        }
        const long long ep = carry_p + s_pc[threadIdx.x] - __popcll(pmw);
        long long ef = carry_f + s_fc[threadIdx.x] - __popcll(fm);
        if (W < wc) {
            pbase[W] = ep;
            u64 f = fm;
            while (f) {
                free_cols[ef++] = 64 * W + ctz64(f);
                f &= f - 1;
            }
        }
        __syncthreads();
        if (threadIdx.x == 1023) {
            carry_p += s_pc[1023];
            carry_f += s_fc[1023];
        }
        __syncthreads();
    }
}

// Copy RREF rows (physical prow[t]) into a compact r x ld matrix.
__global__ void gather_rows_kernel(const u64 *__restrict__ M, i64 ld, const long long *prow,
                                   long long r, i64 wc, u64 *__restrict__ out, i64 ldo)
{
    const i64 total = r * wc;
    for (i64 e = blockIdx.x * (i64)blockDim.x + threadIdx.x; e < total; e += (i64)gridDim.x * blockDim.x) {
        const i64 t = e / wc, x = e - t * wc;
        out[t * ldo + x] = M[prow[t] * ld + x];
    }
}

// Zt row i = e_{f_i} + sum_p R_p[f_i] e_{piv[p]}: word W takes the bits
// [pbase[W], pbase[W]+popc(pm[W])) of Rt row f_i deposited at pm[W].
__global__ void null_rows_kernel(const u64 *__restrict__ Rt, i64 ldrt, const u64 *__restrict__ pm,
                                 const long long *pbase, const long long *free_cols, long long f,
                                 i64 wc, u64 *__restrict__ Zt, i64 ldz)
{
    const i64 total = f * wc;
    for (i64 e = blockIdx.x * (i64)blockDim.x + threadIdx.x; e < total; e += (i64)gridDim.x * blockDim.x) {
        const i64 i = e / wc, W = e - i * wc;
        const long long fc = free_cols[i];
        u64 out = ((fc >> 6) == W) ? (1ull << (fc & 63)) : 0ull;
        u64 mask = pm[W];
        if (mask) {
            const long long s = pbase[W];
            const u64 *src = Rt + fc * ldrt;
            const i64 sw = s >> 6;
            const int sb = (int)(s & 63);
            u64 win = src[sw] >> sb;
            const int len = __popcll(mask);
            if (sb && sb + len > 64) win |= src[sw + 1] << (64 - sb);
            while (mask) {
                const u64 lb = mask & (~mask + 1);
                if (win & 1) out |= lb;
                win >>= 1;
                mask ^= lb;
            }
        }
        Zt[i * ldz + W] = out;
    }
}

// Packed rows -> row-major bytes (row i of Zt = column i of the n x f logical Z).
__global__ void unpack_rows_kernel(const u64 *__restrict__ P, i64 ld, i64 rows, i64 n,
                                   unsigned char *__restrict__ out)
{
    const i64 total = rows * n;
    for (i64 e = (blockIdx.x * (i64)blockDim.x + threadIdx.x) * 4; e < total;
         e += (i64)gridDim.x * blockDim.x * 4) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const i64 x = e + q;
            if (x < total) {
                const i64 i = x / n, j = x - i * n;
                out[x] = (unsigned char)((P[i * ld + (j >> 6)] >> (j & 63)) & 1);
            }
        }
    }
}

// ---------------------------------------------------------------- host side
static int grid_cap(i64 total, int threads)
{
    i64 g = (total + threads - 1) / threads;
    const i64 cap = (i64)sm_count() * 16;
    if (g > cap) g = cap;
    return (int)(g < 1 ? 1 : g);
}

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

ElimLayout elim_layout(i64 m, i64 n)
{
    ElimLayout L{};
    const i64 wc = words_of(n);
    size_t off = 0;
    L.state = off;  off += al256((size_t)m);
    L.stamp = off;  off += al256((size_t)m * 4);
    L.ps = off;     off += al256(sizeof(PanelState));
    L.rbuf = off;   off += al256((size_t)64 * (size_t)(wc ? wc : 1) * 8);
    L.cand = off;   off += al256(3 * sizeof(int));
    L.gb = off;     off += al256(sizeof(GridBar));
    L.ysnap = off;  off += al256((size_t)m * 8);
    L.total = off;
    return L;
}

size_t elim_workspace(i64 m, i64 n)
{
    const size_t a = elim_layout(m, n).total, b = fused_workspace(m, n), c = elim_tc_workspace(m, n);
    const size_t ab = a > b ? a : b;
    return ab > c ? ab : c;
}

mela_status elim_device(int variant_arg, u64 *M, i64 ld, i64 m, i64 n, int rref, long long *d_rank,
                        long long *d_piv, long long *d_prow, void *ws, size_t ws_bytes,
                        cudaStream_t s)
{
    Tuning tune{};
    if (m > 0 && n > 0) variant_arg = resolve_elim_variant(variant_arg, M, ld, m, n, rref, s);
    if (!decode_elim_variant(variant_arg, &tune)) {
        set_error("elimination: bad variant argument 0x%x", variant_arg);
        return MELA_ERR_INVALID;
    }
    const int variant = tune.base;
    if (m == 0 || n == 0) {
        MELA_CUDA_TRY(cudaMemsetAsync(d_rank, 0, sizeof(long long), s));
        return MELA_OK;
    }
    if (m > INT_MAX - 1) {
        set_error("elimination: more than 2^31-2 rows");
        return MELA_ERR_UNSUPPORTED;
    }
    if (variant == MELA_ELIM_FUSED)
        return launch_fused_elim(M, ld, m, n, d_rank, d_piv, d_prow, ws, ws_bytes, s);
    if (variant == MELA_ELIM_TC) return elim_tc_device(M, ld, m, n, rref, d_rank, d_piv, d_prow, ws, ws_bytes, s);
    ElimLayout L = elim_layout(m, n);
    if (ws_bytes < L.total || !ws) {
        set_error("elimination workspace of %zu bytes needed, %zu given", elim_workspace(m, n), ws_bytes);
        return MELA_ERR_INVALID;
    }
    unsigned char *w = (unsigned char *)ws;
    unsigned char *state = w + L.state;
    int *stamp = (int *)(w + L.stamp);
    PanelState *ps = (PanelState *)(w + L.ps);
    u64 *rbuf = (u64 *)(w + L.rbuf);
    int *cand = (int *)(w + L.cand);
    GridBar *gb = (GridBar *)(w + L.gb);
    u64 *ysnap = (u64 *)(w + L.ysnap);
    const i64 wc = words_of(n);

    MELA_CUDA_TRY(cudaMemsetAsync(state, 1, (size_t)m, s));
    if (variant == MELA_ELIM_PLAIN) {
        int init[3] = {INT_MAX, INT_MAX, INT_MAX};
        MELA_CUDA_TRY(cudaMemcpyAsync(cand, init, sizeof init, cudaMemcpyHostToDevice, s));
        MELA_CUDA_TRY(cudaMemsetAsync(gb, 0, sizeof(GridBar), s));
        int dev = 0, per_sm = 0;
        MELA_CUDA_TRY(cudaGetDevice(&dev));
        const size_t smem = (size_t)wc * 8;
        if (smem > 200 * 1024) {
            set_error("plain elimination: rows of %lld words exceed the shared-memory pivot buffer", wc);
            return MELA_ERR_UNSUPPORTED;
        }
        MELA_CUDA_TRY(cudaFuncSetAttribute(ge_plain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        MELA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ge_plain_kernel, 512, smem));
        if (per_sm < 1) {
            set_error("plain elimination kernel cannot be resident");
            return MELA_ERR_UNSUPPORTED;
        }
        i64 blocks = (i64)sm_count();  // one CTA per SM keeps barriers cheap
        const i64 by_rows = (m + 31) / 32;
        if (blocks > by_rows) blocks = by_rows;
        if (blocks < 1) blocks = 1;
        u32 *err = device_error_word();
        long long *rank_out = d_rank;
        void *args[] = {&M, &ld, &m, &n, &rref, &state, &d_piv, &d_prow, &rank_out, &cand, &gb, &err};
        MELA_CUDA_TRY(cudaLaunchCooperativeKernel((void *)ge_plain_kernel, dim3((unsigned)blocks),
                                                  dim3(512), args, smem, s));
        MELA_LAUNCH_CHECK("ge_plain_kernel");
        return MELA_OK;
    }
    if (variant != MELA_ELIM_M4RI && variant != MELA_ELIM_M4RI_K4) {
        set_error("unknown elimination variant %d", variant);
        return MELA_ERR_INVALID;
    }
    MELA_CUDA_TRY(cudaMemsetAsync(stamp, 0xff, (size_t)m * 4, s));
    MELA_CUDA_TRY(cudaMemsetAsync(ps, 0, sizeof(PanelState), s));
    const size_t sel_smem = sizeof(SelSmem);
    MELA_CUDA_TRY(cudaFuncSetAttribute(panel_select_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sel_smem));
    const PanelUpdateFn update = panel_update_for(tune.k);
    if (!update) {
        set_error("blocked elimination: M4RI k = %d (4 or 6..10 supported)", tune.k);
        return MELA_ERR_INVALID;
    }
    const int rt = tune.row_tile;
    if (mela_status st = check_grid_yz((m + rt - 1) / rt, 1, "blocked elimination update"); st != MELA_OK)
        return st;
    if (mela_status st = update(M, ld, m, wc, 0, ps, rbuf, state, stamp, 0, rref, ysnap, rt, s, true);
        st != MELA_OK)
        return st;
    for (i64 pw = 0; pw < wc; ++pw) {  // every word column is one panel
        panel_select_kernel<<<1, 1024, sel_smem, s>>>(M, ld, m, pw, state, stamp, (int)pw, ps,
                                                       d_piv, d_prow, ysnap);
        const i64 rem = wc - pw;
        panel_rows_kernel<<<(unsigned)((rem + 31) / 32), 256, 0, s>>>(M, ld, wc, pw, ps, rbuf);
        update(M, ld, m, wc, pw, ps, rbuf, state, stamp, (int)pw, rref, ysnap, rt, s, false);
    }
    MELA_LAUNCH_CHECK("panel elimination");
    MELA_CUDA_TRY(cudaMemcpyAsync(d_rank, &ps->rank, sizeof(long long), cudaMemcpyDeviceToDevice, s));
    return MELA_OK;
}

NullLayout null_layout(i64 n, i64 rank)
{
    NullLayout L{};
    const i64 wc = words_of(n);
    const i64 ldr = even_words(rank > 0 ? rank : 1);
    size_t off = 0;
    L.pm = off;     off += al256((size_t)wc * 8);
    L.pbase = off;  off += al256((size_t)wc * 8);
    L.free = off;   off += al256((size_t)(n ? n : 1) * 8);
    L.rc = off;     off += al256((size_t)(rank ? rank : 1) * (size_t)(wc ? wc : 1) * 8);
    L.rt = off;     off += al256((size_t)(n ? n : 1) * (size_t)ldr * 8);
    L.ldr = ldr;
    L.total = off;
    return L;
}

mela_status null_basis_device(const u64 *M, i64 ld, i64 m, i64 n, i64 rank, const long long *d_piv,
                              const long long *d_prow, u64 *Zt, i64 ldz, void *ws, size_t ws_bytes,
                              cudaStream_t s)
{
    (void)m;
    const i64 f = n - rank;
    if (f <= 0) return MELA_OK;
    NullLayout L = null_layout(n, rank);
    if (ws_bytes < L.total || !ws) {
        set_error("null-space workspace of %zu bytes needed, %zu given", L.total, ws_bytes);
        return MELA_ERR_INVALID;
    }
    unsigned char *w = (unsigned char *)ws;
    u64 *pm = (u64 *)(w + L.pm);
    long long *pbase = (long long *)(w + L.pbase);
    long long *free_cols = (long long *)(w + L.free);
    u64 *Rc = (u64 *)(w + L.rc);
    u64 *Rt = (u64 *)(w + L.rt);
    const i64 wc = words_of(n);
    MELA_CUDA_TRY(cudaMemsetAsync(pm, 0, (size_t)wc * 8, s));
    if (rank > 0) {
        pivmask_kernel<<<grid_cap(rank, 256), 256, 0, s>>>(d_piv, rank, pm);
        gather_rows_kernel<<<grid_cap(rank * wc, 256), 256, 0, s>>>(M, ld, d_prow, rank, wc, Rc, wc);
        mela_status st = launch_transpose(Rc, wc, rank, n, Rt, L.ldr, s);
        if (st != MELA_OK) return st;
    } else {
        MELA_CUDA_TRY(cudaMemsetAsync(Rt, 0, (size_t)n * L.ldr * 8, s));
    }
    free_cols_kernel<<<1, 1024, 0, s>>>(pm, wc, n, pbase, free_cols);
    null_rows_kernel<<<grid_cap(f * wc, 256), 256, 0, s>>>(Rt, L.ldr, pm, pbase, free_cols, f, wc, Zt, ldz);
    MELA_LAUNCH_CHECK("null basis");
    return MELA_OK;
}

mela_status launch_unpack_rows(const u64 *P, i64 ld, i64 rows, i64 n, unsigned char *out, cudaStream_t s)
{
    if (rows <= 0 || n <= 0) return MELA_OK;
    unpack_rows_kernel<<<grid_cap((rows * n + 3) / 4, 256), 256, 0, s>>>(P, ld, rows, n, out);
    MELA_LAUNCH_CHECK("unpack_rows_kernel");
    return MELA_OK;
}

}  // namespace mela
