// batch.cu -- rank and null space of many matrices in one persistent launch.
//
// Each matrix gets the reference's results (rank as src/mela_rank_gf2.c,
// null-space basis as src/mela_null_gf2.c:189-274, bit for bit) from a
// reduced row echelon form computed by one thread group:
//
//   class  group            storage of the matrix
//   small  one warp         its slice of shared memory (13 KB)
//   mid    128 threads      its slice of shared memory (55 KB)
//   big    the whole CTA    shared memory (up to ~110 KB) or, when it does
//          (256 threads)    not fit, the CTA's L2-resident global scratch;
//                           blocked by 64-column panels (process_big_blocked)
//
// (two CTAs per SM; the single-matrix fused mode runs the same engines in
// one CTA of 512 threads with 220 KB)
//
// The host sorts the matrices into the three classes (largest first inside
// each class); every CTA drains the big queue, then the mid queue (2 groups),
// then the small queue (8 warps), taking the next matrix with an atomic on
// the class counter.  A group eliminates column by column: the rows are
// dealt round-robin to its threads; per column each thread looks for the
// first active row of its own holding the bit, a warp min (+ shared atomic
// for multi-warp groups) picks the pivot, and every thread XORs the pivot row
// into its rows holding the bit.  One group barrier per column suffices: the
// search for column c+1 runs right after the XOR of column c on the same
// thread's own rows.  Rows never move; the null basis is then assembled
// directly: Zt row i = e_{f_i} + sum_p RREF(p, f_i) e_{piv(p)}.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "mela_common.cuh"
#include "mela_internal.h"
#include "mela_host.h"
#include "basis.cuh"

namespace mela {

struct BatchDevItem {
    int m, n;
    int flags;  // bit 0: matrix held in shared memory
    int pad;
    long long in_off, z_off;
};

// Outputs of the single-matrix ("fused") mode: instead of a null basis, the
// RREF rows are written back over the caller's matrix, with the pivot lists.
struct FusedOut {
    u64 *M;
    long long ldm;
    long long *rank, *piv, *prow;
};

namespace {
constexpr int kThreads = 512;
constexpr int kMidGroup = 128;
constexpr int kSmemTotal = 220 * 1024;
constexpr int kMidBudget = kSmemTotal / (kThreads / kMidGroup);  // 55 KB
constexpr int kSmallBudget = kSmemTotal / (kThreads / 32);       // 13.75 KB
// the batch launch: two CTAs of 256 threads per SM, each with half the
// shared memory, so that one CTA's barrier-bound panel steps overlap the
// other's table updates and transposes
constexpr int kBatchThreads = 256;
constexpr int kSmallMaxRows = 192;  // largest m for the warp engine
constexpr int kMidMaxRows = 240;    // the 128-thread engine below this m
constexpr int kBatchSmem = kSmemTotal / (kThreads / kBatchThreads);

__host__ __device__ inline size_t al8(size_t x) { return (x + 7) & ~(size_t)7; }

// Byte size of the per-matrix bookkeeping arrays in a group's region.
__host__ __device__ inline size_t aux_bytes(int m, int n)
{
    const int wc = (n + 63) >> 6, mn = m < n ? m : n;
    return al8((size_t)4 * (2 * (size_t)mn + (size_t)n + (size_t)wc + 1)) + 8 * (size_t)wc +
           al8((size_t)m) + 16;
}
__host__ __device__ inline int smem_ld(int n)
{
    const int wc = (n + 63) >> 6;
    return wc | 1;  // odd pitch: threads on consecutive rows hit different banks
}
}  // namespace

__device__ __forceinline__ void group_sync(int G, int bar_id)
{
    if (G == 32) {
        __syncwarp();
    } else if (G == kThreads) {
        __syncthreads();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(G) : "memory");
    }
}

__device__ __forceinline__ int ctz64b(u64 x) { return __ffsll((long long)x) - 1; }

// RREF + null basis of one matrix by a group of G threads.
template <int G>
__device__ void process_matrix(const BatchDevItem &it, const u64 *__restrict__ in, u64 *__restrict__ zt,
                               long long *ranks, int item, unsigned char *region, u64 *gmat, int gtid,
                               int bar_id, const FusedOut *fo = nullptr)
{
    const int m = it.m, n = it.n, wc = (n + 63) >> 6, mn = m < n ? m : n;
    const bool in_smem = it.flags & 1;
    const int ld = in_smem ? smem_ld(n) : wc;
    u64 *A = in_smem ? reinterpret_cast<u64 *>(region) : gmat;
    unsigned char *aux = region + (in_smem ? (size_t)m * ld * 8 : 0);
    int *piv = reinterpret_cast<int *>(aux);
    int *prow = piv + mn;
    int *fcol = prow + mn;
    int *pbase = fcol + n;
    u64 *pm = reinterpret_cast<u64 *>(aux + al8((size_t)4 * (2 * (size_t)mn + (size_t)n + (size_t)wc + 1)));
    unsigned char *active = reinterpret_cast<unsigned char *>(pm + wc);
    int *slots = reinterpret_cast<int *>(active + al8((size_t)m));
    const int lane = gtid & 31;

    // load the packed matrix, mark every row active
    const u64 *src = in + it.in_off;
    for (long long e = gtid; e < (long long)m * wc; e += G) {
        const int r = (int)(e / wc), x = (int)(e - (long long)r * wc);
        A[(size_t)r * ld + x] = src[e];
    }
    for (int j = gtid; j < m; j += G) active[j] = 1;
    if (gtid < 3) slots[gtid] = INT_MAX;
    group_sync(G, bar_id);

    auto search = [&](int c) {
        if (c >= n) return;
        const int cw = c >> 6;
        const u64 bit = 1ull << (c & 63);
        unsigned best = INT_MAX;
        for (int j = gtid; j < m; j += G)
            if (active[j] && (A[(size_t)j * ld + cw] & bit)) {
                best = (unsigned)j;
                break;
            }
        best = __reduce_min_sync(0xffffffffu, best);
        if (lane == 0 && best != (unsigned)INT_MAX) atomicMin(&slots[c % 3], (int)best);
    };

    int r = 0;
    search(0);
    group_sync(G, bar_id);
    for (int c = 0; c < n && r < m; ++c) {
        const int p = slots[c % 3];
        if (gtid == 0) slots[(c + 2) % 3] = INT_MAX;
        if (p != INT_MAX) {
            if (gtid == 0) {
                piv[r] = c;
                prow[r] = p;
            }
            if (p % G == gtid) active[p] = 0;
            ++r;
            const int cw = c >> 6;
            const u64 bit = 1ull << (c & 63);
            const u64 *pr = A + (size_t)p * ld;
            for (int j = gtid; j < m; j += G) {
                if (j == p) continue;
                u64 *row = A + (size_t)j * ld;
                if (!(row[cw] & bit)) continue;
                for (int t = cw; t < wc; ++t) row[t] ^= pr[t];
            }
        }
        search(c + 1);
        group_sync(G, bar_id);
    }
    if (fo) {
        // single-matrix mode: RREF rows back to the caller, pivot lists, rank
        for (long long e = gtid; e < (long long)m * wc; e += G) {
            const int rr = (int)(e / wc), x = (int)(e - (long long)rr * wc);
            fo->M[(long long)rr * fo->ldm + x] = A[(size_t)rr * ld + x];
        }
        for (int t = gtid; t < r; t += G) {
            fo->piv[t] = piv[t];
            fo->prow[t] = prow[t];
        }
        if (gtid == 0) *fo->rank = r;
        group_sync(G, bar_id);
        return;
    }
    if (gtid == 0) ranks[item] = r;

    // null basis: pivot mask per word, pivots before each word, free columns
    const int f = n - r;
    for (int W = gtid; W < wc; W += G) pm[W] = 0;
    group_sync(G, bar_id);
    for (int t = gtid; t < r; t += G) atomicOr(&pm[piv[t] >> 6], 1ull << (piv[t] & 63));
    group_sync(G, bar_id);
    if (gtid == 0) {
        int pc = 0, fc = 0;
        for (int W = 0; W < wc; ++W) {
            pbase[W] = pc;
            pc += __popcll(pm[W]);
            const int valid = n - 64 * W;
            const u64 vm = valid >= 64 ? ~0ull : ((1ull << valid) - 1);
            u64 fm = ~pm[W] & vm;
            while (fm) {
                fcol[fc++] = 64 * W + ctz64b(fm);
                fm &= fm - 1;
            }
        }
        pbase[wc] = pc;
    }
    group_sync(G, bar_id);
    u64 *Z = zt + it.z_off;
    for (long long e = gtid; e < (long long)f * wc; e += G) {
        const int i = (int)(e / wc), W = (int)(e - (long long)i * wc);
        const int fi = fcol[i], fw = fi >> 6, fb = fi & 63;
        u64 out = (fw == W) ? (1ull << fb) : 0ull;
        for (int q = pbase[W]; q < pbase[W + 1]; ++q)
            out |= ((A[(size_t)prow[q] * ld + fw] >> fb) & 1ull) << (piv[q] & 63);
        Z[e] = out;
    }
    group_sync(G, bar_id);
}

// ---------------------------------------------------------------- big matrices
// Global-scratch layout (words) of one big matrix: A (m x wc), then the
// arrays that do not fit in shared memory.  See big_layout().
struct BigLayout {
    long long A, Rg, ysg, yvg, tagg, ints, pm, active, rt, q, total;  // word offsets
};

__host__ __device__ inline BigLayout big_layout(long long m, long long n)
{
    const long long wc = (n + 63) / 64, mn = m < n ? m : n;
    BigLayout L;
    long long o = 0;
    L.A = o; o += m * wc;
    L.Rg = o; o += 128 * wc;          // stage + reduced rows when shared memory is short
    L.ysg = o; o += m;
    L.yvg = o; o += m;
    L.tagg = o; o += m;
    L.ints = o; o += (2 * mn + 2 * n + wc + 2 + 1) / 2 + 1;  // piv, prow, fcol, cmap, pbase
    L.pm = o; o += wc;
    L.active = o; o += (m + 7) / 8;
    // R^T and (R restricted to free columns), 32-bit words, rows padded to
    // a multiple of 4 words and 16-byte aligned (vector stores)
    o = (o + 1) & ~1LL;
    L.rt = o; o += n * ((mn + 127) / 128) * 2;
    L.q = o; o += mn * ((n + 127) / 128) * 2;
    L.total = (o + 8 + 1) & ~1LL;  // even: every CTA's scratch stays 16-byte aligned
    return L;
}
__host__ __device__ inline long long big_scratch_words(long long m, long long n)
{
    return big_layout(m, n).total;
}

namespace {
constexpr int kRegThreads = 256;  // threads holding a panel in registers (m <= 1024)
constexpr int kRegRows = 4;        // rows per thread there
constexpr int kRegWarps = kRegThreads / 32;
static_assert(kRegWarps == 8, "eight candidate slots");
constexpr int kRegBar = 6;         // their named barrier
constexpr int kSubBar = 5;         // the update warps while warp 0 selects the next panel's pivots
constexpr int kCandMax = 384;      // candidate rows one warp selects pivots among (12 a lane)
template <int TW>
struct BigSmem {
    u64 coef[64];
    int cand[kCandMax];  // the panel's candidate rows, in row order
    int prev_srow[64];   // the pivot rows of the panel being updated (look-ahead)
    int wcnt[16];        // candidates per warp
    int ucnt[16];        // rows to update per warp
    u64 pub[2][kRegWarps][2];  // per warp: its candidate pivot's panel word and tag (by bit parity)
    alignas(16) unsigned wmin[2][kRegWarps];  // per warp: its candidate pivot row
    int bits[64], srow[64];
    int slots[4];
    u64 T[16][16][TW];  // nibble tables of the current chunk (TW words)
    u64 pm;
    int p;
};
// The big-matrix engine for a CTA of NT threads with SMEM bytes of shared
// memory: TW words per update chunk (32, one per lane, for 512 threads; 16,
// two rows per warp instruction, for 256 threads, which halves the tables);
// after BigSmem, kExtra bytes hold the panel stage + reduced rows, then the
// per-row panel words (snapshot, working copy, combination tags) and the
// matrix itself, each when it fits.
template <int NT, int SMEM>
struct BigCfg {
    static constexpr int TW = NT >= 512 ? 32 : 16;
    using Smem = BigSmem<TW>;
    static constexpr size_t kHead = (sizeof(Smem) + 15) & ~(size_t)15;
    static constexpr size_t kExtra = (size_t)SMEM - kHead;
    static_assert(sizeof(Smem) <= (size_t)SMEM, "big-matrix shared memory");
    static_assert(NT >= kRegThreads, "the register panel needs 256 threads");
};
}  // namespace

// v[i] for a lane-local index i < R (R <= 16) by a select tree: no local
// memory and a dependence depth of four selects.
template <int R>
__device__ __forceinline__ u64 pick_reg(const u64 (&v)[R], int i)
{
    u64 a[8], b[4], c[2];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const u64 lo = 2 * j < R ? v[2 * j] : 0ull, hi = 2 * j + 1 < R ? v[2 * j + 1] : 0ull;
        a[j] = (i & 1) ? hi : lo;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) b[j] = (i & 2) ? a[2 * j + 1] : a[2 * j];
#pragma unroll
    for (int j = 0; j < 2; ++j) c[j] = (i & 4) ? b[2 * j + 1] : b[2 * j];
    return (i & 8) ? c[1] : c[0];
}

// Bit b of each of a lane's R words, as an R-bit mask (four independent
// partial masks, so that the dependence chain stays short).
template <int R>
__device__ __forceinline__ u32 bit_mask(const u64 (&y)[R], int b)
{
    const int sh = b & 31;
    u32 h[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const u32 half = (b & 32) ? (u32)(y[i] >> 32) : (u32)y[i];
        h[i & 3] |= ((half >> sh) & 1u) << i;
    }
    return (h[0] | h[1]) | (h[2] | h[3]);
}

// Pivot selection of one panel among its candidate rows (active rows with a
// nonzero panel word; cnt <= 32 R) by one warp, no block barrier: lane l holds
// candidates l + 32 i.  Per bit that some candidate holds (the OR of their
// words: XORs create no other bit), the lowest unused candidate holding it
// becomes pivot k and is XORed into every other candidate holding the bit.
// A step's critical path is a ballot and a shuffle: which rows hold the next
// bit is computed from the words before the XOR (the bit flips in the rows
// that take the pivot where the pivot word has it), and the pivots' bits are
// kept in registers and written out at the end.  The pivots' combination
// tags (which other pivots' original rows make up each reduced pivot row)
// come from a second elimination over the pivots alone, whose pivot rows are
// known: p steps of two shuffles, no ballot.  Writes the pivots' bits, rows
// and tags; returns the pivot count and the pivot mask.
template <int R>
__device__ __forceinline__ int warp_select(const int *cand, int cnt, const u64 *ysnap, u64 *tag, int *bits,
                                           int *srow, u64 *pm_out)
{
    const int lane = threadIdx.x & 31;
    u64 y[R];
    int pb[R];  // the bit a candidate became the pivot of, or -1
    u32 unused = 0;
    u64 orw = 0;
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int c = lane + 32 * i;
        y[i] = c < cnt ? ysnap[cand[c]] : 0ull;
        pb[i] = -1;
        unused |= (c < cnt ? 1u : 0u) << i;
        orw |= y[i];
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) orw |= __shfl_xor_sync(0xffffffffu, orw, o);
    int k = 0;
    u64 pmask = 0;
    u64 rem = orw;
    if (rem) {
        int b = __ffsll((long long)rem) - 1;
        u32 hold = bit_mask<R>(y, b);
        while (true) {
            const u64 rem_n = rem & (rem - 1);
            const int bn = rem_n ? __ffsll((long long)rem_n) - 1 : 0;
            u32 hold_n = bit_mask<R>(y, bn);
            const u32 cm = hold & unused;
            const u32 bal = __ballot_sync(0xffffffffu, cm != 0);
            if (bal) {
                const int src = __ffs((int)bal) - 1;
                const int ib = __ffs((int)cm) - 1;  // meaningful in lane src
                const u64 yp = __shfl_sync(0xffffffffu, pick_reg<R>(y, ib), src);
                const u32 me = lane == src ? (1u << ib) : 0u;
                const u32 hit = hold & ~me;  // every other candidate holding bit b
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    if ((hit >> i) & 1u) y[i] ^= yp;
                    if ((me >> i) & 1u) pb[i] = b;
                }
                unused &= ~me;
                hold_n ^= ((yp >> bn) & 1ull) ? hit : 0u;
                pmask |= 1ull << b;
                ++k;
            }
            if (!rem_n) break;
            rem = rem_n;
            b = bn;
            hold = hold_n;
        }
    }
#pragma unroll
    for (int i = 0; i < R; ++i)
        if (pb[i] >= 0) {
            const int kk = __popcll(pmask & ((1ull << pb[i]) - 1));
            bits[kk] = pb[i];
            srow[kk] = cand[lane + 32 * i];
        }
    __syncwarp();
    // tags: lane l holds pivots l and l + 32 (original panel words)
    u64 v0 = lane < k ? ysnap[srow[lane]] : 0ull, v1 = lane + 32 < k ? ysnap[srow[lane + 32]] : 0ull;
    u64 t0 = 0, t1 = 0;
    for (int q = 0; q < k; ++q) {
        const int bq = bits[q];
        const u64 vq = __shfl_sync(0xffffffffu, q < 32 ? v0 : v1, q & 31);
        const u64 tq = __shfl_sync(0xffffffffu, q < 32 ? t0 : t1, q & 31) ^ (1ull << q);
        if (lane != q && ((v0 >> bq) & 1ull)) {
            v0 ^= vq;
            t0 ^= tq;
        }
        if (lane + 32 != q && ((v1 >> bq) & 1ull)) {
            v1 ^= vq;
            t1 ^= tq;
        }
    }
    if (lane < k) tag[srow[lane]] = t0;
    if (lane + 32 < k) tag[srow[lane + 32]] = t1;
    *pm_out = pmask;
    return k;
}

// Element i (0..3, per thread) of a register array, by a select tree.
__device__ __forceinline__ u64 sel4r(const u64 (&v)[4], int i)
{
    const u64 a0 = (i & 1) ? v[1] : v[0], a1 = (i & 1) ? v[3] : v[2];
    return (i & 2) ? a1 : a0;
}

// 32x32 bit transposes by warp shuffles over a CTA: dst (cols x rows bits,
// 32-bit words, pitch dld) = src^T, where src row r, 32-bit word x is
// srcw(r, x) (rows x cols bits); dst must not overlap what srcw reads.  A
// warp unit is one column tile and four row tiles: each lane ends with four
// consecutive words of its dst row and stores them together (VEC 16: one
// 16-byte store, dst 16-byte aligned with dld % 4 == 0; VEC 8: two 8-byte
// stores, dst 8-byte aligned with dld even), a quarter of the store
// transactions of one word per tile.  A unit spans CW column tiles, read
// as CW consecutive 32-bit words of a source row (srcw(r, xg) = words
// CW xg .. CW xg + CW - 1 of src row r, from one 8- or 16-byte load; four
// reads a lane, all issued before the first shuffle).  dwords: words of a
// dst row that may be written.
template <int CW>
struct TrWords {
    u32 w[CW];
};
template <int NT, int VEC, int CW, typename F>
__device__ void cta_transpose4(F srcw, int rows, int cols, u32 *dst, long long dld, int dwords)
{
    constexpr int kWarps = NT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int rt = (rows + 31) >> 5, ct = (cols + 31) >> 5, rg = (rt + 3) >> 2, cg = (ct + CW - 1) / CW;
    const int total = cg * rg;
    for (int unit = warp; unit < total; unit += kWarps) {
        const int g = unit / cg, tcg = unit - g * cg;
        TrWords<CW> v[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = (4 * g + i) * 32 + lane;
            if (r < rows) {
                v[i] = srcw(r, tcg);
            } else {
#pragma unroll
                for (int h = 0; h < CW; ++h) v[i].w[h] = 0u;
            }
        }
#pragma unroll
        for (int h = 0; h < CW; ++h) {
            u32 o[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) o[i] = transpose32_warp(v[i].w[h]);
            const int c = (CW * tcg + h) * 32 + lane;
            if (c < cols) {
                u32 *d = dst + (long long)c * dld + 4 * g;
                const int left = dwords - 4 * g;
                if (VEC == 16 && left >= 4) {
                    *reinterpret_cast<uint4 *>(d) = make_uint4(o[0], o[1], o[2], o[3]);
                } else if (VEC == 8 && left >= 4) {
                    reinterpret_cast<uint2 *>(d)[0] = make_uint2(o[0], o[1]);
                    reinterpret_cast<uint2 *>(d)[1] = make_uint2(o[2], o[3]);
                } else {
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        if (i < left) d[i] = o[i];
                }
            }
        }
    }
}
// CW consecutive 32-bit words of a row from 8- or 16-byte loads
__device__ __forceinline__ TrWords<2> tr_words2(const u32 *p)
{
    const uint2 x = *reinterpret_cast<const uint2 *>(p);
    return {{x.x, x.y}};
}
__device__ __forceinline__ TrWords<4> tr_words4(const u32 *p)
{
    const uint4 x = *reinterpret_cast<const uint4 *>(p);
    return {{x.x, x.y, x.z, x.w}};
}

// Reduced row echelon form and null basis of a big matrix by the whole CTA,
// 64 columns at a time (the blocked form of elim.cu inside one CTA):
//  * pivot selection among the panel's candidate rows (unused, nonzero
//    panel word) by one warp (warp_select), or, with more than kCandMax
//    candidates, per bit over all rows in registers of eight warps (one named
//    barrier per bit) -- on the panel words only, each pivot carrying a
//    64-bit tag of the pivots folded into it, so pivot k's reduced row is its
//    original row plus the original pivot rows of its tag.  Any independent
//    set of pivot rows spanning the panel gives the same reduced echelon
//    form, hence the same rank and null basis;
//  * the reduced pivot rows R_k are formed from the staged original rows and
//    written over them; every other row is updated with 16 nibble-table
//    lookups per word (tables of the 16 combinations of 4 reduced rows);
//  * look-ahead: words w and w + 1 of every row are updated first (the new
//    word w + 1 is the next panel's snapshot), then one warp selects panel
//    w + 1's pivots while the others update words w + 2 .. over the list of
//    rows that change;
//  * null basis: Zt = (Y)^T with Y row c = (R restricted to free columns)^T
//    row p when c is pivot column p, the unit vector of its free index
//    otherwise -- three 32x32 shuffle transposes, no per-bit gathers.
template <int NT, int SMEM>
__device__ void process_big_blocked(const BatchDevItem &it, const u64 *__restrict__ in,
                                    u64 *__restrict__ zt, long long *ranks, int item,
                                    unsigned char *smem_raw, u64 *g, const FusedOut *fo = nullptr)
{
    using Cfg = BigCfg<NT, SMEM>;
    constexpr int TW = Cfg::TW;
    constexpr size_t kBigExtra = Cfg::kExtra;
    constexpr int kWarps = NT / 32;
    typename Cfg::Smem &S = *reinterpret_cast<typename Cfg::Smem *>(smem_raw);
    const int m = it.m, n = it.n, wc = (n + 63) >> 6, mn = m < n ? m : n;
    const int tid = threadIdx.x, lane = tid & 31;
    const BigLayout L = big_layout(m, n);
    u64 *A = g + L.A;
    int *piv = reinterpret_cast<int *>(g + L.ints);
    int *prow = piv + mn;
    int *fcol = prow + mn;
    int *cmap = fcol + n;
    int *pbase = cmap + n;
    u64 *pm = g + L.pm;
    u32 *Rt = reinterpret_cast<u32 *>(g + L.rt);
    u32 *Q = reinterpret_cast<u32 *>(g + L.q);

    unsigned char *extra = smem_raw + Cfg::kHead;
    const size_t rb_bytes = (size_t)64 * wc * 8, row_bytes = (size_t)m * 8;
    const bool r_in_smem = 2 * rb_bytes <= kBigExtra;
    u64 *stage = r_in_smem ? reinterpret_cast<u64 *>(extra) : g + L.Rg;
    u64 *Rbuf = stage + (size_t)64 * wc;
    size_t used = r_in_smem ? 2 * rb_bytes : 0;
    // row states are read on every bit step: shared memory whenever possible
    const size_t act_bytes = ((size_t)m + 15) & ~(size_t)15;
    unsigned char *active = (used + act_bytes <= kBigExtra) ? extra + used
                                                           : reinterpret_cast<unsigned char *>(g + L.active);
    if (used + act_bytes <= kBigExtra) used += act_bytes;
    const bool rows_in_smem = used + 3 * row_bytes <= kBigExtra;
    u64 *ysnap0 = rows_in_smem ? reinterpret_cast<u64 *>(extra + used) : g + L.ysg;
    u64 *ysnap1 = rows_in_smem ? ysnap0 + m : g + L.yvg;
    u64 *tag = rows_in_smem ? ysnap1 + m : g + L.tagg;
    if (rows_in_smem) used += 3 * row_bytes;
    // the look-ahead's list of rows to update (row order), when it fits
    const size_t ul_bytes = ((size_t)m * 4 + 15) & ~(size_t)15;
    int *ulist = rows_in_smem && used + ul_bytes <= kBigExtra ? reinterpret_cast<int *>(extra + used) : nullptr;
    if (ulist) used += ul_bytes;
    // the matrix itself in shared memory too when it fits (at n = 2m: m up
    // to about 420 with 110 KB, 650 with 220 KB), else in the CTA's
    // L2-resident scratch
    const size_t pre_a_bytes = used;  // shared bytes before the matrix: free again for the null basis
    if (used + (size_t)m * wc * 8 <= kBigExtra) A = reinterpret_cast<u64 *>(extra + used);

    const u64 *src = in + it.in_off;
    for (long long e = tid; e < (long long)m * wc; e += NT) A[e] = src[e];
    for (int j = tid; j < m; j += NT) active[j] = 1;
    __syncthreads();

    // panel words of every row: one buffer for the current panel, the other
    // for the next panel's (look-ahead) or the per-bit path's working copy
    int cur = 0;
    const int warp = tid >> 5;
    // warp q owns rows [q chunk, (q + 1) chunk) for the candidate lists
    const int chunk = (m + 32 * kWarps - 1) / (32 * kWarps) * 32;
    const int jlo = warp * chunk, jhi = min(m, jlo + chunk);
    // the look-ahead's one-word tables (words w and w + 1, 4 KB) live in the
    // stage area, free from the reduced rows of one panel to the next
    const bool lookahead_ok = r_in_smem && 64 * wc >= 2 * 16 * 16;
    bool have_sel = false;  // this panel's pivots were selected during the previous one

    // candidate rows of a panel (active, nonzero panel word) into S.cand in
    // row order, from the per-warp counts in S.wcnt; returns their number
    auto compact = [&](const u64 *ysp) -> int {
        int cbase = 0, total = 0;
        for (int q = 0; q < kWarps; ++q) {
            const int c = S.wcnt[q];
            cbase += q < warp ? c : 0;
            total += c;
        }
        if (total <= kCandMax)
            for (int j0 = jlo; j0 < jhi; j0 += 32) {
                const int j = j0 + lane;
                const bool ok = j < jhi && ysp[j] != 0 && active[j] == 1;
                const u32 bal = __ballot_sync(0xffffffffu, ok);
                if (ok) S.cand[cbase + __popc(bal & ((1u << lane) - 1))] = j;
                cbase += __popc(bal);
            }
        return total;
    };
    // pivots of a panel by one warp over its candidates: S.p, S.pm, S.bits,
    // S.srow and the pivots' tags
    auto select_warp = [&](const u64 *ysp, int ncand) {
        u64 pmk;
        int kk;
        if (ncand <= 64)
            kk = warp_select<2>(S.cand, ncand, ysp, tag, S.bits, S.srow, &pmk);
        else if (ncand <= 128)
            kk = warp_select<4>(S.cand, ncand, ysp, tag, S.bits, S.srow, &pmk);
        else if (ncand <= 192)
            kk = warp_select<6>(S.cand, ncand, ysp, tag, S.bits, S.srow, &pmk);
        else if (ncand <= 256)
            kk = warp_select<8>(S.cand, ncand, ysp, tag, S.bits, S.srow, &pmk);
        else
            kk = warp_select<12>(S.cand, ncand, ysp, tag, S.bits, S.srow, &pmk);
        if (lane == 0) {
            S.p = kk;
            S.pm = pmk;
        }
    };
    // words [x_begin, wc) of every row that is not one of the panel's pivots
    // (or of the rows listed in ul) take the reduced rows of the pivot bits
    // its panel word holds: 16 nibble-table lookups per word, TW words at a
    // time.  wfirst 0: by every warp; wfirst 1: by the warps other than 0 and
    // 4 (warp 0 selects meanwhile; warp 4 shares its scheduler), with a named
    // barrier among them.
    auto update_words = [&](u64 pmask, const u64 *ysp, int x_begin, int wfirst, const int *ul, int nul) {
        const int nw = wfirst ? kWarps - 2 : kWarps, nthr = 32 * nw;
        const int wq = wfirst ? (warp < 4 ? warp - 1 : warp - 2) : warp, t0 = 32 * wq + lane;
        auto bar = [&]() {
            if (wfirst == 0)
                __syncthreads();
            else
                asm volatile("bar.sync %0, %1;" ::"r"(kSubBar), "r"(nthr) : "memory");
        };
        for (int x0 = x_begin; x0 < wc; x0 += TW) {
            for (int e = t0; e < 16 * 5 * TW; e += nthr) {
                const int t = e % TW, gh = e / TW, gi = gh / 5, h = gh % 5;
                if (h == 4) {
                    S.T[gi][0][t] = 0;
                    continue;
                }
                const int bb = 4 * gi + h, x = x0 + t;
                u64 v = 0;
                if (((pmask >> bb) & 1) && x < wc) v = Rbuf[(size_t)bb * wc + x];
                S.T[gi][1 << h][t] = v;
            }
            bar();
            for (int h = 1; h < 4; ++h) {
                const int cnt = (1 << h) - 1;
                for (int e = t0; e < 16 * cnt * TW; e += nthr) {
                    const int t = e % TW, rest = e / TW, gi = rest / cnt, v = (1 << h) + 1 + rest % cnt;
                    S.T[gi][v][t] = S.T[gi][v - (1 << h)][t] ^ S.T[gi][1 << h][t];
                }
                bar();
            }
            // lane (h, xl) = (lane / TW, lane % TW) takes word x0 + xl of
            // rows j0 + 4 h .. + 3 (32 / TW rows per warp instruction); the
            // next rows' words are read while the current ones are combined
            constexpr int RPW = 32 / TW;
            const int kStep = nw * 4 * RPW;
            const int xl = lane % TW, hsel = lane / TW;
            const int x = x0 + xl;
            // rows jb .. jb + 3 (or list entries jb .. jb + 3): their indices,
            // coefficient words (0: skip) and matrix words
            const int nrows = ul ? nul : m;
            auto fetch = [&](int jb, int (&jr)[4], u64 (&y)[4], u64 (&a)[4]) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int i = jb + q;
                    jr[q] = i < nrows ? (ul ? ul[i] : i) : -1;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    y[q] = (jr[q] >= 0 && x < wc && (ul || active[jr[q]] != 2)) ? ysp[jr[q]] & pmask : 0ull;
#pragma unroll
                for (int q = 0; q < 4; ++q) a[q] = y[q] ? A[(size_t)jr[q] * wc + x] : 0ull;
            };
            int jb = wq * 4 * RPW + 4 * hsel;
            if (ul) {
                // listed rows (all to update): their words two steps ahead;
                // coefficient words read from shared memory at use
                auto load = [&](int j0, int (&jr)[4], u64 (&a)[4]) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) jr[q] = (j0 + q < nul && x < wc) ? ul[j0 + q] : -1;
#pragma unroll
                    for (int q = 0; q < 4; ++q) a[q] = jr[q] >= 0 ? A[(size_t)jr[q] * wc + x] : 0ull;
                };
                int j0r[4], j1r[4];
                u64 a0[4], a1[4];
                load(jb, j0r, a0);
                load(jb + kStep, j1r, a1);
                for (; jb - 4 * hsel < nul; jb += kStep) {
                    int j2r[4];
                    u64 a2[4];
                    load(jb + 2 * kStep, j2r, a2);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        if (j0r[q] < 0) continue;
                        const u64 yq = ysp[j0r[q]] & pmask;
                        u64 acc = 0;
#pragma unroll
                        for (int gi = 0; gi < 16; ++gi) acc ^= S.T[gi][(yq >> (4 * gi)) & 15][xl];
                        A[(size_t)j0r[q] * wc + x] = a0[q] ^ acc;
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        j0r[q] = j1r[q];
                        a0[q] = a1[q];
                        j1r[q] = j2r[q];
                        a1[q] = a2[q];
                    }
                }
                bar();
                continue;
            }
            int jr[4];
            u64 y[4], a[4];
            fetch(jb, jr, y, a);
            for (; jb - 4 * hsel < nrows; jb += kStep) {
                int jn[4];
                u64 yn[4], an[4];
                fetch(jb + kStep, jn, yn, an);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (!y[q]) continue;
                    u64 acc = 0;
#pragma unroll
                    for (int gi = 0; gi < 16; ++gi) acc ^= S.T[gi][(y[q] >> (4 * gi)) & 15][xl];
                    A[(size_t)jr[q] * wc + x] = a[q] ^ acc;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    jr[q] = jn[q];
                    y[q] = yn[q];
                    a[q] = an[q];
                }
            }
            bar();
        }
    };

    int r = 0;
    for (int w = 0; w < wc && r < m; ++w) {
        u64 *ysnap = cur ? ysnap1 : ysnap0, *yv = cur ? ysnap0 : ysnap1;
        int k = 0;
        u64 pmask = 0;
        if (have_sel) {
            // selected during the previous panel's update, pivots marked
            k = S.p;
            pmask = S.pm;
        } else {
            // 1. panel words and the per-warp candidate counts
            int ncand = 0;
            for (int j0 = jlo; j0 < jhi; j0 += 128) {
                u64 word[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int j = j0 + 32 * u + lane;
                    word[u] = j < jhi ? A[(size_t)j * wc + w] : 0ull;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int j = j0 + 32 * u + lane;
                    bool ok = false;
                    if (j < jhi) {
                        ysnap[j] = word[u];
                        ok = word[u] != 0 && active[j] == 1;
                    }
                    ncand += __popc(__ballot_sync(0xffffffffu, ok));
                }
            }
            if (lane == 0) S.wcnt[warp] = ncand;
            __syncthreads();
            ncand = compact(ysnap);
            if (ncand <= kCandMax) {
                // 2. pivots by one warp over the candidates (few rows hold a
                // bit of the panel in a sparse matrix)
                __syncthreads();
                if (warp == 0) select_warp(ysnap, ncand);
                __syncthreads();
                k = S.p;
                pmask = S.pm;
                for (int q = tid; q < k; q += NT) active[S.srow[q]] = 2;
                __syncthreads();
            } else if (m <= kRegRows * kRegThreads) {
                // 2. the panel in registers of the first eight warps: thread l
                // holds rows l + 256 i.  Per bit one named barrier: each warp
                // publishes its lowest unused row holding the bit (index, panel
                // word and tag); the lowest of the eight is the pivot.
                if (tid < kRegThreads) {
                    u64 y[kRegRows], t[kRegRows];
                    u32 unused = 0;
#pragma unroll
                    for (int i = 0; i < kRegRows; ++i) {
                        const int j = tid + kRegThreads * i;
                        const int a = j < m ? active[j] : 0;
                        y[i] = a == 1 ? ysnap[j] : 0ull;
                        t[i] = 0;
                        unused |= (a == 1 ? 1u : 0u) << i;
                    }
#pragma unroll
                    for (int half = 0; half < 2; ++half) {
                        for (int bb = 0; bb < 32; ++bb) {
                            const int b = 32 * half + bb;
                            u32 cm = 0;
#pragma unroll
                            for (int i = 0; i < kRegRows; ++i) cm |= (((u32)(y[i] >> (32 * half)) >> bb) & 1u) << i;
                            cm &= unused;
                            const int ib = __ffs((int)cm) - 1;
                            const unsigned jb = ib >= 0 ? (unsigned)(tid + kRegThreads * ib) : (unsigned)INT_MAX;
                            const unsigned wm = __reduce_min_sync(0xffffffffu, jb);
                            const int par = bb & 1;
                            if (jb == wm && wm != (unsigned)INT_MAX) {
                                S.pub[par][warp][0] = sel4r(y, ib);
                                S.pub[par][warp][1] = sel4r(t, ib);
                            }
                            if (lane == 0) S.wmin[par][warp] = wm;
                            asm volatile("bar.sync %0, %1;" ::"r"(kRegBar), "r"(kRegThreads) : "memory");
                            const uint4 wa = reinterpret_cast<const uint4 *>(S.wmin[par])[0];
                            const uint4 wb = reinterpret_cast<const uint4 *>(S.wmin[par])[1];
                            const unsigned pm = min(min(min(wa.x, wa.y), min(wa.z, wa.w)),
                                                    min(min(wb.x, wb.y), min(wb.z, wb.w)));
                            if (pm == (unsigned)INT_MAX) continue;  // no unused row holds bit b
                            const int pr = (int)pm, pw = (pr & (kRegThreads - 1)) >> 5;
                            const u64 yp = S.pub[par][pw][0], tp = S.pub[par][pw][1] ^ (1ull << k);
                            if (tid == 0) {
                                S.bits[k] = b;
                                S.srow[k] = pr;
                            }
                            // every other row holding bit b takes the pivot row (branch-free)
                            const int own = (pr & (kRegThreads - 1)) == tid ? pr / kRegThreads : -1;
#pragma unroll
                            for (int i = 0; i < kRegRows; ++i) {
                                const u64 hit = i == own ? 0ull : 0ull - (u64)(((u32)(y[i] >> (32 * half)) >> bb) & 1u);
                                y[i] ^= yp & hit;
                                t[i] ^= tp & hit;
                            }
                            if (own >= 0) unused &= ~(1u << own);
                            pmask |= 1ull << b;
                            ++k;
                        }
                    }
#pragma unroll
                    for (int i = 0; i < kRegRows; ++i) {
                        const int j = tid + kRegThreads * i;
                        if (j < m) tag[j] = t[i];
                    }
                    if (tid == 0) {
                        S.p = k;
                        S.pm = pmask;
                    }
                }
                __syncthreads();
                k = S.p;
                pmask = S.pm;
                for (int q = tid; q < k; q += NT) active[S.srow[q]] = 2;
                __syncthreads();
            } else {
                // 1. panel words, pivot search for bit 0
                if (tid < 3) S.slots[tid] = INT_MAX;
                __syncthreads();
                unsigned best = INT_MAX;
                for (int j = tid; j < m; j += NT) {
                    const u64 word = A[(size_t)j * wc + w];
                    ysnap[j] = word;
                    const u64 y = active[j] == 1 ? word : 0ull;
                    yv[j] = y;
                    tag[j] = 0;
                    if ((y & 1ull) && best == (unsigned)INT_MAX) best = j;
                }
                best = __reduce_min_sync(0xffffffffu, best);
                if (lane == 0 && best != (unsigned)INT_MAX) atomicMin(&S.slots[0], (int)best);
                __syncthreads();
                // 2. per-bit elimination of the panel words with combination tags
                for (int b = 0; b < 64; ++b) {
                    const int p = S.slots[b % 3];
                    if (tid == 0) S.slots[(b + 2) % 3] = INT_MAX;
                    if (p != INT_MAX) {
                        const u64 yp = yv[p], tp = tag[p] ^ (1ull << k);
                        if (tid == 0) {
                            S.bits[k] = b;
                            S.srow[k] = p;
                        }
                        if (p % NT == tid) active[p] = 2;
                        const u64 bit = 1ull << b;
                        for (int j = tid; j < m; j += NT) {
                            if (j == p || active[j] == 0) continue;
                            if (yv[j] & bit) {
                                yv[j] ^= yp;
                                tag[j] ^= tp;
                            }
                        }
                        pmask |= bit;
                        ++k;
                    }
                    if (b < 63) {
                        const u64 bit = 1ull << (b + 1);
                        best = INT_MAX;
                        for (int j = tid; j < m; j += NT)
                            if (active[j] == 1 && (yv[j] & bit)) {
                                best = j;
                                break;
                            }
                        best = __reduce_min_sync(0xffffffffu, best);
                        if (lane == 0 && best != (unsigned)INT_MAX) atomicMin(&S.slots[(b + 1) % 3], (int)best);
                    }
                    __syncthreads();
                }
            }
        }
        have_sel = false;
        const int p = k;
        if (p == 0) continue;
        for (int t = tid; t < p; t += NT) {
            S.coef[t] = tag[S.srow[t]] ^ (1ull << t);
            piv[r + t] = 64 * w + S.bits[t];
            prow[r + t] = S.srow[t];
            S.prev_srow[t] = S.srow[t];
        }
        const int rem = wc - w;
        // 3. reduced pivot rows from the staged original rows (Rbuf row b:
        // the reduced row of the pivot on bit b)
        __syncthreads();
        {
            constexpr int U = 8;
            for (int e0 = tid; e0 < p * rem; e0 += U * NT) {
                u64 v[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int e = e0 + u * NT;
                    v[u] = e < p * rem ? A[(size_t)S.srow[e / rem] * wc + w + e % rem] : 0ull;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int e = e0 + u * NT;
                    if (e < p * rem) stage[(size_t)(e / rem) * wc + w + e % rem] = v[u];
                }
            }
        }
        __syncthreads();
        for (int e = tid; e < p * rem; e += NT) {
            const int kk = e / rem, x = w + e % rem;
            u64 c = S.coef[kk], v = 0;
            while (c) {
                const int i = ctz64_(c);
                c &= c - 1;
                v ^= stage[(size_t)i * wc + x];
            }
            Rbuf[(size_t)S.bits[kk] * wc + x] = v;
            A[(size_t)S.srow[kk] * wc + x] = v;
        }
        __syncthreads();
        // 4. update every other row (the reduced rows of the pivot bits its
        // panel word holds)
        const bool la = lookahead_ok && w + 1 < wc && r + p < m;
        if (!la) {
            update_words(pmask, ysnap, w, 0, nullptr, 0);
            for (int t = tid; t < p; t += NT) active[S.srow[t]] = 0;
            r += p;
            __syncthreads();
            continue;
        }
        // 4a. look-ahead: words w and w + 1 of every row first (one-word
        // tables), the new word w + 1 being the next panel's snapshot
        u64 *ysn = yv;
        u64(*T01)[16][16] = reinterpret_cast<u64(*)[16][16]>(stage);
        for (int e = tid; e < 2 * 16 * 16; e += NT) {
            const int which = e >> 8, gi = (e >> 4) & 15, v = e & 15;
            u64 acc = 0;
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const int bb = 4 * gi + h;
                if (((v >> h) & 1) && ((pmask >> bb) & 1)) acc ^= Rbuf[(size_t)bb * wc + w + which];
            }
            T01[which][gi][v] = acc;
        }
        __syncthreads();
        int nc = 0, nu = 0;
        u32 ub[4] = {0u, 0u, 0u, 0u};  // which rows of the warp's first 128 to update
        for (int j0 = jlo; j0 < jhi; j0 += 128) {
            u64 a1[4];
            int st[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int j = j0 + 32 * u + lane;
                st[u] = j < jhi ? active[j] : 0;
                a1[u] = j < jhi ? A[(size_t)j * wc + w + 1] : 0ull;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int j = j0 + 32 * u + lane;
                bool ok = false, upd = false;
                if (j < jhi) {
                    const u64 y = st[u] != 2 ? ysnap[j] & pmask : 0ull;
                    if (y) {
                        u64 acc0 = 0, acc1 = 0;
#pragma unroll
                        for (int gi = 0; gi < 16; ++gi) {
                            const int nib = (int)(y >> (4 * gi)) & 15;
                            acc0 ^= T01[0][gi][nib];
                            acc1 ^= T01[1][gi][nib];
                        }
                        A[(size_t)j * wc + w] = ysnap[j] ^ acc0;
                        a1[u] ^= acc1;
                        A[(size_t)j * wc + w + 1] = a1[u];
                    }
                    ysn[j] = a1[u];
                    ok = a1[u] != 0 && st[u] == 1;
                    upd = y != 0;
                }
                nc += __popc(__ballot_sync(0xffffffffu, ok));
                const u32 bu = __ballot_sync(0xffffffffu, upd);
                nu += __popc(bu);
                if (j0 == jlo) ub[u] = bu;
            }
        }
        if (lane == 0) {
            S.wcnt[warp] = nc;
            S.ucnt[warp] = nu;
        }
        __syncthreads();
        const int ncn = compact(ysn);
        // the rows to update, in row order
        int nul = 0;
        if (ulist) {
            int ubase = 0;
            for (int q = 0; q < kWarps; ++q) {
                const int c = S.ucnt[q];
                ubase += q < warp ? c : 0;
                nul += c;
            }
            if (chunk <= 128) {
                // from the ballots kept during the pass above
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if ((ub[u] >> lane) & 1u) ulist[ubase + __popc(ub[u] & ((1u << lane) - 1))] = jlo + 32 * u + lane;
                    ubase += __popc(ub[u]);
                }
            } else {
                for (int j0 = jlo; j0 < jhi; j0 += 32) {
                    const int j = j0 + lane;
                    const bool upd = j < jhi && active[j] != 2 && (ysnap[j] & pmask) != 0;
                    const u32 bal = __ballot_sync(0xffffffffu, upd);
                    if (upd) ulist[ubase + __popc(bal & ((1u << lane) - 1))] = j;
                    ubase += __popc(bal);
                }
            }
        }
        __syncthreads();
        if (ncn <= kCandMax) {
            // 4b. the next panel's pivots by warp 0 while the other warps
            // (but warp 4, which shares warp 0's scheduler) update words
            // w + 2 .. of this one
            if (warp == 0)
                select_warp(ysn, ncn);
            else if (warp != 4)
                update_words(pmask, ysnap, w + 2, 1, ulist, nul);
            __syncthreads();
            for (int t = tid; t < p; t += NT) active[S.prev_srow[t]] = 0;
            const int kn = S.p;
            for (int t = tid; t < kn; t += NT) active[S.srow[t]] = 2;
            have_sel = true;
            cur ^= 1;
        } else {
            update_words(pmask, ysnap, w + 2, 0, ulist, nul);
            for (int t = tid; t < p; t += NT) active[S.prev_srow[t]] = 0;
        }
        r += p;
        __syncthreads();
    }
    if (fo) {
        for (long long e = tid; e < (long long)m * wc; e += NT) {
            const int rr = (int)(e / wc), x = (int)(e - (long long)rr * wc);
            fo->M[(long long)rr * fo->ldm + x] = A[e];
        }
        for (int t = tid; t < r; t += NT) {
            fo->piv[t] = piv[t];
            fo->prow[t] = prow[t];
        }
        if (tid == 0) *fo->rank = r;
        __syncthreads();
        return;
    }
    if (tid == 0) ranks[item] = r;

    // ---- null basis
    const int f = n - r;
    // its index arrays in the elimination's shared memory when they fit
    if ((size_t)wc * 8 + ((size_t)r + 2 * (size_t)n + wc + 1) * 4 <= pre_a_bytes) {
        __syncthreads();
        u64 *pm_s = reinterpret_cast<u64 *>(extra);
        int *prow_s = reinterpret_cast<int *>(pm_s + wc);
        for (int t = tid; t < r; t += NT) prow_s[t] = prow[t];
        pm = pm_s;
        prow = prow_s;
        cmap = prow_s + r;
        fcol = cmap + n;
        pbase = fcol + n;
    }
    for (int W = tid; W < wc; W += NT) pm[W] = 0;
    for (int c = tid; c < n; c += NT) cmap[c] = -1;
    __syncthreads();
    for (int t = tid; t < r; t += NT) {
        atomicOr(&pm[piv[t] >> 6], 1ull << (piv[t] & 63));
        cmap[piv[t]] = t;
    }
    __syncthreads();
    if (tid == 0) {
        int pc = 0;
        for (int W = 0; W < wc; ++W) {
            pbase[W] = pc;
            pc += __popcll(pm[W]);
        }
        pbase[wc] = pc;
    }
    __syncthreads();
    // free columns: word W's free bits go to ranks [64W - pbase[W], ...)
    for (int W = tid; W < wc; W += NT) {
        const int valid = n - 64 * W;
        const u64 vm = valid >= 64 ? ~0ull : ((1ull << valid) - 1);
        u64 fm = ~pm[W] & vm;
        int fc = 64 * W - pbase[W];
        while (fm) {
            const int c = 64 * W + ctz64_(fm);
            fcol[fc] = c;
            cmap[c] = -(fc + 1);
            ++fc;
            fm &= fm - 1;
        }
    }
    __syncthreads();
    if (f == 0) return;
    // row pitches of Rt and Q: multiples of 4 words (their scratch is laid out so)
    const int rt32 = ((r + 127) >> 7) << 2, q32 = ((f + 127) >> 7) << 2;
    if (r > 0) {
        // Rt (n x r) = R^T, R row p = A[prow[p]]
        const u32 *A32 = reinterpret_cast<const u32 *>(A);
        if ((wc & 1) == 0 && (reinterpret_cast<uintptr_t>(A) & 15) == 0)
            cta_transpose4<NT, 16, 4>([&](int row, int xg) { return tr_words4(A32 + ((size_t)prow[row] * wc + 2 * xg) * 2); },
                                      r, n, Rt, rt32, rt32);
        else
            cta_transpose4<NT, 16, 2>([&](int row, int xg) { return tr_words2(A32 + ((size_t)prow[row] * wc + xg) * 2); },
                                      r, n, Rt, rt32, rt32);
        __syncthreads();
        // Q (r x f) = (rows f_i of Rt)^T: row p = RREF row p at the free columns
        cta_transpose4<NT, 16, 4>([&](int row, int xg) { return tr_words4(Rt + (long long)fcol[row] * rt32 + 4 * xg); },
                                  f, r, Q, q32, q32);
        __syncthreads();
    }
    // Zt (f x n) = Y^T, Y row c = Q row p (pivot column c) or e_i (free column i)
    u64 *Z = zt + it.z_off;
    u32 *Z32 = reinterpret_cast<u32 *>(Z);
    if ((n & 63) && (n & 63) <= 32)
        for (int i = tid; i < f; i += NT) Z32[(long long)i * 2 * wc + 2 * wc - 1] = 0;
    auto yrow = [&](int c, int yg) -> TrWords<4> {
        const int mc = cmap[c];
        if (mc >= 0) return tr_words4(Q + (long long)mc * q32 + 4 * yg);
        const int fi = -mc - 1;  // the unit row of free index fi
        TrWords<4> u{{0u, 0u, 0u, 0u}};
#pragma unroll
        for (int h = 0; h < 4; ++h)
            if ((fi >> 5) == 4 * yg + h) u.w[h] = 1u << (fi & 31);
        return u;
    };
    // 16-byte stores where the rows of Zt are 16-byte aligned (even word count)
    if ((wc & 1) == 0 && (reinterpret_cast<uintptr_t>(Z32) & 15) == 0)
        cta_transpose4<NT, 16, 4>(yrow, n, f, Z32, 2LL * wc, (n + 31) >> 5);
    else
        cta_transpose4<NT, 8, 4>(yrow, n, f, Z32, 2LL * wc, (n + 31) >> 5);
    __syncthreads();
}

// NT threads and SMEM bytes of shared memory per CTA, kThreads / NT CTAs per
// SM: a big matrix takes a whole CTA, a medium one a 128-thread group with
// kMidBudget bytes, a small one a warp with kSmallBudget bytes.
template <int NT, int SMEM>
__global__ void __launch_bounds__(NT, kThreads / NT)
batch_kernel(const BatchDevItem *__restrict__ items, const int *__restrict__ order, int n_big,
             int n_mid, int n_small, int *counters, const u64 *__restrict__ in, u64 *__restrict__ zt,
             long long *ranks, u64 *gscratch, long long gscratch_words)
{
    static_assert((NT / kMidGroup) * kMidBudget <= SMEM && (NT / 32) * kSmallBudget <= SMEM,
                  "group regions");
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_next[NT / 32];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    u64 *gmat = gscratch + (long long)blockIdx.x * gscratch_words;

    // big: the whole CTA per matrix
    while (true) {
        if (tid == 0) s_next[0] = atomicAdd(&counters[0], 1);
        __syncthreads();
        const int k = s_next[0];
        __syncthreads();
        if (k >= n_big) break;
        const int item = order[k];
        process_big_blocked<NT, SMEM>(items[item], in, zt, ranks, item, smem, gmat);
    }
    // mid: groups of 128 threads, each with kMidBudget bytes of shared memory
    {
        const int g = tid / kMidGroup, gtid = tid % kMidGroup;
        unsigned char *region = smem + (size_t)g * kMidBudget;
        while (true) {
            if (gtid == 0) s_next[g] = atomicAdd(&counters[1], 1);
            asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(kMidGroup) : "memory");
            const int k = s_next[g];
            asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(kMidGroup) : "memory");
            if (k >= n_mid) break;
            const int item = order[n_big + k];
            process_matrix<kMidGroup>(items[item], in, zt, ranks, item, region, nullptr, gtid, 1 + g);
        }
    }
    __syncthreads();
    // small: one warp per matrix
    {
        unsigned char *region = smem + (size_t)warp * kSmallBudget;
        while (true) {
            int k = 0;
            if (lane == 0) k = atomicAdd(&counters[2], 1);
            k = __shfl_sync(0xffffffffu, k, 0);
            if (k >= n_small) break;
            const int item = order[n_big + n_mid + k];
            process_matrix<32>(items[item], in, zt, ranks, item, region, nullptr, lane, 0);
        }
    }
}

// Logical <-> packed tiles: a block covers one word column (64 columns) of
// up to kPackRows rows of one matrix (tile_mat names the matrix; tile -
// tile_start[matrix] = row chunk * wc + word).  In the column-major logical
// layout each column's rows are contiguous, so the block reads 64 runs of up
// to kPackRows bytes.
constexpr int kPackRows = 512;                   // rows per tile: 32 lanes x 16 rows
constexpr int kPackPieces = kPackRows / 16 + 1;  // 16-byte pieces covering a run at any alignment
constexpr int kPackPitch = kPackPieces * 16;     // bytes per staged run (528)

// bit 7 of each byte of x set where that byte is nonzero
__device__ __forceinline__ u32 byte_nonzero_hi(u32 x)
{
    return (((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x) & 0x80808080u;
}

// the 16 bytes starting at byte s (0..15) of the 32 bytes p:q
__device__ __forceinline__ void realign16(const uint4 &p, const uint4 &q, int s, u32 (&x)[4])
{
    u32 w0, w1, w2, w3, w4;
    switch (s >> 2) {
    case 0: w0 = p.x; w1 = p.y; w2 = p.z; w3 = p.w; w4 = q.x; break;
    case 1: w0 = p.y; w1 = p.z; w2 = p.w; w3 = q.x; w4 = q.y; break;
    case 2: w0 = p.z; w1 = p.w; w2 = q.x; w3 = q.y; w4 = q.z; break;
    default: w0 = p.w; w1 = q.x; w2 = q.y; w3 = q.z; w4 = q.w; break;
    }
    const int sh = 8 * (s & 3);
    x[0] = __funnelshift_r(w0, w1, sh);
    x[1] = __funnelshift_r(w1, w2, sh);
    x[2] = __funnelshift_r(w2, w3, sh);
    x[3] = __funnelshift_r(w3, w4, sh);
}

// logical column-major inputs -> packed rows, for every matrix of the batch.
//  1. staging: the 64 column runs land in shared memory by 16-byte cp.async
//     copies from 16-byte aligned addresses (each run keeps its offset s
//     within its first piece; pieces past the run are zero-filled);
//  2. gather: warp o takes columns 8o .. 8o + 7, lane l rows 16l .. 16l + 15:
//     per column two 16-byte shared reads realigned by s give 16 row bytes,
//     and for 0/1 bytes one shift-add per 4 bytes puts column c's bit at
//     bit c % 8 of each row's byte (a lane that saw any other byte value
//     recomputes with the exact nonzero test);
//  3. a 4 x 4 byte transpose (byte_perm) turns the 8 octet bytes of a row
//     into its 64-bit packed word, one store per row.
__global__ void __launch_bounds__(256, 6) batch_pack_kernel(const BatchDevItem *__restrict__ items,
                                                            const long long *byte_off,
                                                            const long long *tile_start,
                                                            const int *__restrict__ tile_mat,
                                                            const unsigned char *__restrict__ in,
                                                            long long total, u64 *__restrict__ out)
{
    // 34 KB, so that six CTAs share an SM
    __shared__ __align__(16) unsigned char col[64][kPackPitch];
    __shared__ int off[64];
    const long long b = blockIdx.x;
    const int lo = tile_mat[b];
    const BatchDevItem it = items[lo];
    const long long tile = b - tile_start[lo];
    const int wc = (it.n + 63) >> 6;
    const int rc = (int)(tile / wc), w = (int)(tile % wc);
    const int r0 = rc * kPackRows;
    const int rows = (it.m - r0) < kPackRows ? (it.m - r0) : kPackRows;
    const int cols = (it.n - w * 64) < 64 ? (it.n - w * 64) : 64;
    const long long base = byte_off[lo] + (long long)w * 64 * it.m + r0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned long long ib = reinterpret_cast<unsigned long long>(in);
    // 1. staging: a warp per run (runs warp, warp + 8, ...), lane l piece l
    //    (lanes 0-7 also piece 32 of runs warp + 8 * lane)
    auto stage = [&](int c, int q) {
        const unsigned long long ga = ib + (unsigned long long)(base + (long long)c * it.m);
        const int s = (int)(ga & 15);
        const int need = (s + rows + 15) >> 4;
        const long long a = (long long)(ga & ~15ULL) - (long long)ib + 16LL * q;  // piece offset in the input
        unsigned char *dst = &col[c][16 * q];
        if (q < need && a >= 0 && a + 16 <= total) {
            const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(in + a) : "memory");
        } else {
            u32 v[4] = {0u, 0u, 0u, 0u};
            if (q < need) {
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (a + i >= 0 && a + i < total) v[i >> 2] |= (u32)in[a + i] << (8 * (i & 3));
            }
            *reinterpret_cast<uint4 *>(dst) = make_uint4(v[0], v[1], v[2], v[3]);
        }
    };
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int c = warp + 8 * i;
        if (c < cols) stage(c, lane);
    }
    if (lane < 8 && warp + 8 * lane < cols) stage(warp + 8 * lane, kPackPieces - 1);
    if (lane == 0) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int c = warp + 8 * i;
            if (c < cols) off[c] = (int)((ib + (unsigned long long)(base + (long long)c * it.m)) & 15);
        }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    // 2. gather
    u32 acc[4] = {0u, 0u, 0u, 0u};
    u32 bad = 0;
#pragma unroll
    for (int cc = 0; cc < 8; ++cc) {
        const int c = 8 * warp + cc;
        if (c < cols) {
            const uint4 p = *reinterpret_cast<const uint4 *>(&col[c][16 * lane]);
            const uint4 q = *reinterpret_cast<const uint4 *>(&col[c][16 * lane + 16]);
            u32 x[4];
            realign16(p, q, off[c], x);
            bad |= x[0] | x[1] | x[2] | x[3];
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[k] += x[k] << cc;
        }
    }
    if (bad & 0xFEFEFEFEu) {  // bytes other than 0 and 1: nonzero -> 1
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] = 0u;
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
            const int c = 8 * warp + cc;
            if (c < cols) {
                const uint4 p = *reinterpret_cast<const uint4 *>(&col[c][16 * lane]);
                const uint4 q = *reinterpret_cast<const uint4 *>(&col[c][16 * lane + 16]);
                u32 x[4];
                realign16(p, q, off[c], x);
#pragma unroll
                for (int k = 0; k < 4; ++k) acc[k] |= byte_nonzero_hi(x[k]) >> (7 - cc);
            }
        }
    }
    // byte r of oct(o) = row r's bits for columns 8o .. 8o + 7; warp o has
    // read only its own runs 8o .. 8o + 7, so oct(o) overwrites run 8o
    __syncwarp();
    *reinterpret_cast<uint4 *>(&col[8 * warp][16 * lane]) = make_uint4(acc[0], acc[1], acc[2], acc[3]);
    __syncthreads();
    // 3. thread t < 128 writes rows 4t .. 4t + 3
    const int t = threadIdx.x;
    if (t < kPackRows / 4 && 4 * t < rows) {
        u32 o[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) o[i] = reinterpret_cast<const u32 *>(col[8 * i])[t];
        u32 lo4[4], hi4[4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const u32 *v = o + 4 * h;
            u32 *r = h ? hi4 : lo4;
            const u32 t0 = __byte_perm(v[0], v[1], 0x5140), t1 = __byte_perm(v[0], v[1], 0x7362);
            const u32 t2 = __byte_perm(v[2], v[3], 0x5140), t3 = __byte_perm(v[2], v[3], 0x7362);
            r[0] = __byte_perm(t0, t2, 0x5410);
            r[1] = __byte_perm(t0, t2, 0x7632);
            r[2] = __byte_perm(t1, t3, 0x5410);
            r[3] = __byte_perm(t1, t3, 0x7632);
        }
        u64 *dst = out + it.in_off + (long long)(r0 + 4 * t) * wc + w;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (4 * t + k < rows) dst[(long long)k * wc] = ((u64)hi4[k] << 32) | lo4[k];
    }
}

// packed rows -> logical column-major inputs, for every matrix of the batch
// (same tiles; thread t writes the 64 bytes of rows t, t + 256, ...)
__global__ void __launch_bounds__(256) batch_unpack_kernel(const BatchDevItem *__restrict__ items,
                                                           const long long *byte_off,
                                                           const long long *tile_start,
                                                           const int *__restrict__ tile_mat,
                                                           const u64 *__restrict__ in,
                                                           unsigned char *__restrict__ out)
{
    const long long b = blockIdx.x;
    const int lo = tile_mat[b];
    const BatchDevItem it = items[lo];
    const long long tile = b - tile_start[lo];
    const int wc = (it.n + 63) >> 6;
    const int rc = (int)(tile / wc), w = (int)(tile % wc);
    const int r0 = rc * kPackRows;
    const int rows = (it.m - r0) < kPackRows ? (it.m - r0) : kPackRows;
    const int cols = (it.n - w * 64) < 64 ? (it.n - w * 64) : 64;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
        const u64 word = in[it.in_off + (long long)(r0 + r) * wc + w];
        unsigned char *p = out + byte_off[lo] + (long long)w * 64 * it.m + r0 + r;
        for (int j = 0; j < cols; ++j) p[(long long)j * it.m] = (unsigned char)((word >> j) & 1);
    }
}

// ---------------------------------------------------------------- single matrix
// RREF of one matrix by one CTA in one launch: in shared memory by the
// column-by-column engine when it fits, else by the blocked engine over
// global scratch.  Reads the packed matrix M (row pitch ldm, any pitch >=
// ceil(n/64)) and writes the RREF rows back over it.
__global__ void __launch_bounds__(kThreads, 1)
fused_elim_kernel(BatchDevItem it, const u64 *__restrict__ in_compact, FusedOut fo, u64 *scratch)
{
    extern __shared__ __align__(16) unsigned char smem[];
    if (it.flags & 1)
        process_matrix<kThreads>(it, in_compact, nullptr, nullptr, 0, smem, nullptr, threadIdx.x, 0, &fo);
    else
        process_big_blocked<kThreads, kSmemTotal>(it, in_compact, nullptr, nullptr, 0, smem, scratch, &fo);
}

size_t fused_workspace(i64 m, i64 n)
{
    const i64 wc = words_of(n);
    // compact copy of the input (pitch ceil(n/64)) + big-engine scratch
    return (size_t)(m * wc + big_scratch_words(m, n)) * 8;
}

mela_status launch_fused_elim(u64 *M, i64 ld, i64 m, i64 n, long long *d_rank, long long *d_piv,
                              long long *d_prow, void *ws, size_t ws_bytes, cudaStream_t s)
{
    if (m > INT_MAX / 2 || n > INT_MAX / 2) {
        set_error("fused elimination: matrix too large");
        return MELA_ERR_UNSUPPORTED;
    }
    const size_t need = fused_workspace(m, n);
    if (ws_bytes < need || !ws) {
        set_error("fused elimination workspace of %zu bytes needed, %zu given", need, ws_bytes);
        return MELA_ERR_INVALID;
    }
    const i64 wc = words_of(n);
    u64 *compact = (u64 *)ws;
    u64 *scratch = compact + m * wc;
    MELA_CUDA_TRY(cudaMemcpy2DAsync(compact, (size_t)wc * 8, M, (size_t)ld * 8, (size_t)wc * 8, (size_t)m,
                                    cudaMemcpyDeviceToDevice, s));
    BatchDevItem it{};
    it.m = (int)m;
    it.n = (int)n;
    it.in_off = 0;
    it.z_off = 0;
    const size_t aux = aux_bytes((int)m, (int)n);
    const size_t mat = (size_t)m * smem_ld((int)n) * 8;
    it.flags = (aux + mat <= (size_t)kSmemTotal) ? 1 : 0;
    FusedOut fo{M, ld, d_rank, d_piv, d_prow};
    MELA_CUDA_TRY(cudaFuncSetAttribute(fused_elim_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kSmemTotal));
    fused_elim_kernel<<<1, kThreads, kSmemTotal, s>>>(it, compact, fo, scratch);
    MELA_LAUNCH_CHECK("fused_elim_kernel");
    return MELA_OK;
}

// ---------------------------------------------------------------- host side
struct BatchPlanImpl {
    int count = 0, n_big = 0, n_mid = 0, n_small = 0;
    BatchDevItem *d_items = nullptr;
    int *d_order = nullptr;
    int *d_counters = nullptr;
    u64 *d_gscratch = nullptr;
    long long gscratch_words = 0;
    int grid = 0;
    // logical-input path
    long long *d_byte_off = nullptr, *d_tile_start = nullptr;
    int *d_tile_mat = nullptr;  // matrix of each packing tile
    long long pack_tiles = 0;
    long long logical_total = 0;  // bytes of the logical input
    u64 *d_packed = nullptr;
    long long packed_words = 0;
    // CUDA graph of the last run
    cudaGraphExec_t exec = nullptr;
    const void *g_in = nullptr;
    void *g_zt = nullptr, *g_ranks = nullptr;
    int g_logical = -1;
    cudaStream_t cap_stream = nullptr;  // private stream the graph is captured on
    // statistics
    long long class_count[3] = {0, 0, 0};
};

static mela_status plan_free(BatchPlanImpl *P)
{
    if (!P) return MELA_OK;
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->cap_stream) cudaStreamDestroy(P->cap_stream);
    cudaFree(P->d_items);
    cudaFree(P->d_order);
    cudaFree(P->d_counters);
    cudaFree(P->d_gscratch);
    cudaFree(P->d_byte_off);
    cudaFree(P->d_tile_start);
    cudaFree(P->d_tile_mat);
    cudaFree(P->d_packed);
    delete P;
    return MELA_OK;
}

// Engine per matrix.  policy -1: by fit and size (the fixed rule below);
// 0/1/2: that engine wherever the matrix fits its region; -2: the installed
// cost model's cheapest engine among those the matrix fits, given its shape,
// its density and the batch mix (matrix count, mean log2(m*n)) -- the fixed
// rule when no model is installed.
static mela_status plan_create(const mela_batch_item *h, long long count, int force_class,
                               const double *densities, BatchPlanImpl **out)
{
    *out = nullptr;
    if (count < 0 || (count > 0 && !h) || count > INT_MAX) {
        set_error("batch: bad item list");
        return MELA_ERR_INVALID;
    }
    const bool learned = force_class == -2 && costmodel_loaded();
    double mix = 0.0;
    if (learned) {
        for (long long i = 0; i < count; ++i) {
            const double cells = (double)h[i].m * (double)h[i].n;
            mix += std::log2(cells > 1 ? cells : 1);
        }
        mix /= (double)(count ? count : 1);
    }
    BatchPlanImpl *P = new BatchPlanImpl();
    P->count = (int)count;
    std::vector<BatchDevItem> items((size_t)count);
    std::vector<int> cls((size_t)count);
    std::vector<double> cost((size_t)count);
    long long max_big_words = 0;
    for (long long i = 0; i < count; ++i) {
        const long long m = h[i].m, n = h[i].n;
        if (m < 0 || n < 0 || m > INT_MAX / 2 || n > INT_MAX / 2 || h[i].in_offset < 0 || h[i].z_offset < 0) {
            plan_free(P);
            set_error("batch: item %lld has a bad shape or offset", i);
            return MELA_ERR_INVALID;
        }
        BatchDevItem d{};
        d.m = (int)m;
        d.n = (int)n;
        d.in_off = h[i].in_offset;
        d.z_off = h[i].z_offset;
        const size_t aux = aux_bytes((int)m, (int)n);
        const size_t mat = (size_t)m * smem_ld((int)n) * 8;
        // Class by fit and size: with two CTAs per SM the blocked CTA engine
        // beats the 128-thread column engine from m = 240 up (parity-check
        // matrices, n = 2m: 7% faster at m in [230, 300), 23% at [380, 460)),
        // and the column engine beats a warp from m = 160 up.
        int c;
        if (aux + mat <= (size_t)kSmallBudget && m <= kSmallMaxRows) c = 2;
        else if (aux + mat <= (size_t)kMidBudget && m < kMidMaxRows) c = 1;
        else c = 0;
        if (force_class >= 0 && force_class <= 2) {
            // a forced class must still fit its region; otherwise fall back to big
            const size_t budget = force_class == 2 ? kSmallBudget : force_class == 1 ? kMidBudget : kSmemTotal;
            if (force_class == 0 || aux + mat <= budget) c = force_class;
        } else if (learned) {
            float y[MELA_MLP_OUT];
            const double dens = densities ? densities[i] : 0.5;
            if (costmodel_predict(MELA_OP_BATCH, (double)m, (double)n, 0.0, dens, (double)count, mix, y)) {
                c = 0;
                if (aux + mat <= (size_t)kMidBudget && y[1] < y[c]) c = 1;
                if (aux + mat <= (size_t)kSmallBudget && y[2] < y[c]) c = 2;
            }
        }
        if (c == 0) {
            d.flags = 0;  // big matrices live in the CTA's global scratch
            max_big_words = std::max(max_big_words, big_scratch_words(m, n));
        } else {
            d.flags = 1;
        }
        items[(size_t)i] = d;
        cls[(size_t)i] = c;
        cost[(size_t)i] = (double)m * (double)n * (double)((n + 63) / 64);
        P->class_count[c]++;
    }
    std::vector<int> order((size_t)count);
    for (int i = 0; i < (int)count; ++i) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        if (cls[(size_t)a] != cls[(size_t)b]) return cls[(size_t)a] < cls[(size_t)b];
        return cost[(size_t)a] > cost[(size_t)b];
    });
    P->n_big = (int)P->class_count[0];
    P->n_mid = (int)P->class_count[1];
    P->n_small = (int)P->class_count[2];
    P->grid = (kThreads / kBatchThreads) * sm_count();
    P->gscratch_words = max_big_words;

    // logical-input packing tiles
    std::vector<long long> byte_off((size_t)count), tiles((size_t)count);
    long long boff = 0, t = 0;
    for (long long i = 0; i < count; ++i) {
        byte_off[(size_t)i] = boff;
        boff += h[i].m * h[i].n;
        tiles[(size_t)i] = t;
        const long long wc = (h[i].n + 63) / 64;
        t += ((h[i].m + kPackRows - 1) / kPackRows) * wc;
        P->packed_words = std::max(P->packed_words, h[i].in_offset + h[i].m * wc);
    }
    P->pack_tiles = t;
    P->logical_total = boff;
    std::vector<int> tile_mat((size_t)(t > 0 ? t : 1), 0);
    for (long long i = 0; i < count; ++i) {
        const long long end = i + 1 < count ? tiles[(size_t)i + 1] : t;
        for (long long q = tiles[(size_t)i]; q < end; ++q) tile_mat[(size_t)q] = (int)i;
    }

    auto dmal = [&](void **p, size_t bytes) -> mela_status {
        cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
        if (e != cudaSuccess) return cuda_status(e, "cudaMalloc (batch plan)");
        return MELA_OK;
    };
    mela_status st;
    if ((st = dmal((void **)&P->d_items, items.size() * sizeof(BatchDevItem))) != MELA_OK ||
        (st = dmal((void **)&P->d_order, order.size() * sizeof(int))) != MELA_OK ||
        (st = dmal((void **)&P->d_counters, 4 * sizeof(int))) != MELA_OK ||
        (st = dmal((void **)&P->d_gscratch, (size_t)P->grid * (size_t)max_big_words * 8)) != MELA_OK ||
        (st = dmal((void **)&P->d_byte_off, byte_off.size() * 8)) != MELA_OK ||
        (st = dmal((void **)&P->d_tile_start, tiles.size() * 8)) != MELA_OK ||
        (st = dmal((void **)&P->d_tile_mat, tile_mat.size() * 4)) != MELA_OK) {
        plan_free(P);
        return st;
    }
    cudaMemcpy(P->d_items, items.data(), items.size() * sizeof(BatchDevItem), cudaMemcpyHostToDevice);
    cudaMemcpy(P->d_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(P->d_byte_off, byte_off.data(), byte_off.size() * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(P->d_tile_start, tiles.data(), tiles.size() * 8, cudaMemcpyHostToDevice);
    cudaError_t e = cudaMemcpy(P->d_tile_mat, tile_mat.data(), tile_mat.size() * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        plan_free(P);
        return cuda_status(e, "batch plan upload");
    }
    *out = P;
    return MELA_OK;
}

static mela_status enqueue(BatchPlanImpl *P, const u64 *in, u64 *zt, long long *ranks, cudaStream_t s)
{
    MELA_CUDA_TRY(cudaMemsetAsync(P->d_counters, 0, 4 * sizeof(int), s));
    if (P->count == 0) return MELA_OK;
    batch_kernel<kBatchThreads, kBatchSmem><<<P->grid, kBatchThreads, kBatchSmem, s>>>(
        P->d_items, P->d_order, P->n_big, P->n_mid, P->n_small, P->d_counters, in, zt, ranks,
        P->d_gscratch, P->gscratch_words);
    MELA_LAUNCH_CHECK("batch_kernel");
    return MELA_OK;
}

static mela_status enqueue_logical(BatchPlanImpl *P, const unsigned char *in, u64 *zt, long long *ranks,
                                   cudaStream_t s)
{
    if (P->count && P->pack_tiles) {
        batch_pack_kernel<<<(unsigned)P->pack_tiles, 256, 0, s>>>(P->d_items, P->d_byte_off,
                                                                   P->d_tile_start, P->d_tile_mat, in,
                                                                   P->logical_total, P->d_packed);
        MELA_LAUNCH_CHECK("batch_pack_kernel");
    }
    return enqueue(P, P->d_packed, zt, ranks, s);
}

// Dynamic shared memory limit of the batch kernel, once per device (and
// before any stream capture).
static mela_status batch_attrs()
{
    static bool done[64] = {};
    int dev = 0;
    MELA_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || done[dev]) return MELA_OK;
    MELA_CUDA_TRY(cudaFuncSetAttribute(batch_kernel<kBatchThreads, kBatchSmem>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kBatchSmem));
    done[dev] = true;
    return MELA_OK;
}

static mela_status run(BatchPlanImpl *P, const void *in, int logical, u64 *zt, long long *ranks,
                       cudaStream_t s, int use_graph)
{
    {
        const mela_status st = batch_attrs();
        if (st != MELA_OK) return st;
    }
    if (logical && !P->d_packed) {
        cudaError_t e = cudaMalloc((void **)&P->d_packed, (size_t)(P->packed_words ? P->packed_words : 1) * 8);
        if (e != cudaSuccess) return cuda_status(e, "cudaMalloc (batch packed buffer)");
    }
    if (!use_graph) {
        return logical ? enqueue_logical(P, (const unsigned char *)in, zt, ranks, s)
                       : enqueue(P, (const u64 *)in, zt, ranks, s);
    }
    if (!P->exec || P->g_in != in || P->g_zt != zt || P->g_ranks != ranks ||
        P->g_logical != logical) {
        if (P->exec) {
            cudaGraphExecDestroy(P->exec);
            P->exec = nullptr;
        }
        // Captured on a private stream (the caller's may be the legacy default
        // stream, which cannot be captured); launched on the caller's stream.
        if (!P->cap_stream) MELA_CUDA_TRY(cudaStreamCreateWithFlags(&P->cap_stream, cudaStreamNonBlocking));
        const cudaStream_t cs = P->cap_stream;
        cudaGraph_t g;
        MELA_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        mela_status st = logical ? enqueue_logical(P, (const unsigned char *)in, zt, ranks, cs)
                                 : enqueue(P, (const u64 *)in, zt, ranks, cs);
        cudaError_t e = cudaStreamEndCapture(cs, &g);
        if (st != MELA_OK) return st;
        if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&P->exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate");
        P->g_in = in;
        P->g_zt = zt;
        P->g_ranks = ranks;
        P->g_logical = logical;
    }
    MELA_CUDA_TRY(cudaGraphLaunch(P->exec, s));
    return MELA_OK;
}

}  // namespace mela

using namespace mela;

struct mela_batch_plan {
    BatchPlanImpl *impl;
};

extern "C" mela_status mela_batch_plan_create(const mela_batch_item *items, int64_t count,
                                              int32_t force_class, mela_batch_plan **plan)
{
    return mela_batch_plan_create_ex(items, count, nullptr, force_class, plan);
}

extern "C" mela_status mela_batch_plan_create_ex(const mela_batch_item *items, int64_t count,
                                                 const double *densities, int32_t policy,
                                                 mela_batch_plan **plan)
{
    if (!plan) {
        set_error("null plan pointer");
        return MELA_ERR_INVALID;
    }
    *plan = nullptr;
    if (policy < -2 || policy > 2) {
        set_error("batch: engine policy %d (-2 .. 2)", policy);
        return MELA_ERR_INVALID;
    }
    BatchPlanImpl *P = nullptr;
    mela_status st = plan_create(items, count, policy, densities, &P);
    if (st != MELA_OK) return st;
    *plan = new mela_batch_plan{P};
    return MELA_OK;
}

namespace mela {
// d_counts[i] += ones of item i (one CTA per item, grid-stride over items).
static __global__ void __launch_bounds__(256)
batch_popcount_kernel(const mela_batch_item *items, long long count, const u64 *in, long long *counts)
{
    for (long long i = blockIdx.x; i < count; i += gridDim.x) {
        const mela_batch_item it = items[i];
        const long long wc = (it.n + 63) / 64, total = it.m * wc;
        const u64 last = (it.n & 63) ? ((1ull << (it.n & 63)) - 1) : ~0ull;
        unsigned long long c = 0;
        for (long long e = threadIdx.x; e < total; e += blockDim.x) {
            u64 v = in[it.in_offset + e];
            if (e % wc == wc - 1) v &= last;
            c += __popcll(v);
        }
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if ((threadIdx.x & 31) == 0 && c) atomicAdd((unsigned long long *)&counts[i], c);
    }
}
}  // namespace mela

extern "C" mela_status mela_batch_popcounts(const mela_batch_item *items, int64_t count, const uint64_t *d_in,
                                            int64_t *d_counts, void *stream)
{
    if (count < 0 || (count > 0 && (!items || !d_in || !d_counts))) {
        set_error("mela_batch_popcounts: bad arguments");
        return MELA_ERR_INVALID;
    }
    if (count == 0) return MELA_OK;
    for (int64_t i = 0; i < count; ++i) {
        if (items[i].m < 0 || items[i].n < 0 || items[i].in_offset < 0) {
            set_error("mela_batch_popcounts: item %lld has a bad shape or offset", (long long)i);
            return MELA_ERR_INVALID;
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    DevBuf d_items;
    mela_status st = d_items.alloc((size_t)count * sizeof(mela_batch_item), s);
    if (st != MELA_OK) return st;
    MELA_CUDA_TRY(cudaMemcpyAsync(d_items.p, items, (size_t)count * sizeof(mela_batch_item),
                                  cudaMemcpyHostToDevice, s));
    MELA_CUDA_TRY(cudaMemsetAsync(d_counts, 0, (size_t)count * 8, s));
    const long long grid = count < (long long)sm_count() * 16 ? count : (long long)sm_count() * 16;
    batch_popcount_kernel<<<(unsigned)grid, 256, 0, s>>>((const mela_batch_item *)d_items.p, count,
                                                         (const u64 *)d_in, (long long *)d_counts);
    MELA_LAUNCH_CHECK("batch_popcount_kernel");
    return MELA_OK;  // the item copy is released on s, after the kernel
}

extern "C" void mela_batch_plan_destroy(mela_batch_plan *plan)
{
    if (!plan) return;
    plan_free(plan->impl);
    delete plan;
}

extern "C" mela_status mela_batch_plan_stats(const mela_batch_plan *plan, int64_t *big, int64_t *mid,
                                             int64_t *small)
{
    if (!plan) return MELA_ERR_INVALID;
    if (big) *big = plan->impl->class_count[0];
    if (mid) *mid = plan->impl->class_count[1];
    if (small) *small = plan->impl->class_count[2];
    return MELA_OK;
}

extern "C" mela_status mela_batch_rank_null(mela_batch_plan *plan, const uint64_t *d_in,
                                            uint64_t *d_zt, int64_t *d_ranks, int32_t use_graph,
                                            void *stream)
{
    if (!plan || (plan->impl->count && (!d_in || !d_zt || !d_ranks))) {
        set_error("mela_batch_rank_null: null argument");
        return MELA_ERR_INVALID;
    }
    return run(plan->impl, d_in, 0, (u64 *)d_zt, (long long *)d_ranks, (cudaStream_t)stream, use_graph);
}

extern "C" mela_status mela_batch_unpack_logical(mela_batch_plan *plan, const uint64_t *d_packed,
                                                 uint8_t *d_logical, void *stream)
{
    if (!plan || (plan->impl->count && (!d_packed || !d_logical))) {
        set_error("mela_batch_unpack_logical: null argument");
        return MELA_ERR_INVALID;
    }
    BatchPlanImpl *P = plan->impl;
    if (P->count && P->pack_tiles) {
        batch_unpack_kernel<<<(unsigned)P->pack_tiles, 256, 0, (cudaStream_t)stream>>>(
            P->d_items, P->d_byte_off, P->d_tile_start, P->d_tile_mat, (const u64 *)d_packed, d_logical);
        MELA_LAUNCH_CHECK("batch_unpack_kernel");
    }
    return MELA_OK;
}

extern "C" mela_status mela_batch_pack_logical(mela_batch_plan *plan, const uint8_t *d_logical,
                                               uint64_t *d_packed, void *stream)
{
    if (!plan || (plan->impl->count && (!d_logical || !d_packed))) {
        set_error("mela_batch_pack_logical: null argument");
        return MELA_ERR_INVALID;
    }
    BatchPlanImpl *P = plan->impl;
    if (P->count && P->pack_tiles) {
        batch_pack_kernel<<<(unsigned)P->pack_tiles, 256, 0, (cudaStream_t)stream>>>(
            P->d_items, P->d_byte_off, P->d_tile_start, P->d_tile_mat, d_logical, P->logical_total,
            (u64 *)d_packed);
        MELA_LAUNCH_CHECK("batch_pack_kernel");
    }
    return MELA_OK;
}

extern "C" mela_status mela_batch_rank_null_logical(mela_batch_plan *plan, const uint8_t *d_in,
                                                    uint64_t *d_zt, int64_t *d_ranks,
                                                    int32_t use_graph, void *stream)
{
    if (!plan || (plan->impl->count && (!d_in || !d_zt || !d_ranks))) {
        set_error("mela_batch_rank_null_logical: null argument");
        return MELA_ERR_INVALID;
    }
    return run(plan->impl, d_in, 1, (u64 *)d_zt, (long long *)d_ranks, (cudaStream_t)stream, use_graph);
}
