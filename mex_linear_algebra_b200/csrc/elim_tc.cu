// elim_tc.cu -- blocked GF(2) elimination whose trailing (Schur) update runs
// on the sm_100a tensor cores.
//
// Results are those of the other forms (elim.cu): the rank of
// bitrank_packed / rank_m4ri (src/mela_rank_gf2.c:27-121,
// src/mela_rank_m4ri.c:94-279), the greedy pivot columns and the unique RREF
// rows of gf2_rref_standard (src/mela_null_gf2.c:88-131).  Rows never move:
// pivot t lives in physical row prow[t].
//
// One window of 256 columns (4 words) at a time:
//   window_factor   one CTA.  Walks the list of active rows in chunks of 320.
//                   Each row's window part is reduced by the basis found so
//                   far (reduced row echelon, lowest set bit leading) through
//                   64 tables of the 16 combinations of 4 basis vectors; the
//                   rows left nonzero are eliminated among themselves by a
//                   CTA-wide Gauss-Jordan (a thread per row, one barrier per
//                   pivot: the next pivot is the row with the lowest leading
//                   bit, found by a warp min-reduction and a shared-memory
//                   atomicMin); the older basis vectors are then reduced by the
//                   new ones.  Every basis vector carries its combination
//                   ("tag") over the rows P_j that entered the basis, so
//                   R_window = T * A[P, window].  The walk stops as soon as the
//                   basis spans every column of the window.  The walked part of
//                   the list is then compacted in place (pivot rows and rows
//                   found zero from the window on are dropped, order kept).
//   window_combine  R_t = sum_j T[t][j] A[P_j] over the words from the window
//                   on, into the panel buffer (a block per 4 words, 4-bit
//                   tables over the P rows).
//   window_coef     every other row to update (rank: the active rows; RREF: all
//                   rows) whose bits at the window's pivot columns are not all
//                   zero gets a slot; those bits become a row of 0/1 bytes.
//   window_rt       R transposed as 0/1 bytes, Rt8[j][t] = bit j of R_t, and
//                   R_t written over row P_t.
//   tc_update       A[row(slot), w..] ^= parity(X8[slot] . Rt8^T): tcgen05
//                   kind::i8 128 x 256 tiles with K = 256.  A persistent CTA
//                   keeps a 256-column strip of Rt8 in shared memory and
//                   streams 128-row tiles of X8 through a 4-stage ring into two
//                   TMEM accumulators; sixteen epilogue warps XOR the parity
//                   bits into the packed rows while the next tile is
//                   multiplied, and flag the rows that are still nonzero.
// Since the basis is reduced, a row's coefficient for R_t is its own bit at
// pivot column t, and XORing sum_t x_t R_t clears every pivot column of the
// window; a row whose window part lies in the basis' span (every active row,
// once the scan has ended) is then zero across the window.
#include <climits>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "mela_common.cuh"
#include "mela_internal.h"
#include "mela_host.h"
#include "elim.h"
#include "tc_ptx.cuh"

namespace mela {

namespace {

constexpr int WW = 4;         // words per window
constexpr int WBITS = 256;    // columns per window
constexpr int WF_THREADS = 320;  // a chunk of rows; 320 random rows span 256 columns but with probability 2^-64

struct WinState {
    long long rank;         // pivots so far (every window)
    int rt;                 // pivots of the current window
    int nu;                 // rows to update in the current window
    int na;                 // rows in the active-row list
    int lbase;              // the list is list[lbase .. lbase + na)
    u64 have[WW];           // window-relative pivot columns
    int prow[WBITS];        // physical row of P-index j
    u64 tag[WBITS][WW];     // pivot t (ascending column): R_t = sum_j bit j * A[prow[j]]
};

struct WfSmem {
    u64 bd[WBITS][WW];        // basis vector whose leading bit is b
    u64 bt[WBITS][WW];        // its tag
    u64 tab[64][16][WW];      // nibble tables of the basis
    u64 tabt[64][16][WW];     // the same over the tags
    u64 cx[WF_THREADS][WW];   // rows of the current chunk (residual)
    u64 ct[WF_THREADS][WW];   //   and their tags
    int newslot[WBITS];       // chunk slot of the k-th new basis vector
    int newlead[WBITS];       //   and its leading bit
    int prow[WBITS];          // physical row of P-index j
    u64 have[WW];
    unsigned keys[3];         // smallest key, rotating by iteration
    int nb, cnt;
    int wsum[32];
};

__device__ __forceinline__ int ctz64w(u64 x) { return __ffsll((long long)x) - 1; }

// Word q of a 4-word vector held in registers (selects, no local memory).
__device__ __forceinline__ u64 sel4(const u64 (&v)[WW], int q)
{
    return q == 0 ? v[0] : (q == 1 ? v[1] : (q == 2 ? v[2] : v[3]));
}
__device__ __forceinline__ bool bit_of(const u64 (&v)[WW], int b) { return (sel4(v, b >> 6) >> (b & 63)) & 1; }
__device__ __forceinline__ void or_word(u64 (&v)[WW], int q, u64 x)
{
#pragma unroll
    for (int i = 0; i < WW; ++i) v[i] |= (i == q) ? x : 0ull;
}
__device__ __forceinline__ void xor4s(u64 (&a)[WW], const u64 *b)
{
#pragma unroll
    for (int q = 0; q < WW; ++q) a[q] ^= b[q];
}
__device__ __forceinline__ bool any4(const u64 (&v)[WW]) { return (v[0] | v[1] | v[2] | v[3]) != 0; }


// Exclusive position of this thread's flag among the block's flags (thread
// order) and the block total; every thread of the block must call it.
__device__ __forceinline__ int block_slot(bool flag, int *wsum, int &total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned bal = __ballot_sync(0xffffffffu, flag);
    if (lane == 0) wsum[warp] = __popc(bal);
    __syncthreads();
    if (warp == 0) {
        int v = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, off);
            if (lane >= off) v += u;
        }
        wsum[lane] = v;
    }
    __syncthreads();
    total = wsum[31];
    const int slot = (warp ? wsum[warp - 1] : 0) + __popc(bal & ((1u << lane) - 1));
    __syncthreads();  // wsum may be rewritten by the next call
    return slot;
}

}  // namespace

// ---------------------------------------------------------------- window_factor
__global__ void __launch_bounds__(WF_THREADS, 1)
window_factor_kernel(const u64 *__restrict__ M, i64 ld, i64 m, i64 n, i64 w, int *list, const unsigned char *live,
                     unsigned char *state, int *stamp, int wid, const WinState *prev, WinState *ws, long long *piv,
                     long long *prow)
{
    extern __shared__ __align__(16) unsigned char wf_raw[];
    WfSmem &S = *reinterpret_cast<WfSmem *>(wf_raw);
    const int tid = threadIdx.x, lane = tid & 31;
    const i64 wc = words_of(n);
    const int wn = (wc - w) < WW ? (int)(wc - w) : WW;
    const i64 vb = n - 64 * w;
    const int valid = vb < WBITS ? (int)vb : WBITS;  // columns of this window inside the matrix
    const int na = prev->na;
    int *L0 = list + prev->lbase;
    constexpr unsigned NOKEY = 0xFFFFFFFFu;

    for (int e = tid; e < 64 * 16 * WW; e += WF_THREADS) {
        (&S.tab[0][0][0])[e] = 0;
        (&S.tabt[0][0][0])[e] = 0;
    }
    if (tid < WW) S.have[tid] = 0;
    if (tid == 0) S.nb = 0;
    __syncthreads();

    int walked = 0;
    for (int base = 0; base < na; base += WF_THREADS) {
        if (S.nb >= valid) break;
        walked = base + WF_THREADS < na ? base + WF_THREADS : na;
        const int nb0 = S.nb;
        u64 hv[WW];
#pragma unroll
        for (int q = 0; q < WW; ++q) hv[q] = S.have[q];
        const int k = base + tid;
        int row = -1;
        u64 x[WW] = {0, 0, 0, 0};
        if (k < na) {
            row = L0[k];
#pragma unroll
            for (int q = 0; q < WW; ++q)
                if (q < wn) x[q] = M[(i64)row * ld + w + q];
        }
        u64 cx[WW] = {x[0], x[1], x[2], x[3]}, ct[WW] = {0, 0, 0, 0};
        if (any4(x) && nb0) {
#pragma unroll
            for (int g = 0; g < 64; ++g) {
                const int q = g >> 4, sh = 4 * (g & 15);
                const u64 hn = (hv[q] >> sh) & 15;
                if (hn) {
                    const int nib = (int)((x[q] >> sh) & hn);
                    if (nib) xor4s(cx, S.tab[g][nib]);
                }
            }
            if (any4(cx)) {
#pragma unroll
                for (int g = 0; g < 64; ++g) {
                    const int q = g >> 4, sh = 4 * (g & 15);
                    const u64 hn = (hv[q] >> sh) & 15;
                    if (hn) {
                        const int nib = (int)((x[q] >> sh) & hn);
                        if (nib) xor4s(ct, S.tabt[g][nib]);
                    }
                }
            }
        }
        // Gauss-Jordan among the chunk's residual rows, a pivot per barrier,
        // one 64-column word of the window at a time.  A row's key is
        // (leading bit, slot); the next pivot is the smallest key.  Inside
        // word q every unused row is zero in the words before q, so its key
        // comes from word q alone and a pivot row is XORed in from word q on;
        // word q is done once no unused row has a bit left there.  Only the
        // row holding its warp's smallest key publishes itself to shared
        // memory, its tag already carrying the P-index it would enter as, so
        // the pivot is always published.
        bool used = false;
        int myj = -1;
        unsigned key = NOKEY;
        auto publish = [&](unsigned *kslot, int jn) {
            const unsigned mk = __reduce_min_sync(0xffffffffu, key);
            if (key == mk && key != NOKEY) {
                ulonglong2 *dv = reinterpret_cast<ulonglong2 *>(S.cx[tid]);
                ulonglong2 *dt = reinterpret_cast<ulonglong2 *>(S.ct[tid]);
                const u64 e = 1ull << (jn & 63);
                const int jq = jn >> 6;
                dv[0] = make_ulonglong2(cx[0], cx[1]);
                dv[1] = make_ulonglong2(cx[2], cx[3]);
                dt[0] = make_ulonglong2(ct[0] ^ (jq == 0 ? e : 0ull), ct[1] ^ (jq == 1 ? e : 0ull));
                dt[1] = make_ulonglong2(ct[2] ^ (jq == 2 ? e : 0ull), ct[3] ^ (jq == 3 ? e : 0ull));
            }
            if (lane == 0 && mk != NOKEY) atomicMin(kslot, mk);
        };
        int nnew = 0;
#pragma unroll
        for (int q = 0; q < WW; ++q) {
            if (nb0 + nnew >= valid) break;  // uniform
            key = (!used && cx[q]) ? ((unsigned)(64 * q + ctz64w(cx[q])) << 10 | (unsigned)tid) : NOKEY;
            __syncthreads();  // the previous word's last keys have been read
            if (tid < 3) S.keys[tid] = NOKEY;
            __syncthreads();
            publish(&S.keys[0], nb0 + nnew);
            __syncthreads();
            int kr = 0;  // slot holding this iteration's key
            for (;;) {
                const unsigned kk = S.keys[kr];
                if (kk == NOKEY || nb0 + nnew >= valid) break;
                const int kn = kr == 2 ? 0 : kr + 1, kz = kn == 2 ? 0 : kn + 1;
                if (tid == 0) S.keys[kz] = NOKEY;  // read last in the previous iteration
                const int p = (int)(kk & 1023u), L = (int)(kk >> 10);
                if (tid == p) {
                    used = true;
                    myj = nb0 + nnew;
                    key = NOKEY;
                    S.newslot[nnew] = p;
                    S.newlead[nnew] = L;
                    S.prow[myj] = row;
                } else if ((cx[q] >> (L & 63)) & 1) {
                    const u64 *pv = S.cx[p];
                    const ulonglong2 *pt = reinterpret_cast<const ulonglong2 *>(S.ct[p]);
                    const ulonglong2 t0 = pt[0], t1 = pt[1];
#pragma unroll
                    for (int qq = q; qq < WW; ++qq) cx[qq] ^= pv[qq];
                    ct[0] ^= t0.x;
                    ct[1] ^= t0.y;
                    ct[2] ^= t1.x;
                    ct[3] ^= t1.y;
                    if (!used) key = cx[q] ? ((unsigned)(64 * q + ctz64w(cx[q])) << 10 | (unsigned)tid) : NOKEY;
                }
                ++nnew;
                publish(&S.keys[kn], nb0 + nnew);
                kr = kn;
                __syncthreads();
            }
        }
        __syncthreads();  // every key is read before the next chunk publishes
        if (nnew == 0) continue;  // uniform
        if (used) {
            ct[0] ^= (myj >> 6) == 0 ? (1ull << (myj & 63)) : 0ull;
            ct[1] ^= (myj >> 6) == 1 ? (1ull << (myj & 63)) : 0ull;
            ct[2] ^= (myj >> 6) == 2 ? (1ull << (myj & 63)) : 0ull;
            ct[3] ^= (myj >> 6) == 3 ? (1ull << (myj & 63)) : 0ull;
#pragma unroll
            for (int q = 0; q < WW; ++q) {
                S.cx[tid][q] = cx[q];
                S.ct[tid][q] = ct[q];
            }
        }
        __syncthreads();
        // older basis vectors: clear the new leading bits (the new vectors are
        // reduced among themselves and zero at the older leads)
        if (nb0 && tid < WBITS && ((S.have[tid >> 6] >> (tid & 63)) & 1)) {
            u64 v[WW], t[WW];
#pragma unroll
            for (int q = 0; q < WW; ++q) {
                v[q] = S.bd[tid][q];
                t[q] = S.bt[tid][q];
            }
            const u64 ov[WW] = {v[0], v[1], v[2], v[3]};
            for (int e = 0; e < nnew; ++e) {
                if (bit_of(ov, S.newlead[e])) {
                    xor4s(v, S.cx[S.newslot[e]]);
                    xor4s(t, S.ct[S.newslot[e]]);
                }
            }
#pragma unroll
            for (int q = 0; q < WW; ++q) {
                S.bd[tid][q] = v[q];
                S.bt[tid][q] = t[q];
            }
        }
        __syncthreads();
        if (tid < nnew) {
            const int Ld = S.newlead[tid], sl = S.newslot[tid];
#pragma unroll
            for (int q = 0; q < WW; ++q) {
                S.bd[Ld][q] = S.cx[sl][q];
                S.bt[Ld][q] = S.ct[sl][q];
            }
        }
        if (tid == 0) {
            for (int e = 0; e < nnew; ++e) S.have[S.newlead[e] >> 6] |= 1ull << (S.newlead[e] & 63);
            S.nb = nb0 + nnew;
        }
        __syncthreads();
        if (S.nb < valid && base + WF_THREADS < na) {
            // tables of the 16 combinations of basis vectors 4g..4g+3
            for (int e = tid; e < 64 * 16; e += WF_THREADS) {
                const int g = e >> 4, v = e & 15;
                u64 a[WW] = {0, 0, 0, 0}, b[WW] = {0, 0, 0, 0};
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const int bb = 4 * g + h;
                    if (((v >> h) & 1) && ((S.have[bb >> 6] >> (bb & 63)) & 1)) {
                        xor4s(a, S.bd[bb]);
                        xor4s(b, S.bt[bb]);
                    }
                }
#pragma unroll
                for (int q = 0; q < WW; ++q) {
                    S.tab[g][v][q] = a[q];
                    S.tabt[g][v][q] = b[q];
                }
            }
            __syncthreads();
        }
    }

    // results: pivot t = t-th leading bit; P-index t is its physical row
    const int nb = S.nb;
    const long long r0 = prev->rank;
    if (tid < WBITS && ((S.have[tid >> 6] >> (tid & 63)) & 1)) {
        int t = 0;
        for (int q = 0; q < (tid >> 6); ++q) t += __popcll(S.have[q]);
        t += __popcll(S.have[tid >> 6] & ((1ull << (tid & 63)) - 1));
#pragma unroll
        for (int q = 0; q < WW; ++q) ws->tag[t][q] = S.bt[tid][q];
        piv[r0 + t] = 64 * w + tid;
    }
    if (tid < nb) {
        const int r = S.prow[tid];
        ws->prow[tid] = r;
        prow[r0 + tid] = r;
        state[r] = 0;
        stamp[r] = wid;
    }
    if (tid < WW) ws->have[tid] = S.have[tid];
    if (tid == 0) S.cnt = walked;
    __syncthreads();
    // compact the walked part [0, walked) of the list to its right end, in
    // order, dropping this window's pivot rows and rows known to be zero from
    // the window on; chunks go from the last to the first, so every write lands
    // at or after the chunk being read
    for (int c0 = ((walked - 1) / WF_THREADS) * WF_THREADS; walked > 0 && c0 >= 0; c0 -= WF_THREADS) {
        const int k = c0 + tid;
        int row = -1;
        if (k < walked) row = L0[k];
        const bool keep = row >= 0 && state[row] && live[row];
        int total;
        const int slot = block_slot(keep, S.wsum, total);
        const int wpos = S.cnt - total;
        if (keep) L0[wpos + slot] = row;
        __syncthreads();
        if (tid == 0) S.cnt = wpos;
        __syncthreads();
    }
    if (tid == 0) {
        ws->rt = nb;
        ws->nu = 0;
        ws->lbase = prev->lbase + S.cnt;  // S.cnt = entries dropped
        ws->na = na - S.cnt;
        ws->rank = r0 + nb;
    }
}

// ---------------------------------------------------------------- window_combine
// Block: CB_W words x every pivot.  R_t = XOR_j T[t][j] A[P_j] is evaluated
// four P-indices at a time from 64 tables of the 16 combinations of P rows
// 4g..4g+3 (restricted to the block's words).
namespace {
constexpr int CB_W = 4;
struct CbSmem {
    u64 tab[64][16][CB_W];  // 32 KB
    u64 rows[WBITS][CB_W];  // the P rows' words
    u64 tag[WBITS][WW];
};
}

__global__ void __launch_bounds__(256)
window_combine_kernel(const u64 *__restrict__ M, i64 ld, i64 wc, i64 w, const WinState *ws,
                      u64 *__restrict__ Rbuf, i64 ldr)
{
    extern __shared__ __align__(16) unsigned char cb_raw[];
    CbSmem &S = *reinterpret_cast<CbSmem *>(cb_raw);
    const int rt = ws->rt;
    if (rt == 0) return;
    const int tid = threadIdx.x;
    const i64 w0 = w + (i64)blockIdx.x * CB_W;
    {
        const int j = tid;  // 256 threads: one P row each
        u64 v[CB_W];
        if (j < rt) {
            const u64 *src = M + (i64)ws->prow[j] * ld + w0;
#pragma unroll
            for (int q = 0; q < CB_W; ++q) v[q] = (w0 + q < wc) ? src[q] : 0ull;
        } else {
#pragma unroll
            for (int q = 0; q < CB_W; ++q) v[q] = 0;
        }
#pragma unroll
        for (int q = 0; q < CB_W; ++q) S.rows[j][q] = v[q];
#pragma unroll
        for (int q = 0; q < WW; ++q) S.tag[j][q] = j < rt ? ws->tag[j][q] : 0ull;
    }
    __syncthreads();
    for (int e = tid; e < 64 * 16; e += 256) {
        const int g = e >> 4, v = e & 15;
        u64 a[CB_W] = {};
#pragma unroll
        for (int h = 0; h < 4; ++h)
            if ((v >> h) & 1) {
#pragma unroll
                for (int q = 0; q < CB_W; ++q) a[q] ^= S.rows[4 * g + h][q];
            }
#pragma unroll
        for (int q = 0; q < CB_W; ++q) S.tab[g][v][q] = a[q];
    }
    __syncthreads();
    // thread: word q = tid % CB_W, pivots t = tid / CB_W + 64 i
    const int q = tid % CB_W;
    for (int t = tid / CB_W; t < rt; t += 256 / CB_W) {
        u64 acc = 0;
#pragma unroll
        for (int qq = 0; qq < WW; ++qq) {
            const u64 tg = S.tag[t][qq];
#pragma unroll
            for (int g = 0; g < 16; ++g) acc ^= S.tab[16 * qq + g][(tg >> (4 * g)) & 15][q];
        }
        if (w0 + q < wc) Rbuf[(i64)t * ldr + (w0 + q - w)] = acc;
    }
}

// ---------------------------------------------------------------- window_coef
// 4 bits -> 4 bytes of 0/1.
__device__ __forceinline__ u32 nib_bytes(u32 v) { return ((v & 15u) * 0x00204081u) & 0x01010101u; }

// Rows to update: rank form, the list of active rows (pivot rows of this
// window already removed); RREF form, every row except this window's pivots.
__global__ void __launch_bounds__(256)
window_coef_kernel(const u64 *__restrict__ M, i64 ld, i64 m, i64 wc, i64 w, const int *__restrict__ list,
                   const int *stamp, int wid, int rref, WinState *ws, int *ulist, unsigned char *X8,
                   unsigned char *live)
{
    if (ws->rt == 0) return;
    u64 hv[WW];
#pragma unroll
    for (int q = 0; q < WW; ++q) hv[q] = ws->have[q];
    const i64 cnt = rref ? m : (i64)ws->na;
    list += ws->lbase;
    const int wn = (wc - w) < WW ? (int)(wc - w) : WW;
    const int lane = threadIdx.x & 31;
    const i64 stride = (i64)gridDim.x * blockDim.x;
    for (i64 i0 = (i64)blockIdx.x * blockDim.x; i0 < cnt; i0 += stride) {
        const i64 idx = i0 + threadIdx.x;
        i64 row = -1;
        if (idx < cnt) {
            row = rref ? idx : (i64)list[idx];
            if (rref && stamp[row] == wid) row = -1;
        }
        u64 xc[WW] = {0, 0, 0, 0};
        if (row >= 0) {
            int pos = 0;
#pragma unroll
            for (int q = 0; q < WW; ++q) {
                const u64 h = hv[q];
                if (q >= wn || !h) continue;
                const u64 x = M[row * ld + w + q];
                u64 e;
                int c;
                if (h == ~0ull) {
                    e = x;
                    c = 64;
                } else {
                    e = 0;
                    c = 0;
                    u64 hh = h;
                    while (hh) {
                        const u64 lb = hh & (~hh + 1);
                        if (x & lb) e |= 1ull << c;
                        ++c;
                        hh ^= lb;
                    }
                }
                const int wq = pos >> 6, sb = pos & 63;
                or_word(xc, wq, e << sb);
                if (sb && sb + c > 64) or_word(xc, wq + 1, e >> (64 - sb));
                pos += c;
            }
        }
        const bool nz = any4(xc);
        const unsigned b = __ballot_sync(0xffffffffu, nz);
        int basepos = 0;
        if (b) {
            if (lane == 0) basepos = atomicAdd(&ws->nu, __popc(b));
            basepos = __shfl_sync(0xffffffffu, basepos, 0);
        }
        if (nz) {
            const int slot = basepos + __popc(b & ((1u << lane) - 1));
            ulist[slot] = (int)row;
            live[row] = 0;  // set again by the update if the row stays nonzero
            uint4 *dst = reinterpret_cast<uint4 *>(X8 + (size_t)slot * WBITS);
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                const u32 bits = (u32)(xc[c >> 2] >> (16 * (c & 3))) & 0xFFFFu;
                dst[c] = make_uint4(nib_bytes(bits), nib_bytes(bits >> 4), nib_bytes(bits >> 8), nib_bytes(bits >> 12));
            }
        }
    }
}

// ---------------------------------------------------------------- window_rt
// Block W (word w + W): Rt8 rows 64W..64W+63 and word w + W of every row P_t.
__global__ void __launch_bounds__(256)
window_rt_kernel(u64 *__restrict__ M, i64 ld, i64 w, const u64 *__restrict__ Rbuf, i64 ldr, const WinState *ws,
                 unsigned char *Rt8)
{
    __shared__ u64 col[WBITS];
    const int rt = ws->rt;
    if (rt == 0) return;
    const int tid = threadIdx.x;
    const i64 W = blockIdx.x;
    const u64 v = tid < rt ? Rbuf[(i64)tid * ldr + W] : 0ull;
    col[tid] = v;
    if (tid < rt) M[(i64)ws->prow[tid] * ld + w + W] = v;
    __syncthreads();
    for (int e = tid; e < 64 * 16; e += 256) {
        const int jl = e >> 4, c = e & 15;
        u32 o[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            u32 x = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) x |= (u32)((col[16 * c + 4 * r + b] >> jl) & 1) << (8 * b);
            o[r] = x;
        }
        *reinterpret_cast<uint4 *>(Rt8 + ((size_t)(W * 64 + jl)) * WBITS + 16 * c) = make_uint4(o[0], o[1], o[2], o[3]);
    }
}

// ---------------------------------------------------------------- tc_update
namespace {
constexpr int UM = 128, UN = 256;             // output tile
constexpr int UBOX = 128;                     // K bytes per TMA box (128-byte swizzle)
constexpr int UA_BOX = UM * UBOX;             // 16 KB
constexpr int UB_BOX = UN * UBOX;             // 32 KB
constexpr int UA_BYTES = 2 * UA_BOX;          // K = 256
constexpr int UB_BYTES = 2 * UB_BOX;
constexpr int U_STAGES = 4;                   // X8 tiles in flight
constexpr int U_BSTAGES = 1;                  // Rt8 strips in shared memory
constexpr int U_STAGE_BYTES = 2 * 2 * UM * 4 * 8;  // per accumulator, two 128-row x 4-word stages
constexpr int U_SMEM = U_BSTAGES * UB_BYTES + U_STAGES * UA_BYTES + U_STAGE_BYTES + 1024 + 256;
constexpr int U_MCH = 8;                      // row tiles per work unit (far part)
constexpr int U_EPI_THREADS = 256;           // warps draining one accumulator: 2 per TMEM lane quarter
constexpr int U_THREADS = 64 + 2 * U_EPI_THREADS;  // and the same for the other accumulator

// bit `pos` of base := bit 0 of src
__device__ __forceinline__ u32 bfi1(u32 src, u32 base, u32 pos)
{
    u32 d;
    asm("bfi.b32 %0, %1, %2, %3, 1;" : "=r"(d) : "r"(src), "r"(base), "r"(pos));
    return d;
}

struct UCtl {
    u64 bfull[U_BSTAGES], bempty[U_BSTAGES];
    u64 afull[U_STAGES], aempty[U_STAGES];
    u64 accfull[2], accempty[2];
    u64 drain;
    u32 tmem;
    int abort;
};

}  // namespace

__global__ void __launch_bounds__(U_THREADS, 1)
tc_update_kernel(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmR,
                 u64 *__restrict__ M, i64 ld, i64 wc, i64 w, const WinState *ws, const int *__restrict__ ulist,
                 unsigned char *live, int strip_lo, int strip_hi, int skip, int mch, u32 *err)
{
    // strips strip_lo .. strip_hi-1 (256 columns each, from the window's first
    // column) except strip `skip` (-1: none); work units of mch row tiles
    const int rt = ws->rt, nu = ws->nu;
    if (rt == 0 || nu == 0) return;
    const i64 lw = wc - w;
    const int s_end = (int)((lw + 3) / 4) < strip_hi ? (int)((lw + 3) / 4) : strip_hi;
    const int strips = s_end - strip_lo - (skip >= strip_lo && skip < s_end ? 1 : 0);
    if (strips <= 0) return;
    auto strip_of = [&](long long vs) -> int {
        const int st = strip_lo + (int)vs;
        return (skip >= 0 && st >= skip) ? st + 1 : st;
    };
    const int mt = (nu + UM - 1) / UM;
    const int chunks = (mt + mch - 1) / mch;
    const long long units = (long long)strips * chunks;
    const long long ub = units * blockIdx.x / gridDim.x, ue = units * (blockIdx.x + 1) / gridDim.x;
    if (ub >= ue) return;

    extern __shared__ unsigned char u_raw[];
    unsigned char *smem =
        reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(u_raw) + 1023) & ~(uintptr_t)1023);
    unsigned char *sB = smem;
    unsigned char *sA = smem + U_BSTAGES * UB_BYTES;
    u64 *stage = reinterpret_cast<u64 *>(sA + U_STAGES * UA_BYTES);  // [acc][2][UM][4]
    UCtl *ctl = reinterpret_cast<UCtl *>(sA + U_STAGES * UA_BYTES + U_STAGE_BYTES);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < U_BSTAGES; ++s) {
            ptx::mbar_init(&ctl->bfull[s], 1);
            ptx::mbar_init(&ctl->bempty[s], 1);
        }
        for (int s = 0; s < U_STAGES; ++s) {
            ptx::mbar_init(&ctl->afull[s], 1);
            ptx::mbar_init(&ctl->aempty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            ptx::mbar_init(&ctl->accfull[a], 1);
            ptx::mbar_init(&ctl->accempty[a], U_EPI_THREADS);
        }
        ptx::mbar_init(&ctl->drain, 1);
        ctl->abort = 0;
        ptx::fence_barrier_init();
    }
    if (warp == 0 && lane == 0) {
        ptx::prefetch_tmap(&tmX);
        ptx::prefetch_tmap(&tmR);
    }
    if (warp == 1) {
        ptx::tmem_alloc(&ctl->tmem, 512);
        ptx::tmem_relinquish();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const u32 tmem = ctl->tmem;
    volatile int *abort_flag = &ctl->abort;

    if (warp == 0) {
        if (lane == 0) {
            // strip loads (nbl) and tile loads (it) in the order the MMA warp consumes them
            int nbl = 0, it = 0, prev_strip = -1;
            int last_a[U_STAGES], last_b[U_BSTAGES];
#pragma unroll
            for (int q = 0; q < U_STAGES; ++q) last_a[q] = -1;
#pragma unroll
            for (int q = 0; q < U_BSTAGES; ++q) last_b[q] = -1;
            bool ok = true;
            for (long long u = ub; u < ue && ok; ++u) {
                const int strip = strip_of(u / chunks), chunk = (int)(u % chunks);
                if (strip != prev_strip) {
                    const int bs = nbl % U_BSTAGES;
                    if (nbl >= U_BSTAGES && !ptx::mbar_wait(&ctl->bempty[bs], ((nbl / U_BSTAGES) - 1) & 1, err)) {
                        ok = false;
                        break;
                    }
                    if (*abort_flag) {
                        ok = false;
                        break;
                    }
                    unsigned char *b = sB + bs * UB_BYTES;
                    ptx::mbar_arrive_expect_tx(&ctl->bfull[bs], UB_BYTES);
                    ptx::tma_load_2d(b, &tmR, &ctl->bfull[bs], 0, strip * UN);
                    ptx::tma_load_2d(b + UB_BOX, &tmR, &ctl->bfull[bs], UBOX, strip * UN);
                    last_b[bs] = nbl / U_BSTAGES;
                    ++nbl;
                    prev_strip = strip;
                }
                const int t1 = (chunk + 1) * mch < mt ? (chunk + 1) * mch : mt;
                for (int tile = chunk * mch; tile < t1; ++tile, ++it) {
                    const int s = it % U_STAGES;
                    if (it >= U_STAGES && !ptx::mbar_wait(&ctl->aempty[s], ((it / U_STAGES) - 1) & 1, err)) {
                        ok = false;
                        break;
                    }
                    if (*abort_flag) {
                        ok = false;
                        break;
                    }
                    unsigned char *a = sA + s * UA_BYTES;
                    ptx::mbar_arrive_expect_tx(&ctl->afull[s], UA_BYTES);
                    ptx::tma_load_2d(a, &tmX, &ctl->afull[s], 0, tile * UM);
                    ptx::tma_load_2d(a + UA_BOX, &tmX, &ctl->afull[s], UBOX, tile * UM);
                    last_a[s] = it / U_STAGES;
                }
            }
            if (!ok) {
                *abort_flag = 1;
                // let every issued copy land before the CTA's shared memory goes away
                for (int s = 0; s < U_BSTAGES; ++s)
                    if (last_b[s] >= 0) ptx::mbar_wait(&ctl->bfull[s], last_b[s] & 1, nullptr);
                for (int s = 0; s < U_STAGES; ++s)
                    if (last_a[s] >= 0) ptx::mbar_wait(&ctl->afull[s], last_a[s] & 1, nullptr);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr u32 idesc = ptx::idesc_i8(UM, UN);
            int nbl = 0, it = 0, prev_strip = -1, bs = 0;
            bool ok = true;
            for (long long u = ub; u < ue && ok; ++u) {
                const int strip = strip_of(u / chunks), chunk = (int)(u % chunks);
                if (strip != prev_strip) {
                    bs = nbl % U_BSTAGES;
                    if (!ptx::mbar_wait(&ctl->bfull[bs], (nbl / U_BSTAGES) & 1, err) || *abort_flag) {
                        ok = false;
                        break;
                    }
                    ++nbl;
                    prev_strip = strip;
                }
                const u32 b0 = ptx::smem_u32(sB + bs * UB_BYTES);
                const int t1 = (chunk + 1) * mch < mt ? (chunk + 1) * mch : mt;
                for (int tile = chunk * mch; tile < t1; ++tile, ++it) {
                    const int s = it % U_STAGES, acc = it & 1;
                    if (!ptx::mbar_wait(&ctl->afull[s], (it / U_STAGES) & 1, err) ||
                        (it >= 2 && !ptx::mbar_wait(&ctl->accempty[acc], ((it >> 1) - 1) & 1, err)) ||
                        *abort_flag) {
                        ok = false;
                        break;
                    }
                    ptx::tc_fence_after();
                    const u32 a0 = ptx::smem_u32(sA + s * UA_BYTES);
                    const u32 d = tmem + (u32)(acc * UN);
#pragma unroll
                    for (int kb = 0; kb < 2; ++kb)
#pragma unroll
                        for (int kk = 0; kk < UBOX / 32; ++kk)
                            ptx::umma_i8(d, ptx::desc_k_sw128(a0 + kb * UA_BOX + kk * 32),
                                         ptx::desc_k_sw128(b0 + kb * UB_BOX + kk * 32), idesc, (kb | kk) != 0);
                    ptx::umma_commit(&ctl->aempty[s]);
                    ptx::umma_commit(&ctl->accfull[acc]);
                }
                if (!ok) break;
                // the strip's buffer is free once this unit's products are done
                const bool next_same = (u + 1 < ue) && (strip_of((u + 1) / chunks) == strip);
                if (!next_same) ptx::umma_commit(&ctl->bempty[bs]);
            }
            if (!ok) {
                *abort_flag = 1;
                ptx::umma_commit(&ctl->drain);
                ptx::mbar_wait(&ctl->drain, 0, nullptr);
            }
        }
        __syncwarp();
    } else {
        // Sixteen warps: for each of the two accumulators (tiles with
        // it % 2 == g), two warps per TMEM lane quarter, one per 128-column
        // half.  A tile's packed parity words go through shared memory, so
        // that the read-modify-write of the rows is done with 32 contiguous
        // bytes per row (4 lanes a row, 8 rows a warp instruction).  The
        // rows' current words for a tile are fetched before the previous
        // tile is drained.
        const int e = warp - 2;
        const int ew = warp & 3;          // TMEM lane quarter of this warp
        const int g = (e >> 2) & 1;       // accumulator
        const int half = e >> 3;          // columns 128*half .. +127 (words 2*half, 2*half+1)
        const int gt = ((e >> 3) << 7) | ((e & 3) << 5) | lane;  // 0..255 within the group
        u64 *gstage = stage + (size_t)g * 2 * UM * 4;
        int it = 0, k = 0;
        bool ok = true;
        // previous own tile
        int p_it = 0;
        i64 p_w0 = 0;
        int p_nw = 0;
        int p_row[2] = {-1, -1};
        u64 p_old[2] = {0, 0};
        // Every warp of the group reaches the group barrier once per tile, on
        // the error path too (a failed wait skips the work, not the barrier).
        auto drain_and_write = [&]() -> bool {
            const int acc = p_it & 1;
            const bool good = !*abort_flag && ptx::mbar_wait(&ctl->accfull[acc], (p_it >> 1) & 1, err);
            if (!good) *abort_flag = 1;
            u32 pb0 = 0, pb1 = 0, pb2 = 0, pb3 = 0;
            if (good) {
                ptx::tc_fence_after();
                const u32 tbase = tmem + ((u32)(ew * 32) << 16) + (u32)(acc * UN + half * 128);
#pragma unroll 1
                for (int h = 0; h < 4; ++h) {
                    u32 r[32];
                    ptx::tmem_ld_32x32b_x32(tbase + (u32)(h * 32), r);
                    ptx::tmem_ld_wait();
                    u32 b = r[0] & 1u;
#pragma unroll
                    for (int j = 1; j < 32; ++j) b = bfi1(r[j], b, (u32)j);
                    pb0 = h == 0 ? b : pb0;
                    pb1 = h == 1 ? b : pb1;
                    pb2 = h == 2 ? b : pb2;
                    pb3 = h == 3 ? b : pb3;
                }
                ptx::tc_fence_before();
                ptx::mbar_arrive(&ctl->accempty[acc]);
            }
            // stage row (ew*32 + lane), words 2*half, 2*half+1
            u64 *st = gstage + (size_t)((k - 1) & 1) * UM * 4 + (size_t)(ew * 32 + lane) * 4 + 2 * half;
            *reinterpret_cast<ulonglong2 *>(st) =
                make_ulonglong2((u64)pb0 | ((u64)pb1 << 32), (u64)pb2 | ((u64)pb3 << 32));
            asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(U_EPI_THREADS) : "memory");
            // items gt and gt + 256: row = item / 4, word = item % 4
            const u64 *sb = gstage + (size_t)((k - 1) & 1) * UM * 4;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int item = gt + 256 * c;
                const int q = item & 3;
                u64 v = 0;
                if (good && p_row[c] >= 0 && q < p_nw) {
                    v = p_old[c] ^ sb[item];
                    M[(i64)p_row[c] * ld + p_w0 + q] = v;
                }
                // one flag per row: the four lanes of a row combine their words
                v |= __shfl_xor_sync(0xffffffffu, v, 1);
                v |= __shfl_xor_sync(0xffffffffu, v, 2);
                if (q == 0 && p_row[c] >= 0 && v) live[p_row[c]] = 1;
            }
            return good;
        };
        for (long long u = ub; u < ue; ++u) {
            const int strip = strip_of(u / chunks), chunk = (int)(u % chunks);
            const i64 w0 = w + (i64)strip * 4;
            const int nw = (wc - w0) < 4 ? (int)(wc - w0) : 4;
            const int t1 = (chunk + 1) * mch < mt ? (chunk + 1) * mch : mt;
            for (int tile = chunk * mch; tile < t1; ++tile, ++it) {
                if ((it & 1) != g) continue;
                // fetch this tile's words (coalesced layout), then finish the previous tile
                int row[2] = {-1, -1};
                u64 old[2] = {0, 0};
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const int item = gt + 256 * c;
                    const int slot = tile * UM + (item >> 2), q = item & 3;
                    if (slot < nu) {
                        row[c] = ulist[slot];
                        if (q < nw) old[c] = M[(i64)row[c] * ld + w0 + q];
                    }
                }
                if (k > 0 && !drain_and_write()) ok = false;
                ++k;
                p_it = it;
                p_w0 = w0;
                p_nw = nw;
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    p_row[c] = row[c];
                    p_old[c] = old[c];
                }
            }
        }
        if (k > 0 && !drain_and_write()) ok = false;
        if (!ok) *abort_flag = 1;
    }

    ptx::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        ptx::tc_fence_after();
        ptx::tmem_dealloc(tmem, 512);
    }
}

// ---------------------------------------------------------------- host side
static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// The first window's list: every row, in order.
__global__ void list_init_kernel(int *list, i64 m, WinState *ws)
{
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < m; i += (i64)gridDim.x * blockDim.x)
        list[i] = (int)i;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ws->na = (int)m;
        ws->lbase = 0;
    }
}

static int grid_for(i64 total)
{
    i64 g = (total + 255) / 256;
    const i64 cap = (i64)sm_count() * 8;
    return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

namespace {
struct TcLayout {
    size_t state, stamp, live, ws, ulist, list, x8, rt8, rbuf, total;
    i64 mpad, npad;
};

TcLayout tc_layout(i64 m, i64 n)
{
    TcLayout L{};
    const i64 wc = words_of(n);
    L.mpad = (m + UM - 1) / UM * UM;
    L.npad = (64 * wc + UN - 1) / UN * UN;
    size_t off = 0;
    L.state = off;  off += al256((size_t)m);
    L.stamp = off;  off += al256((size_t)m * 4);
    L.live = off;   off += 2 * al256((size_t)m);          // one flag array per window parity
    L.ws = off;     off += 2 * al256(sizeof(WinState));   // one state per window parity
    L.ulist = off;  off += al256((size_t)m * 4);
    L.list = off;   off += al256((size_t)m * 4);
    L.x8 = off;     off += al256((size_t)L.mpad * WBITS);
    L.rt8 = off;    off += al256((size_t)L.npad * WBITS);
    L.rbuf = off;   off += al256((size_t)WBITS * (size_t)wc * 8);
    L.total = off;
    return L;
}
}  // namespace

size_t elim_tc_workspace(i64 m, i64 n) { return tc_layout(m, n).total; }

namespace {
// Captured eliminations, kept for the life of the process (at most
// kMaxElimGraphs; further shapes or buffers run without a graph).
struct ElimGraphKey {
    int dev;
    const void *p[5];
    long long v[4];
};
struct ElimGraph {
    ElimGraphKey k;
    cudaGraphExec_t exec;
};
constexpr size_t kMaxElimGraphs = 16;
constexpr size_t kMaxElimSeen = 64;
std::mutex g_elim_graph_mu;
std::vector<ElimGraph> *g_elim_graphs = nullptr;
std::vector<ElimGraphKey> *g_elim_seen = nullptr;  // calls made once, without a graph
size_t g_elim_seen_next = 0;                       // the oldest entry, replaced once the list is full

bool elim_graphs_enabled()
{
    const char *e = std::getenv("MELA_ELIM_GRAPH");
    return !(e && e[0] == '0');
}
cudaGraphExec_t elim_graph_lookup(const ElimGraphKey &k)
{
    if (!elim_graphs_enabled()) return nullptr;
    std::lock_guard<std::mutex> lk(g_elim_graph_mu);
    if (!g_elim_graphs) return nullptr;
    for (const ElimGraph &g : *g_elim_graphs)
        if (std::memcmp(&g.k, &k, sizeof k) == 0) return g.exec;
    return nullptr;
}
// Capture now: the same call (device, buffers, shape, form) was made before
// -- a one-off call does not pay for instantiating a graph --, the stream is
// not being captured by the caller and there is room to keep one more graph.
bool elim_graph_capturable(const ElimGraphKey &k, cudaStream_t s)
{
    if (!elim_graphs_enabled()) return false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return false;
    }
    std::lock_guard<std::mutex> lk(g_elim_graph_mu);
    if (g_elim_graphs && g_elim_graphs->size() >= kMaxElimGraphs) return false;
    if (!g_elim_seen) g_elim_seen = new std::vector<ElimGraphKey>();
    for (const ElimGraphKey &q : *g_elim_seen)
        if (std::memcmp(&q, &k, sizeof k) == 0) return true;
    // remember the call; a full list forgets its oldest entry, so a stream of
    // one-off shapes never keeps a repeated call from being captured
    if (g_elim_seen->size() < kMaxElimSeen) {
        g_elim_seen->push_back(k);
    } else {
        (*g_elim_seen)[g_elim_seen_next] = k;
        g_elim_seen_next = (g_elim_seen_next + 1) % kMaxElimSeen;
    }
    return false;
}
void elim_graph_store(const ElimGraphKey &k, cudaGraphExec_t exec)
{
    std::lock_guard<std::mutex> lk(g_elim_graph_mu);
    if (!g_elim_graphs) g_elim_graphs = new std::vector<ElimGraph>();
    g_elim_graphs->push_back(ElimGraph{k, exec});
}
}  // namespace

mela_status elim_tc_device(u64 *M, i64 ld, i64 m, i64 n, int rref, long long *d_rank, long long *d_piv,
                           long long *d_prow, void *wsp, size_t ws_bytes, cudaStream_t s)
{
    const TcLayout L = tc_layout(m, n);
    if (!wsp || ws_bytes < L.total) {
        set_error("elimination workspace of %zu bytes needed, %zu given", L.total, ws_bytes);
        return MELA_ERR_INVALID;
    }
    if (L.mpad / UM > INT_MAX / 2 || L.npad > ((i64)1 << 31)) {
        set_error("tensor-core elimination: matrix too large");
        return MELA_ERR_UNSUPPORTED;
    }
    unsigned char *b = (unsigned char *)wsp;
    unsigned char *state = b + L.state;
    int *stamp = (int *)(b + L.stamp);
    WinState *wsv[2] = {(WinState *)(b + L.ws), (WinState *)(b + L.ws + al256(sizeof(WinState)))};
    int *ulist = (int *)(b + L.ulist);
    unsigned char *X8 = b + L.x8;
    unsigned char *Rt8 = b + L.rt8;
    u64 *Rbuf = (u64 *)(b + L.rbuf);
    int *list = (int *)(b + L.list);
    unsigned char *livev[2] = {b + L.live, b + L.live + al256((size_t)m)};
    const i64 wc = words_of(n);

    CUtensorMap mx, mr;
    mela_status st = make_u8_kmajor_map(&mx, X8, L.mpad, WBITS, UM);
    if (st != MELA_OK) return st;
    st = make_u8_kmajor_map(&mr, Rt8, L.npad, WBITS, UN);
    if (st != MELA_OK) return st;
    cudaStream_t s2;
    if ((st = side_stream(&s2)) != MELA_OK) return st;
    cudaStream_t s3;  // the coefficient pass, beside the combine and transpose
    if ((st = aux_stream(&s3)) != MELA_OK) return st;

    const size_t wf_smem = sizeof(WfSmem);
    MELA_CUDA_TRY(cudaFuncSetAttribute(window_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)wf_smem));
    MELA_CUDA_TRY(cudaFuncSetAttribute(tc_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, U_SMEM));
    const int cb_smem = (int)sizeof(CbSmem);
    MELA_CUDA_TRY(cudaFuncSetAttribute(window_combine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, cb_smem));
    const int sms = sm_count();
    const i64 coef_blocks_full = (m + 255) / 256;
    const int coef_blocks = (int)(coef_blocks_full < (i64)sms * 8 ? coef_blocks_full : (i64)sms * 8);
    const i64 tiles_max = L.mpad / UM, chunks_max = (tiles_max + U_MCH - 1) / U_MCH;
    u32 *err = device_error_word();

    // Look-ahead: the update of window w is split into its second strip
    // (window w+1's columns), run on the caller's stream before window w+1 is
    // factored, and the rest, forked to the side stream so that it runs while
    // window w+1 is factored (on an SM the fork leaves free).
    // Window w+1's combine waits for it: it reads the pivot rows' later words,
    // and its coefficient and R buffers are the ones the rest still reads.
    // Window states and row flags alternate by window parity so that the
    // factorization of w+1 never writes what the update of w reads.
    // The coefficient pass of a window reads only rows that are not its pivot
    // rows, which the transpose kernel overwrites, so it runs on a third
    // stream beside the combine and the transpose and rejoins before the
    // update.
    cudaEvent_t evs[4] = {};
    for (int i = 0; i < 4; ++i) {
        if (cudaEventCreateWithFlags(&evs[i], cudaEventDisableTiming) != cudaSuccess) {
            for (int j = 0; j < i; ++j) cudaEventDestroy(evs[j]);
            set_error("cudaEventCreate failed");
            return MELA_ERR_CUDA;
        }
    }
    cudaEvent_t ev_fork = evs[0], ev_join = evs[1], ev_cfork = evs[2], ev_cjoin = evs[3];
    cudaStream_t sx = s;  // the stream the launches go to (a capture stream while capturing)
    auto run = [&]() -> mela_status {
        MELA_CUDA_TRY(cudaMemsetAsync(state, 1, (size_t)m, sx));
        MELA_CUDA_TRY(cudaMemsetAsync(stamp, 0xff, (size_t)m * 4, sx));
        MELA_CUDA_TRY(cudaMemsetAsync(b + L.live, 1, 2 * al256((size_t)m), sx));
        MELA_CUDA_TRY(cudaMemsetAsync(b + L.ws, 0, 2 * al256(sizeof(WinState)), sx));
        list_init_kernel<<<grid_for(m), 256, 0, sx>>>(list, m, wsv[1]);  // the state "before" window 0
        bool forked = false;
        int wid = 0;
        for (i64 w = 0; w < wc; w += WW, ++wid) {
            const i64 lw = wc - w;
            WinState *cur = wsv[wid & 1], *prev = wsv[(wid + 1) & 1];
            unsigned char *live = livev[wid & 1];  // flags of window wid-2 (complete); then this window's
            window_factor_kernel<<<1, WF_THREADS, wf_smem, sx>>>(M, ld, m, n, w, list, live, state, stamp, wid, prev,
                                                                cur, d_piv, d_prow);
            if (forked) {
                MELA_CUDA_TRY(cudaStreamWaitEvent(sx, ev_join, 0));
                forked = false;
            }
            MELA_CUDA_TRY(cudaEventRecord(ev_cfork, sx));
            MELA_CUDA_TRY(cudaStreamWaitEvent(s3, ev_cfork, 0));
            window_coef_kernel<<<coef_blocks, 256, 0, s3>>>(M, ld, m, wc, w, list, stamp, wid, rref, cur, ulist, X8,
                                                           live);
            MELA_CUDA_TRY(cudaEventRecord(ev_cjoin, s3));
            window_combine_kernel<<<(unsigned)((lw + CB_W - 1) / CB_W), 256, cb_smem, sx>>>(M, ld, wc, w, cur, Rbuf,
                                                                                           wc);
            window_rt_kernel<<<(unsigned)lw, 256, 0, sx>>>(M, ld, w, Rbuf, wc, cur, Rt8);
            MELA_CUDA_TRY(cudaStreamWaitEvent(sx, ev_cjoin, 0));
            // near: strip 1 (the next window's columns, all the next
            // factorization reads), one row tile per CTA; far: strip 0 (the
            // window's own columns: only the RREF needs them -- for the rank
            // every updated row is in the window basis' span and its window
            // part becomes zero) and strips 2.., on the side stream
            const i64 strips = (lw + 3) / 4;
            if (strips >= 2) {
                const int grid_near = (int)(tiles_max < sms ? tiles_max : sms);
                tc_update_kernel<<<grid_near, U_THREADS, U_SMEM, sx>>>(mx, mr, M, ld, wc, w, cur, ulist, live, 1, 2,
                                                                      -1, 1, err);
            }
            const int far_lo = rref ? 0 : 2, far_skip = (rref && strips >= 2) ? 1 : -1;
            const i64 far_strips = (strips > far_lo ? strips - far_lo : 0) - (far_skip >= 0 ? 1 : 0);
            if (far_strips > 0) {
                const i64 units = far_strips * chunks_max;
                const int cap = sms > 4 ? sms - 2 : sms;  // SMs left for the next factorization
                const int grid_far = (int)(units < cap ? units : cap);
                MELA_CUDA_TRY(cudaEventRecord(ev_fork, sx));
                MELA_CUDA_TRY(cudaStreamWaitEvent(s2, ev_fork, 0));
                tc_update_kernel<<<grid_far, U_THREADS, U_SMEM, s2>>>(mx, mr, M, ld, wc, w, cur, ulist, live, far_lo,
                                                                     (int)strips, far_skip, U_MCH, err);
                MELA_CUDA_TRY(cudaEventRecord(ev_join, s2));
                forked = true;
            }
        }
        if (forked) MELA_CUDA_TRY(cudaStreamWaitEvent(sx, ev_join, 0));
        MELA_LAUNCH_CHECK("tensor-core elimination");
        WinState *last = wsv[(wid + 1) & 1];  // the state written by the last window (wid-1)
        MELA_CUDA_TRY(cudaMemcpyAsync(d_rank, &last->rank, sizeof(long long), cudaMemcpyDeviceToDevice, sx));
        return MELA_OK;
    };
    // The launch sequence depends only on the shape and the buffers, so from
    // the second call on it is captured once into a CUDA graph per (device,
    // buffers, shape, form), on the thread's capture stream, and replayed on
    // the caller's stream: about
    // 1.4 ms less per 16384 x 32768 call than launching the 770 kernels and
    // events one by one.  A caller that is itself capturing gets the launches
    // in its own graph.
    ElimGraphKey key;
    std::memset(&key, 0, sizeof key);
    cudaGetDevice(&key.dev);
    key.p[0] = M;
    key.p[1] = d_rank;
    key.p[2] = d_piv;
    key.p[3] = d_prow;
    key.p[4] = wsp;
    key.v[0] = ld;
    key.v[1] = m;
    key.v[2] = n;
    key.v[3] = rref;
    cudaGraphExec_t exec = elim_graph_lookup(key);
    cudaStream_t cap = nullptr;
    if (exec) {
        st = cudaGraphLaunch(exec, s) == cudaSuccess ? MELA_OK : MELA_ERR_CUDA;
        if (st != MELA_OK) set_error("cudaGraphLaunch (tensor-core elimination) failed");
    } else if (elim_graph_capturable(key, s) && capture_stream(&cap) == MELA_OK) {
        st = MELA_OK;
        if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            st = run();
        } else {
            sx = cap;
            const mela_status bst = run();
            sx = s;
            cudaGraph_t g = nullptr;
            const cudaError_t ee = cudaStreamEndCapture(cap, &g);
            cudaGraphExec_t ex = nullptr;
            if (bst == MELA_OK && ee == cudaSuccess && g && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess) {
                elim_graph_store(key, ex);
                st = cudaGraphLaunch(ex, s) == cudaSuccess ? MELA_OK : MELA_ERR_CUDA;
                if (st != MELA_OK) set_error("cudaGraphLaunch (tensor-core elimination) failed");
            } else {
                cudaGetLastError();
                st = bst != MELA_OK ? bst : run();  // not capturable here: launch directly
            }
            if (g) cudaGraphDestroy(g);
        }
    } else {
        st = run();
    }
    for (cudaEvent_t e : evs) cudaEventDestroy(e);
    return st;
}

}  // namespace mela
