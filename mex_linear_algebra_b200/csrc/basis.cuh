// basis.cuh -- warp-level XOR bases of 64-bit panel words, shared by the
// blocked elimination of single matrices (elim.cu) and of batches (batch.cu).
//
// A basis holds at most 64 vectors, each stored under its lowest set bit
// ("leading bit"); the set of leading bits of any such basis of a space is
// the space's set of greedy pivot columns.  Alongside each reduced vector
// the basis keeps the ORIGINAL word and the row it came from, so the rows
// that entered a basis are original rows spanning the same space.
#pragma once

#include "mela_common.cuh"

namespace mela {

struct WarpBasis {
    u64 B[64];  // reduced vector with leading bit b
    u64 O[64];  // original word of the row that entered at b
    int R[64];  // that row
};

__device__ __forceinline__ int ctz64_(u64 x) { return __ffsll((long long)x) - 1; }

// Insert the 32 lane values x (original word o, row r) into `wb`, whose
// occupied leading bits are `have` (warp-uniform).  Lanes reduce their value
// by the basis from the lowest bit up; among lanes left with a new leading
// bit the lowest lane enters first, then the others reduce by it, until no
// lane holds a nonzero value.
__device__ inline void warp_basis_insert(WarpBasis &wb, u64 x, u64 o, int r, u64 &have)
{
    const int lane = threadIdx.x & 31;
    while (true) {
        while (x) {
            const u64 lb = x & (~x + 1);
            if (!(lb & have)) break;
            x ^= wb.B[ctz64_(lb)];
        }
        const unsigned bal = __ballot_sync(0xffffffffu, x != 0);
        if (!bal) break;
        const int src = __ffs(bal) - 1;
        const u64 xb = __shfl_sync(0xffffffffu, x, src);
        const u64 ob = __shfl_sync(0xffffffffu, o, src);
        const int rb = __shfl_sync(0xffffffffu, r, src);
        const int b = ctz64_(xb);
        if (lane == 0) {
            wb.B[b] = xb;
            wb.O[b] = ob;
            wb.R[b] = rb;
        }
        have |= 1ull << b;
        if (lane == src) x = 0;
        __syncwarp();
    }
}

// Insert every vector of basis `src` (occupied bits `src_have`) into `dst`
// by its original word.
__device__ inline void warp_basis_merge(WarpBasis &dst, u64 &have, const WarpBasis &src, u64 src_have)
{
    const int lane = threadIdx.x & 31;
    for (int half = 0; half < 2; ++half) {
        const int b = half * 32 + lane;
        u64 o = 0;
        int r = 0;
        if ((src_have >> b) & 1) {
            o = src.O[b];
            r = src.R[b];
        }
        warp_basis_insert(dst, o, o, r, have);
    }
}

// Gauss-Jordan on the final basis (one warp).  With the p = popc(pm) entered
// rows S_k (k in order of increasing leading bit), finds for each pivot bit
// b_t (t-th set bit of pm, increasing) the combination coef[t] (bit k set:
// S_k included) whose restriction to the pivot bits is the unit vector of
// b_t.  Writes bits[t] = b_t, coef[t], srow[t] (the S row that receives
// the reduced row t) and sel[k] = S_k.  Returns p.
__device__ inline int warp_panel_gauss_jordan(const WarpBasis &wb, u64 pm, int *bits, u64 *coef,
                                              int *srow, int *sel)
{
    const int lane = threadIdx.x & 31;
    const int p = __popcll(pm);
    u64 q[2], a[2];
    int rowk[2], step[2] = {-1, -1};
    bool used[2] = {false, false};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int k = lane + 32 * h;
        q[h] = 0;
        a[h] = 0;
        rowk[h] = -1;
        if (k < p) {
            u64 t = pm;
            for (int i = 0; i < k; ++i) t &= t - 1;
            const int b = ctz64_(t);
            q[h] = wb.O[b] & pm;
            a[h] = 1ull << k;
            rowk[h] = wb.R[b];
        }
    }
    // The row chosen at step t keeps being reduced by later steps, so its
    // combination is final only after the loop.
    u64 rest = pm;
    for (int t = 0; t < p; ++t) {
        const int b = ctz64_(rest);
        rest &= rest - 1;
        const u64 bit = 1ull << b;
        const unsigned c0 = __ballot_sync(0xffffffffu, !used[0] && (q[0] & bit));
        const unsigned c1 = __ballot_sync(0xffffffffu, !used[1] && (q[1] & bit));
        const int src = c0 ? (__ffs(c0) - 1) : (__ffs(c1) - 1);
        const int sh = c0 ? 0 : 1;
        const u64 qs = __shfl_sync(0xffffffffu, sh ? q[1] : q[0], src);
        const u64 as = __shfl_sync(0xffffffffu, sh ? a[1] : a[0], src);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const bool me = (lane == src && h == sh);
            if (!me && (q[h] & bit)) {
                q[h] ^= qs;
                a[h] ^= as;
            }
            if (me) {
                used[h] = true;
                step[h] = t;
            }
        }
        if (lane == 0) bits[t] = b;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int k = lane + 32 * h;
        if (k < p) {
            const int t = step[h];
            sel[k] = rowk[h];
            coef[t] = a[h];
            srow[t] = rowk[h];
        }
    }
    __syncwarp();
    return p;
}

}  // namespace mela
