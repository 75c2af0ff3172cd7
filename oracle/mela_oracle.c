/*
 * mela_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference library's GF(2) algorithms
 * (HCPhy/mex_linear_algebra, src/mela_*.c), used as the checker for the
 * CUDA path: tests/ compare the GPU results with these functions on the
 * same seeded inputs, and bench.py times them as a CPU baseline.  Nothing
 * in the shipped library links, loads or calls this file.
 *
 * Parity pinning: tests/test_oracle_pins.py checks every function here
 * against (a) the known-answer cases of the reference's own tests
 * (run_ci_tests.m, compile_mex.m, gf2null/gf2null.m) and (b) the reference
 * MEX gateways themselves, compiled from the reference sources by
 * oracle/Makefile into oracle/_ref and driven through the non-MATLAB MEX
 * host, on seeded random inputs (fixtures in tests/golden/).
 *
 * Layout ("packed"): row-major uint64 words, bit j of row i in word
 * i*ld + (j >> 6) at bit (j & 63) -- the reference's own convention
 * (src/mela_matmul_gf2.c:33-36, src/mela_null_gf2.c:33-40).  Bits at
 * columns >= n in the last word of a row are kept zero.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef int64_t i64;
typedef uint64_t u64;

#define WORDS(n) (((n) + 63) >> 6)

/* ------------------------------------------------------------------ */
/* Seeded generator (counter-based splitmix64).                        */
/* word(seed, stream, i) is output number i of a splitmix64 stream      */
/* whose state starts at key(seed, stream); any slice can be produced   */
/* independently, so CPU and GPU generate identical bits.               */
/* ------------------------------------------------------------------ */
static inline u64 mix64(u64 z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

u64 orc_stream_key(u64 seed, u64 stream)
{
    return mix64(seed * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL) ^
           mix64(stream + 0xD1B54A32D192ED03ULL);
}

u64 orc_rand_word(u64 key, u64 i)
{
    return mix64(key + (i + 1) * 0x9E3779B97F4A7C15ULL);
}

void orc_rand_words(u64 seed, u64 stream, u64 start, i64 count, u64 *out)
{
    u64 key = orc_stream_key(seed, stream);
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < count; ++i) out[i] = orc_rand_word(key, start + (u64)i);
}

/* Dense Bernoulli(1/2) m x n packed matrix: row i, word w takes word
 * number i*WORDS(n)+w of the stream, with bits >= n masked off. */
void orc_rand_dense(u64 seed, u64 stream, i64 m, i64 n, u64 *out, i64 ld)
{
    u64 key = orc_stream_key(seed, stream);
    i64 wc = WORDS(n);
    u64 tail = (n & 63) ? ((1ULL << (n & 63)) - 1) : ~0ULL;
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < m; ++i) {
        for (i64 w = 0; w < wc; ++w) {
            u64 v = orc_rand_word(key, (u64)(i * wc + w));
            if (w == wc - 1) v &= tail;
            out[i * ld + w] = v;
        }
        for (i64 w = wc; w < ld; ++w) out[i * ld + w] = 0;
    }
}

/* ------------------------------------------------------------------ */
/* Packing (reference: pack_rows_logical / pack_rows_double,            */
/* src/mela_matmul_gf2.c:42-69; inline packs src/mela_rank_gf2.c:154-176 */
/* src/mela_null_gf2.c:169-187).  A double is read as ((int)x) & 1.     */
/* On x86-64 the conversion of a NaN or of a value outside the int      */
/* range yields INT_MIN (even), so those read as 0; this restatement    */
/* spells that out instead of relying on undefined behaviour.           */
/* ------------------------------------------------------------------ */
int orc_parity_double(double x)
{
    if (!(x >= -2147483648.0 && x < 2147483648.0)) return 0;
    int v = (int)x;
    return v & 1;
}

void orc_pack_colmajor(int kind, i64 m, i64 n, const void *in, u64 *out, i64 ld)
{
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < m; ++i) {
        u64 *row = out + i * ld;
        for (i64 w = 0; w < ld; ++w) row[w] = 0;
        for (i64 j = 0; j < n; ++j) {
            int bit;
            if (kind == 1) bit = orc_parity_double(((const double *)in)[i + j * m]);
            else bit = ((const uint8_t *)in)[i + j * m] != 0;
            if (bit) row[j >> 6] |= 1ULL << (j & 63);
        }
    }
}

/* Reference unpack: src/mela_matmul_gf2.c:193-205 (C column-major). */
void orc_unpack_colmajor(const u64 *in, i64 ld, i64 m, i64 n, uint8_t *out)
{
#pragma omp parallel for schedule(static)
    for (i64 j = 0; j < n; ++j)
        for (i64 i = 0; i < m; ++i)
            out[i + j * m] = (uint8_t)((in[i * ld + (j >> 6)] >> (j & 63)) & 1);
}

/* ------------------------------------------------------------------ */
/* Products.                                                            */
/* ------------------------------------------------------------------ */

/* Plain product, the reference's loop order (src/mela_matmul_gf2.c:111-
 * 190): per block of C rows, for each k, every row i with A(i,k) = 1
 * XORs packed row k of B into C row i. */
void orc_matmul(const u64 *A, i64 lda, const u64 *B, i64 ldb, u64 *C, i64 ldc,
                i64 m, i64 k, i64 n)
{
    i64 wc = WORDS(n);
    const i64 BR = 256;
#pragma omp parallel for schedule(dynamic, 1)
    for (i64 ib = 0; ib < m; ib += BR) {
        i64 ie = ib + BR < m ? ib + BR : m;
        for (i64 i = ib; i < ie; ++i)
            for (i64 w = 0; w < wc; ++w) C[i * ldc + w] = 0;
        for (i64 kk = 0; kk < k; ++kk) {
            const u64 *bk = B + kk * ldb;
            for (i64 i = ib; i < ie; ++i) {
                if ((A[i * lda + (kk >> 6)] >> (kk & 63)) & 1) {
                    u64 *ci = C + i * ldc;
                    for (i64 w = 0; w < wc; ++w) ci[w] ^= bk[w];
                }
            }
        }
    }
}

/* Four-Russians product (src/mela_matmul_m4ri.c:113-229): per strip of
 * `kk` rows of B build the 2^kk table of XOR combinations (doubling
 * construction, :113-137), then each C row XORs the entry indexed by its
 * kk bits of A.  Same result as orc_matmul. */
void orc_matmul_m4ri(const u64 *A, i64 lda, const u64 *B, i64 ldb, u64 *C, i64 ldc,
                     i64 m, i64 k, i64 n, int kk)
{
    i64 wc = WORDS(n);
    const i64 BR = 256;
    if (kk < 1) kk = 1;
    if (kk > 12) kk = 12;
#pragma omp parallel
    {
        u64 *T = (u64 *)calloc((size_t)(1 << kk) * (size_t)(wc ? wc : 1), sizeof(u64));
#pragma omp for schedule(dynamic, 1)
        for (i64 ib = 0; ib < m; ib += BR) {
            i64 ie = ib + BR < m ? ib + BR : m;
            for (i64 i = ib; i < ie; ++i)
                for (i64 w = 0; w < wc; ++w) C[i * ldc + w] = 0;
            for (i64 kb = 0; kb < k; kb += kk) {
                int kc = (int)((kb + kk <= k) ? kk : (k - kb));
                for (i64 w = 0; w < wc; ++w) T[w] = 0;
                int size = 1;
                for (int b = 0; b < kc; ++b) {
                    const u64 *rb = B + (kb + b) * ldb;
                    for (int j = 0; j < size; ++j) {
                        u64 *dst = T + (size_t)(size + j) * wc;
                        const u64 *src = T + (size_t)j * wc;
                        for (i64 w = 0; w < wc; ++w) dst[w] = src[w] ^ rb[w];
                    }
                    size <<= 1;
                }
                for (i64 i = ib; i < ie; ++i) {
                    unsigned idx = 0;
                    for (int b = 0; b < kc; ++b) {
                        i64 col = kb + b;
                        idx |= (unsigned)((A[i * lda + (col >> 6)] >> (col & 63)) & 1) << b;
                    }
                    if (idx) {
                        u64 *ci = C + i * ldc;
                        const u64 *t = T + (size_t)idx * wc;
                        for (i64 w = 0; w < wc; ++w) ci[w] ^= t[w];
                    }
                }
            }
        }
        free(T);
    }
}

/* ------------------------------------------------------------------ */
/* Elimination.                                                         */
/* ------------------------------------------------------------------ */

static inline int getb(const u64 *row, i64 c) { return (int)((row[c >> 6] >> (c & 63)) & 1); }

static void swap_rows(u64 *a, u64 *b, i64 wc)
{
    for (i64 w = 0; w < wc; ++w) {
        u64 t = a[w];
        a[w] = b[w];
        b[w] = t;
    }
}

static void xor_into(u64 *dst, const u64 *src, i64 wc)
{
    for (i64 w = 0; w < wc; ++w) dst[w] ^= src[w];
}

/* Forward Gaussian elimination rank (src/mela_rank_gf2.c:27-121): per
 * column, first row at or below the current pivot row with the bit set
 * becomes the pivot (swap), which is XORed into every lower row that has
 * the bit.  M is overwritten. */
i64 orc_rank_ge(u64 *M, i64 ld, i64 m, i64 n)
{
    i64 wc = WORDS(n);
    i64 r = 0;
    for (i64 c = 0; c < n && r < m; ++c) {
        i64 p = -1;
        for (i64 i = r; i < m; ++i)
            if (getb(M + i * ld, c)) {
                p = i;
                break;
            }
        if (p < 0) continue;
        if (p != r) swap_rows(M + p * ld, M + r * ld, wc);
        const u64 *prow = M + r * ld;
#pragma omp parallel for schedule(static) if (m - r > 512)
        for (i64 i = r + 1; i < m; ++i)
            if (getb(M + i * ld, c)) xor_into(M + i * ld, prow, wc);
        ++r;
    }
    return r;
}

/* Blocked Four-Russians rank (src/mela_rank_m4ri.c:94-279), k columns per
 * block: pivots are searched in a row window [r, limit) that grows k rows
 * at a time, new window rows being cleaned against the block's pivots
 * (:157-183); pivots inside the block are reduced against each other
 * (:222-234); a 2^p table of pivot-row combinations (:65-88) then clears
 * the block's pivot columns from every row below the window (:250-267).
 * M is overwritten. */
i64 orc_rank_m4ri(u64 *M, i64 ld, i64 m, i64 n, int k)
{
    i64 wc = WORDS(n);
    if (k < 1) k = 1;
    if (k > 16) k = 16;
    u64 *T = (u64 *)calloc((size_t)(1 << k) * (size_t)(wc ? wc : 1), sizeof(u64));
    i64 *pcol = (i64 *)malloc(sizeof(i64) * (size_t)k);
    u64 **prow = (u64 **)malloc(sizeof(u64 *) * (size_t)k);
    i64 r = 0, c = 0;
    while (r < m && c < n) {
        int kc = (int)((c + k <= n) ? k : (n - c));
        int p = 0;
        i64 limit = r + k < m ? r + k : m;
        for (int b = 0; b < kc; ++b) {
            if (r + p >= m) break;
            i64 col = c + b;
            i64 piv = -1;
            for (i64 i = r + p; i < limit; ++i)
                if (getb(M + i * ld, col)) {
                    piv = i;
                    break;
                }
            while (piv < 0 && limit < m) {
                i64 old = limit;
                limit = limit + k <= m ? limit + k : m;
                for (int q = 0; q < p; ++q)
                    for (i64 j = old; j < limit; ++j)
                        if (getb(M + j * ld, pcol[q])) xor_into(M + j * ld, prow[q], wc);
                for (i64 i = old; i < limit; ++i)
                    if (getb(M + i * ld, col)) {
                        piv = i;
                        break;
                    }
            }
            if (piv < 0) continue;
            if (piv != r + p) swap_rows(M + (r + p) * ld, M + piv * ld, wc);
            u64 *pr = M + (r + p) * ld;
            for (i64 j = r + p + 1; j < limit; ++j)
                if (getb(M + j * ld, col)) xor_into(M + j * ld, pr, wc);
            prow[p] = pr;
            pcol[p] = col;
            ++p;
        }
        if (p > 0) {
            for (int i = 0; i < p; ++i)
                for (int j = 0; j < i; ++j)
                    if (getb(prow[j], pcol[i])) xor_into(prow[j], prow[i], wc);
            for (i64 w = 0; w < wc; ++w) T[w] = 0;
            int size = 1;
            for (int b = 0; b < p; ++b) {
                for (int j = 0; j < size; ++j) {
                    u64 *dst = T + (size_t)(size + j) * wc;
                    const u64 *src = T + (size_t)j * wc;
                    for (i64 w = 0; w < wc; ++w) dst[w] = src[w] ^ prow[b][w];
                }
                size <<= 1;
            }
#pragma omp parallel for schedule(static) if (m - limit > 512)
            for (i64 j = limit; j < m; ++j) {
                u64 *row = M + j * ld;
                unsigned idx = 0;
                for (int i = 0; i < p; ++i) idx |= (unsigned)getb(row, pcol[i]) << i;
                if (idx) xor_into(row, T + (size_t)idx * wc, wc);
            }
            r += p;
        }
        c += kc;
    }
    free(T);
    free(pcol);
    free(prow);
    return r;
}

/* Full reduced row echelon form (src/mela_null_gf2.c:88-131): per column,
 * pivot search at or below the pivot row, swap, then the pivot row is
 * XORed into every OTHER row holding the bit.  Pivot columns are written
 * to `pivots` (ascending); returns the rank. */
i64 orc_rref(u64 *M, i64 ld, i64 m, i64 n, i64 *pivots)
{
    i64 wc = WORDS(n);
    i64 r = 0;
    for (i64 c = 0; c < n && r < m; ++c) {
        i64 p = -1;
        for (i64 i = r; i < m; ++i)
            if (getb(M + i * ld, c)) {
                p = i;
                break;
            }
        if (p < 0) continue;
        if (p != r) swap_rows(M + p * ld, M + r * ld, wc);
        pivots[r] = c;
        const u64 *prow = M + r * ld;
#pragma omp parallel for schedule(static) if (m > 512)
        for (i64 i = 0; i < m; ++i)
            if (i != r && getb(M + i * ld, c)) xor_into(M + i * ld, prow, wc);
        ++r;
    }
    return r;
}

/* Echelon form of the reference's Four-Russians null space
 * (src/mela_null_m4ri.c:92-240): up to k pivots per block by ordinary
 * elimination of all rows below (:116-159), then a 2^p table of the
 * block's pivot rows (:177-198) clears the block's pivot columns from
 * every row outside the block (:210-231).  Pivot rows inside a block are
 * not reduced against each other, so the result is echelon, not RREF;
 * back-substitution (orc_null_backsub) still yields the same basis. */
i64 orc_echelon_m4ri(u64 *M, i64 ld, i64 m, i64 n, int k, i64 *pivots)
{
    i64 wc = WORDS(n);
    if (k < 1) k = 1;
    if (k > 16) k = 16;
    i64 *cp = (i64 *)malloc(sizeof(i64) * (size_t)k);
    i64 *crow = (i64 *)malloc(sizeof(i64) * (size_t)k);
    u64 *T = (u64 *)calloc((size_t)(1 << k) * (size_t)(wc ? wc : 1), sizeof(u64));
    i64 prow = 0, npiv = 0;
    i64 cb = 0;
    while (cb < n && prow < m) {
        int kp = 0;
        i64 c = cb;
        while (c < n && kp < k && prow + kp < m) {
            i64 start = prow + kp, p = -1;
            for (i64 i = start; i < m; ++i)
                if (getb(M + i * ld, c)) {
                    p = i;
                    break;
                }
            if (p >= 0) {
                if (p != start) swap_rows(M + p * ld, M + start * ld, wc);
                cp[kp] = c;
                crow[kp] = start;
                pivots[npiv++] = c;
                const u64 *pr = M + start * ld;
                for (i64 i = start + 1; i < m; ++i)
                    if (getb(M + i * ld, c)) xor_into(M + i * ld, pr, wc);
                ++kp;
            }
            ++c;
        }
        if (kp == 0) {
            if (c >= n) break;
            cb = c;
            continue;
        }
        int ne = 1 << kp;
        for (i64 w = 0; w < wc; ++w) T[w] = 0;
        for (int i = 1; i < ne; ++i) {
            int b = 0;
            while (!((i >> b) & 1)) ++b;
            const u64 *src = T + (size_t)(i ^ (1 << b)) * wc;
            const u64 *pr = M + crow[b] * ld;
            u64 *dst = T + (size_t)i * wc;
            for (i64 w = 0; w < wc; ++w) dst[w] = src[w] ^ pr[w];
        }
#pragma omp parallel for schedule(static) if (m > 512)
        for (i64 r = 0; r < m; ++r) {
            if (r >= prow && r < prow + kp) continue;
            u64 *row = M + r * ld;
            unsigned idx = 0;
            for (int j = 0; j < kp; ++j) idx |= (unsigned)getb(row, cp[j]) << j;
            if (idx) xor_into(row, T + (size_t)idx * wc, wc);
        }
        prow += kp;
        cb = c;
    }
    free(cp);
    free(crow);
    free(T);
    return npiv;
}

/* Null-space basis by back-substitution (src/mela_null_gf2.c:189-274,
 * src/mela_null_m4ri.c:298-401): free columns are the non-pivot columns in
 * ascending order; basis vector i starts as e_{f_i}, and for pivots from
 * the last up, v[c_p] = parity(row_p without bit c_p, AND v).  Works on
 * RREF and on the echelon form above.  Vector i is written packed as row i
 * of Zt (ldz words per row), i.e. column i of the reference's n x f
 * logical output.  Returns the nullity f = n - rank. */
i64 orc_null_backsub(const u64 *M, i64 ld, i64 n, const i64 *pivots, i64 rank,
                     u64 *Zt, i64 ldz)
{
    i64 wc = WORDS(n);
    uint8_t *isp = (uint8_t *)calloc((size_t)(n ? n : 1), 1);
    for (i64 p = 0; p < rank; ++p) isp[pivots[p]] = 1;
    i64 f = 0;
    for (i64 c = 0; c < n; ++c) f += !isp[c];
    i64 *fc = (i64 *)malloc(sizeof(i64) * (size_t)(f ? f : 1));
    for (i64 c = 0, t = 0; c < n; ++c)
        if (!isp[c]) fc[t++] = c;
#pragma omp parallel for schedule(dynamic, 16) if (f > 64)
    for (i64 t = 0; t < f; ++t) {
        u64 *v = Zt + t * ldz;
        for (i64 w = 0; w < ldz; ++w) v[w] = 0;
        v[fc[t] >> 6] |= 1ULL << (fc[t] & 63);
        for (i64 p = rank - 1; p >= 0; --p) {
            i64 c = pivots[p];
            const u64 *row = M + p * ld;
            u64 acc = 0;
            for (i64 w = 0; w < wc; ++w) {
                u64 s = row[w];
                if (w == (c >> 6)) s &= ~(1ULL << (c & 63));
                acc ^= s & v[w];
            }
            int par = __builtin_parityll(acc);
            if (par) v[c >> 6] |= 1ULL << (c & 63);
            else v[c >> 6] &= ~(1ULL << (c & 63));
        }
    }
    free(isp);
    free(fc);
    return f;
}

/* Greedy pivot columns without modifying the input (copy + RREF). */
i64 orc_pivot_columns(const u64 *M, i64 ld, i64 m, i64 n, i64 *pivots)
{
    u64 *W = (u64 *)malloc(sizeof(u64) * (size_t)(m * ld ? m * ld : 1));
    memcpy(W, M, sizeof(u64) * (size_t)(m * ld));
    i64 r = orc_rref(W, ld, m, n, pivots);
    free(W);
    return r;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
