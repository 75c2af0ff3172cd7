/*
 * mela.h -- C ABI of the B200 (sm_100a) GF(2) linear-algebra library.
 *
 * Drop-in boundary for the six MEX functions of HCPhy/mex_linear_algebra:
 *
 *   reference gateway (file:line of its mexFunction)     replaced by
 *   mela_matmul_gf2   src/mela_matmul_gf2.c:72-211       mela_matmul_gf2()
 *   mela_matmul_m4ri  src/mela_matmul_m4ri.c:140-251     mela_matmul_m4ri()
 *   mela_rank_gf2     src/mela_rank_gf2.c:126-186        mela_rank_gf2()
 *   mela_rank_m4ri    src/mela_rank_m4ri.c:286-341       mela_rank_m4ri()
 *   mela_null_gf2     src/mela_null_gf2.c:142-281        mela_null_gf2()
 *   mela_null_m4ri    src/mela_null_m4ri.c:251-408       mela_null_m4ri()
 *
 * The host entry points take MATLAB-layout (column-major) logical or double
 * arrays in host memory, exactly what a MEX gateway receives, and return
 * status codes instead of long-jumping; the MEX gateways in
 * mex_linear_algebra_b200/mex/ map each status to the reference's own error
 * text.  The mela_dev_* entry points work on device-resident bit-packed
 * matrices and are stream-ordered.
 *
 * Packed layout: row-major uint64_t words, bit j of row i in word
 * i*ld + j/64 at bit j%64 (the reference's convention,
 * src/mela_matmul_gf2.c:33-36).  Bits past the last column are zero.
 *
 * Every result is bit-exact: products, ranks and null-space bases equal the
 * reference's on every input.  Nothing is computed on the CPU.
 */
#ifndef MELA_H
#define MELA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MELA_OK = 0,
    MELA_ERR_INVALID = 1,      /* bad pointer / size / variant */
    MELA_ERR_SPARSE = 2,       /* sparse input where the reference rejects it */
    MELA_ERR_DIM = 3,          /* inner dimensions disagree */
    MELA_ERR_TYPE = 4,         /* input neither logical nor double */
    MELA_ERR_NOMEM = 5,        /* device or host allocation failed */
    MELA_ERR_CUDA = 6,         /* CUDA runtime error (see mela_last_error) */
    MELA_ERR_TIMEOUT = 7,      /* a bounded device wait ran out */
    MELA_ERR_UNSUPPORTED = 8,  /* no sm_100 device, or size beyond a limit */
    MELA_ERR_NO_DEVICE = 9     /* no CUDA device visible */
} mela_status;

/* Element kinds of a MATLAB array as the gateways see it. */
typedef enum {
    MELA_KIND_LOGICAL = 0,  /* mxLogical, 1 byte, nonzero = 1 */
    MELA_KIND_DOUBLE = 1,   /* double, read as ((int)x) & 1 */
    MELA_KIND_OTHER = 2     /* any other class: rejected like the reference */
} mela_kind;

/* A MATLAB array handed to a gateway: column-major, rows x cols. */
typedef struct {
    int32_t kind;     /* mela_kind */
    int32_t sparse;   /* nonzero if the MATLAB array is sparse */
    int64_t rows;
    int64_t cols;
    const void *data; /* host pointer, rows*cols elements */
} mela_host_matrix;

/* Product variants (the autotuned choice decides only how, never what). */
typedef enum {
    MELA_GEMM_AUTO = 0,
    MELA_GEMM_PLAIN = 1,  /* bit-packed AND + popcount parity on CUDA cores */
    MELA_GEMM_M4RI = 2,   /* Four-Russians tables in shared memory */
    MELA_GEMM_TC = 3,     /* tcgen05 kind::i8 tensor cores, parity of the s32 sum */
    MELA_GEMM_TC_FP4 = 4  /* tcgen05 kind::mxf4 (e2m1 0/1, unit scales), parity of the exact
                             f32 sum; k < 2^23 */
} mela_gemm_variant;

/* Elimination variants (rank / RREF / null space); results are identical. */
typedef enum {
    MELA_ELIM_AUTO = 0,
    MELA_ELIM_PLAIN = 1,  /* per-pivot warp-ballot search + broadcast-XOR sweep */
    MELA_ELIM_M4RI = 2,   /* 64-column panels, Four-Russians tables in shared memory (k = 8 unless tuned) */
    MELA_ELIM_M4RI_K4 = 3, /* the same panels with 4-bit tables (M4RI k = 4) */
    MELA_ELIM_FUSED = 4,   /* the whole elimination by one CTA in one launch */
    MELA_ELIM_TC = 5       /* 256-column windows, trailing update on the tensor cores (tcgen05 kind::i8) */
} mela_elim_variant;

/* Tuning fields of a variant argument.  A variant argument is a base
 * variant (above) in bits 0-7, optionally ORed with these fields; a field of
 * 0 keeps the variant's default.  They change how a result is computed,
 * never the result.  The reference fixes its Four-Russians k per function
 * (k = 8 in src/mela_matmul_m4ri.c:33 and src/mela_null_m4ri.c:28, k = 10
 * in src/mela_rank_m4ri.c:18); here it is a parameter.
 *   MELA_TUNE_K(k)     MELA_ELIM_M4RI: table width k in {4, 6, 7, 8, 9, 10}
 *                      (MELA_ELIM_M4RI_K4 takes only 4; MELA_GEMM_M4RI only 8).
 *   MELA_TUNE_TILE(t)  MELA_ELIM_M4RI / _K4: rows per update CTA, t = 1: 256,
 *                      2: 1024 (default), 3: 4096.
 *                      MELA_GEMM_TC / _TC_FP4: t = 1: one CTA per 128 x 256
 *                      tile; 2: CTA pairs per 256 x 256 tile (the default
 *                      where the padded row count allows).
 *                      MELA_GEMM_M4RI: t = 1: 8 warps of 64 rows per CTA;
 *                      2: 16 warps of 32 rows (the default). */
#define MELA_VARIANT_BASE(v) ((int32_t)(v) & 0xff)
#define MELA_TUNE_K(k) ((int32_t)(k) << 8)
#define MELA_TUNE_TILE(t) ((int32_t)(t) << 12)

/* ------------------------------------------------------------------ */
/* library                                                             */
/* ------------------------------------------------------------------ */
int mela_version(void);
const char *mela_status_string(mela_status s);
/* Detail text of the last failure on the calling thread. */
const char *mela_last_error(void);
/* Device-side error bits (timeouts of bounded waits); `clear` resets them. */
mela_status mela_device_error_flags(uint32_t *flags, int clear);
/* Host-array uploads of the calling thread since the last reset: bytes sent
 * through the page-locked staging slots (column blocks of 2 MiB and larger
 * arrays, host copies overlapping the uploads) and bytes copied directly,
 * with the host time spent copying into the slots and waiting for a slot. */
typedef struct {
    int64_t blocked_bytes;
    int64_t direct_bytes;
    int64_t blocks;
    double host_copy_us;
    double slot_wait_us;
} mela_upload_stats;
void mela_upload_stats_get(mela_upload_stats *out, int reset);
/* Diagnostic of the failure path (no reference counterpart): one kernel whose
 * wait nothing will satisfy -- kind 0 a device flag, kind 1 an mbarrier with
 * tensor memory held -- runs out after limit_ns (1 us .. 1 s), sets the
 * timeout bit of the device error word, frees what it holds and returns.
 * d_out (device, 2 words): [0] = 1 when the wait ran out, [1] = 1 when kind
 * 1 freed its tensor memory.  sync = 0: stream-ordered, the bit stays set
 * for mela_device_error_flags; sync = 1: waits for the stream and returns
 * MELA_ERR_TIMEOUT, clearing the bit, as every synchronous entry point does
 * after a timed-out wait. */
mela_status mela_diag_wait_timeout(int32_t kind, uint64_t limit_ns, uint32_t *d_out, int32_t sync,
                                   void *stream);

/* ------------------------------------------------------------------ */
/* host entry points (MATLAB layout in, MATLAB layout out)              */
/* ------------------------------------------------------------------ */

/* C = A*B over GF(2).  C is rows(A) x cols(B) logical, column-major,
 * caller-allocated (all bytes written).  Validation order and failure
 * classes follow src/mela_matmul_gf2.c:75-88: sparse -> MELA_ERR_SPARSE,
 * inner dimension mismatch -> MELA_ERR_DIM, other classes -> MELA_ERR_TYPE. */
mela_status mela_matmul_gf2(const mela_host_matrix *A, const mela_host_matrix *B,
                            uint8_t *C);
/* Same result through the Four-Russians kernel (src/mela_matmul_m4ri.c). */
mela_status mela_matmul_m4ri(const mela_host_matrix *A, const mela_host_matrix *B,
                             uint8_t *C);

/* Output allocator for the null-space entry points: returns a buffer of
 * rows*cols bytes for the rows x cols logical result (column-major), or NULL
 * when rows*cols is 0.  Called once, after the rank is known. */
typedef uint8_t *(*mela_alloc_fn)(void *ctx, int64_t rows, int64_t cols);

/* Rank over GF(2) (forward elimination, src/mela_rank_gf2.c:27-121 and
 * src/mela_rank_m4ri.c:94-279).  Empty inputs have rank 0. */
mela_status mela_rank_gf2(const mela_host_matrix *A, double *rank);
mela_status mela_rank_m4ri(const mela_host_matrix *A, double *rank);

/* Null-space basis Z (n x nullity logical, column-major): free columns f_i
 * ascending, Z(f_i, i) = 1, Z(pivot column p, i) = RREF(p, f_i) -- the basis
 * of src/mela_null_gf2.c:189-274 and src/mela_null_m4ri.c:298-401, bit for
 * bit.  Sparse input -> MELA_ERR_SPARSE, other classes -> MELA_ERR_TYPE.
 * m = 0 gives the identity (nullity n); n = 0 gives an empty result. */
mela_status mela_null_gf2(const mela_host_matrix *H, mela_alloc_fn alloc, void *ctx,
                          int64_t *nullity);
mela_status mela_null_m4ri(const mela_host_matrix *H, mela_alloc_fn alloc, void *ctx,
                           int64_t *nullity);

/* Sparse input.  No counterpart in the reference, whose gateways reject
 * sparse arrays or read their values as if dense.  MATLAB's own layout:
 * column j holds entries colptr[j] .. colptr[j+1]-1 (colptr[0] = 0,
 * non-decreasing) with 0-based rows rowidx[e] (MATLAB's jc / ir); values is
 * NULL (every entry 1) or one logical byte / double per entry (a double read
 * as ((int)x) & 1, like dense input).  Repeated (row, column) entries add
 * mod 2.  Bad pointers or indices -> MELA_ERR_INVALID (checked on the host
 * before any device work). */
typedef struct {
    int32_t kind; /* MELA_KIND_LOGICAL or MELA_KIND_DOUBLE: the type of values */
    int64_t rows;
    int64_t cols;
    const int64_t *colptr; /* cols + 1 entries */
    const int64_t *rowidx; /* colptr[cols] entries */
    const void *values;    /* NULL or colptr[cols] entries */
} mela_host_csc;
/* Rank over GF(2) of a sparse matrix (the same result as mela_rank_gf2 on
 * its dense form; the elimination variant is chosen by the dispatcher). */
mela_status mela_rank_csc(const mela_host_csc *H, int64_t *rank);
/* Null-space basis of a sparse matrix: the output of mela_null_gf2 on its
 * dense form (n x nullity logical, column-major, through `alloc`). */
mela_status mela_null_csc(const mela_host_csc *H, mela_alloc_fn alloc, void *ctx, int64_t *nullity);

/* ------------------------------------------------------------------ */
/* gateway semantics (shared by the MEX files and other front ends)     */
/* ------------------------------------------------------------------ */
typedef enum {
    MELA_FN_MATMUL_GF2 = 0,
    MELA_FN_MATMUL_M4RI = 1,
    MELA_FN_RANK_GF2 = 2,
    MELA_FN_RANK_M4RI = 3,
    MELA_FN_NULL_GF2 = 4,
    MELA_FN_NULL_M4RI = 5
} mela_function;

/* Creates output `index` (kind MELA_KIND_LOGICAL or MELA_KIND_DOUBLE,
 * rows x cols, column-major) and returns its data pointer. */
typedef void *(*mela_gateway_alloc_fn)(void *ctx, int32_t index, int32_t kind, int64_t rows,
                                       int64_t cols);
typedef struct {
    char id[64];   /* MATLAB error identifier ("" when the reference uses none) */
    char msg[256]; /* error message text */
} mela_gateway_error;

/* Runs one reference gateway (mexFunction of src/mela_*.c) on host arrays:
 * same argument checks in the same order, same error identifiers and
 * messages, same outputs.  Returns 0 on success, 1 with *err filled. */
int mela_gateway(int32_t fn, int32_t nlhs, int32_t nrhs, const mela_host_matrix *prhs,
                 mela_gateway_alloc_fn alloc, void *ctx, mela_gateway_error *err);

/* Host-resident packed product (copies in, computes, copies out). */
mela_status mela_matmul_packed_host(const uint64_t *A, int64_t lda, const uint64_t *B,
                                    int64_t ldb, uint64_t *C, int64_t ldc, int64_t m,
                                    int64_t k, int64_t n, int32_t variant);

/* ------------------------------------------------------------------ */
/* device entry points (packed, stream-ordered)                         */
/* ------------------------------------------------------------------ */

/* Seeded Bernoulli(1/2) packed matrix: word w of row i is output number
 * i*ceil(n/64)+w of a counter-based splitmix64 stream keyed by
 * (seed, stream_id); bits past column n are zero. */
mela_status mela_dev_rand_dense(uint64_t seed, uint64_t stream_id, int64_t m, int64_t n,
                                uint64_t *d_out, int64_t ld, void *stream);

/* Seeded Bernoulli(density) packed matrix: entry (i, j), e = i*n + j, is 1
 * when 16-bit slice e%4 of stream word e/4 is below density*65536. */
mela_status mela_dev_rand_bernoulli(uint64_t seed, uint64_t stream_id, int64_t m, int64_t n,
                                    double density, uint64_t *d_out, int64_t ld, void *stream);

/* Column-major logical (kind 0) or double (kind 1) m x n -> packed rows.
 * Replaces pack_rows_logical/pack_rows_double (src/mela_matmul_gf2.c:42-69)
 * and the inline packs of the other gateways. */
mela_status mela_dev_pack(int32_t kind, int64_t m, int64_t n, const void *d_in,
                          uint64_t *d_out, int64_t ld, void *stream);
/* Sparse (CSC, device arrays; see mela_host_csc) -> packed rows.  Row
 * indices outside [0, m) are skipped and flagged in the device error word
 * (mela_device_error_flags). */
mela_status mela_dev_pack_csc(const int64_t *d_colptr, const int64_t *d_rowidx, const void *d_values,
                              int32_t kind, int64_t m, int64_t n, uint64_t *d_out, int64_t ld,
                              void *stream);
/* Packed rows -> column-major logical bytes (src/mela_matmul_gf2.c:193-205). */
mela_status mela_dev_unpack(const uint64_t *d_in, int64_t ld, int64_t m, int64_t n,
                            uint8_t *d_out, void *stream);
/* Bit transpose: out (cols x rows) = in (rows x cols)^T. */
mela_status mela_dev_transpose(const uint64_t *d_in, int64_t ld_in, int64_t rows,
                               int64_t cols, uint64_t *d_out, int64_t ld_out, void *stream);

/* Workspace bytes mela_dev_matmul needs for this variant and shape. */
size_t mela_matmul_workspace_size(int32_t variant, int64_t m, int64_t k, int64_t n);
/* C = A*B mod 2 on packed device matrices (A m x k, B k x n, C m x n).
 * Replaces the product loops of src/mela_matmul_gf2.c:111-208 and
 * src/mela_matmul_m4ri.c:179-248.  `workspace` must hold
 * mela_matmul_workspace_size() bytes (may be NULL when that is 0). */
mela_status mela_dev_matmul(int32_t variant, const uint64_t *dA, int64_t lda,
                            const uint64_t *dB, int64_t ldb, uint64_t *dC, int64_t ldc,
                            int64_t m, int64_t k, int64_t n, void *workspace,
                            size_t workspace_bytes, void *stream);

/* The two halves of mela_dev_matmul, for callers that overlap or time them
 * separately: operand preparation into the workspace (B transposed; for the
 * tensor-core form also the 0/1 byte expansion of A and B^T), then the
 * product kernel over the prepared operands.  Same arguments and workspace
 * as mela_dev_matmul; run must follow prepare on the same stream. */
mela_status mela_dev_matmul_prepare(int32_t variant, const uint64_t *dA, int64_t lda,
                                    const uint64_t *dB, int64_t ldb, int64_t m, int64_t k,
                                    int64_t n, void *workspace, size_t workspace_bytes,
                                    void *stream);
mela_status mela_dev_matmul_run(int32_t variant, const uint64_t *dA, int64_t lda,
                                const uint64_t *dB, int64_t ldb, uint64_t *dC, int64_t ldc,
                                int64_t m, int64_t k, int64_t n, void *workspace,
                                size_t workspace_bytes, void *stream);

/* Workspace for mela_dev_rank / mela_dev_rref on an m x n matrix. */
size_t mela_elim_workspace_size(int64_t m, int64_t n);
/* Rank of the packed m x n matrix dM (overwritten).  Writes the rank to
 * d_rank (device int64), the pivot columns to d_pivcols and the physical row
 * holding each pivot row to d_pivrows (min(m, n) entries each). */
mela_status mela_dev_rank(int32_t variant, uint64_t *dM, int64_t ld, int64_t m, int64_t n,
                          int64_t *d_rank, int64_t *d_pivcols, int64_t *d_pivrows,
                          void *workspace, size_t workspace_bytes, void *stream);
/* Reduced row echelon form in place (gf2_rref_standard,
 * src/mela_null_gf2.c:88-131): RREF row t is row d_pivrows[t] of dM, with
 * its leading one in column d_pivcols[t] (ascending); rows that are not
 * pivot rows end up zero. */
mela_status mela_dev_rref(int32_t variant, uint64_t *dM, int64_t ld, int64_t m, int64_t n,
                          int64_t *d_rank, int64_t *d_pivcols, int64_t *d_pivrows,
                          void *workspace, size_t workspace_bytes, void *stream);
size_t mela_null_workspace_size(int64_t n, int64_t rank);
/* Null-space basis from an RREF (mela_dev_rref's outputs; `rank` on the
 * host): Zt (n - rank rows of ldz words), row i = basis vector i, i.e.
 * column i of the reference's n x nullity logical output. */
mela_status mela_dev_null_basis(const uint64_t *dR, int64_t ld, int64_t m, int64_t n,
                                int64_t rank, const int64_t *d_pivcols, const int64_t *d_pivrows,
                                uint64_t *dZt, int64_t ldz, void *workspace,
                                size_t workspace_bytes, void *stream);
/* On-device check of a null-space basis: *d_bad_rows (device) = the number
 * of rows i of A (m x n, packed) with A_i . z != 0 for some basis vector z,
 * where Zt holds the f basis vectors as packed rows of n bits (the layout of
 * mela_dev_null_basis); 0 means A Z = 0.  Bits past column n of A and Zt
 * must be zero (the packed convention).  Workspace:
 * mela_null_verify_workspace_size(m, f) bytes.  No reference counterpart
 * (the reference's tests check A Z = 0 on the host). */
size_t mela_null_verify_workspace_size(int64_t m, int64_t f);
mela_status mela_dev_null_verify(const uint64_t *dA, int64_t lda, int64_t m, int64_t n,
                                 const uint64_t *dZt, int64_t ldz, int64_t f, int64_t *d_bad_rows,
                                 void *workspace, size_t workspace_bytes, void *stream);
/* Packed rows -> row-major bytes (rows x n). */
mela_status mela_dev_unpack_rows(const uint64_t *d_in, int64_t ld, int64_t rows, int64_t n,
                                 uint8_t *d_out, void *stream);

/* ------------------------------------------------------------------ */
/* batched rank + null space                                            */
/* ------------------------------------------------------------------ */
/* No counterpart in the reference (which handles one matrix per call).
 * Many matrices of uneven shape are ranked and null-spaced in one
 * persistent launch (replayed as a CUDA graph): a warp per small matrix, a
 * 128-thread group per medium one, a whole CTA per large one.  Item i is
 * packed at word offset in_offset of the input buffer (m rows of
 * ceil(n/64) words; for the logical entry point: an m x n column-major
 * logical array at byte offset sum_{j<i} m_j*n_j); its null-space basis is
 * written at word offset z_offset of the output buffer as n - rank rows of
 * ceil(n/64) words (room for n rows must be reserved), its rank to
 * d_ranks[i].  Results equal mela_rank_gf2 / mela_null_gf2 per matrix. */
typedef struct {
    int64_t m, n;
    int64_t in_offset; /* words */
    int64_t z_offset;  /* words */
} mela_batch_item;
typedef struct mela_batch_plan mela_batch_plan;

/* force_class: -1 = size-based (normal); 0/1/2 = run every item that fits
 * with the CTA / 128-thread / warp engine (for testing the engines). */
mela_status mela_batch_plan_create(const mela_batch_item *items, int64_t count,
                                   int32_t force_class, mela_batch_plan **plan);
/* The same with the engine policy -2 available: each matrix goes to the
 * engine the installed cost model prices lowest among those whose shared
 * memory it fits, from its shape, its density (densities[i], the fraction of
 * ones; NULL: 0.5 for all) and the batch mix (the matrix count and mean
 * log2(m*n) of this batch) -- the size rule of policy -1 when no model is
 * installed.  Policies -1, 0, 1, 2 as force_class above. */
mela_status mela_batch_plan_create_ex(const mela_batch_item *items, int64_t count,
                                      const double *densities, int32_t policy,
                                      mela_batch_plan **plan);
/* d_counts[i] = number of ones of item i of a packed batch (in_offset
 * layout), stream-ordered: the densities mela_batch_plan_create_ex takes. */
mela_status mela_batch_popcounts(const mela_batch_item *items, int64_t count, const uint64_t *d_in,
                                 int64_t *d_counts, void *stream);
void mela_batch_plan_destroy(mela_batch_plan *plan);
mela_status mela_batch_plan_stats(const mela_batch_plan *plan, int64_t *big, int64_t *mid,
                                  int64_t *small);
mela_status mela_batch_rank_null(mela_batch_plan *plan, const uint64_t *d_in, uint64_t *d_zt,
                                 int64_t *d_ranks, int32_t use_graph, void *stream);
mela_status mela_batch_rank_null_logical(mela_batch_plan *plan, const uint8_t *d_in,
                                         uint64_t *d_zt, int64_t *d_ranks, int32_t use_graph,
                                         void *stream);
/* Every matrix of the batch from its logical column-major form (the byte
 * layout of the logical entry point, any alignment; nonzero bytes read as 1)
 * to packed rows in the in_offset layout: the packing step of
 * mela_batch_rank_null_logical on its own.  Words between the matrices are
 * not written. */
mela_status mela_batch_pack_logical(mela_batch_plan *plan, const uint8_t *d_logical,
                                    uint64_t *d_packed, void *stream);
/* Every matrix of the batch from packed rows (in_offset layout) to its
 * logical column-major form (the byte layout of the logical entry point). */
mela_status mela_batch_unpack_logical(mela_batch_plan *plan, const uint64_t *d_packed,
                                      uint8_t *d_logical, void *stream);

/* ------------------------------------------------------------------ */
/* learned dispatch: the cost model                                      */
/* ------------------------------------------------------------------ */
/* No counterpart in the reference.  A small MLP predicts the log2 running
 * time (microseconds) of each configuration of a request -- a variant with
 * its tuning fields, or for a matrix inside a batched launch the engine
 * that runs it -- from the request's shape, density and batch mix; the
 * dispatcher takes the fastest prediction.  It only chooses how a result is
 * computed: every configuration returns the same bits.
 * Inputs (MELA_MLP_IN): log2 m, log2 n, log2 p (products), density, the op
 * (rank, null space, product, batched rank + null space: one-hot), log2 of
 * the number of matrices in the batch, and the batch mix: the mean
 * log2(m * n) over the batch.  Outputs: one per configuration of the op
 * (mela_costmodel_config).  Parameters: one float array
 * W1[IN][H1] b1[H1] W2[H1][H2] b2[H2] W3[H2][OUT] b3[OUT]. */
#define MELA_MLP_IN 10
#define MELA_MLP_H1 32
#define MELA_MLP_H2 32
#define MELA_MLP_OUT 10
#define MELA_MLP_PARAMS 1738
typedef enum { MELA_OP_RANK = 0, MELA_OP_NULL = 1, MELA_OP_MATMUL = 2, MELA_OP_BATCH = 3 } mela_op;

/* Configurations of an op, in the model's output order: their count, and
 * the variant argument of configuration `index` (for MELA_OP_BATCH the
 * batch engine: 0 = a CTA, 1 = a 128-thread group, 2 = a warp per matrix);
 * -1 when out of range. */
int32_t mela_costmodel_config_count(int32_t op);
int32_t mela_costmodel_config(int32_t op, int32_t index);
/* Y (N x OUT) = network(X (N x IN)) on the device. */
mela_status mela_mlp_forward(const float *d_params, const float *d_X, int64_t N, float *d_Y,
                             void *stream);
/* d_grad = gradient of the masked mean squared error between the network's
 * outputs and targets T (N x OUT, mask 1 where observed), scaled by inv_count
 * = 1/(observed count); d_loss_sum (optional) = sum of squared errors. */
mela_status mela_mlp_gradient(const float *d_params, const float *d_X, const float *d_T,
                              const float *d_mask, int64_t N, float inv_count, float *d_grad,
                              float *d_loss_sum, void *stream);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8); step counts from 1. */
mela_status mela_mlp_adam_step(float *d_params, const float *d_grad, float *d_m1, float *d_m2,
                               int64_t step, float lr, void *stream);
/* Install (or, with NULL, remove) the dispatch model from host memory. */
mela_status mela_costmodel_load(const float *h_params);
/* Configuration index the installed model picks for a request, or -1 when
 * none is installed (the dispatcher then uses its fixed rule).  Single calls
 * pass batch_count = 1 and batch_log2_cells = log2(m * n). */
int32_t mela_costmodel_choose(int32_t op, int64_t m, int64_t n, int64_t p, double density,
                              int64_t batch_count, double batch_log2_cells);
/* The installed model's predicted log2 microseconds of every configuration
 * of the request into y (mela_costmodel_config_count(op) values); returns
 * that count, or -1 when no model is installed. */
int32_t mela_costmodel_predict(int32_t op, int64_t m, int64_t n, int64_t p, double density,
                               int64_t batch_count, double batch_log2_cells, float *y);
/* What an AUTO call decides before it sees the data (ops rank, null space,
 * product): the configuration index whose worst predicted loss over
 * densities 0.001, 0.01, 0.1 and 0.5 is smallest, and in *measure whether
 * that loss exceeds the cost of measuring the density (about 15 us), in
 * which case the call counts the input's ones and asks the model again.
 * -1 without a model. */
int32_t mela_costmodel_plan(int32_t op, int64_t m, int64_t n, int64_t p, int32_t *measure);
/* The variant argument the calling thread's last AUTO call resolved to (-1
 * before any), and in *density the density it measured on the device for
 * the choice, or a negative value when none was needed (mela_costmodel_plan). */
int32_t mela_dispatch_last(double *density);
/* The MELA_MLP_IN input features of a request. */
void mela_costmodel_features(int32_t op, int64_t m, int64_t n, int64_t p, double density,
                             int64_t batch_count, double batch_log2_cells, float *x);
/* Number of ones of the packed m x n device matrix into *d_count (device),
 * stream-ordered: the density the dispatcher feeds the model.  The AUTO
 * variants of mela_dev_matmul / mela_dev_rank / mela_dev_rref measure it
 * this way when a model is installed and its choice depends on the density
 * -- which waits for the stream (the count is read back) unless the stream
 * is being captured, where 0.5 is assumed. */
mela_status mela_dev_popcount(const uint64_t *dM, int64_t ld, int64_t m, int64_t n, int64_t *d_count,
                              void *stream);

/* ------------------------------------------------------------------ */
/* allocation-free product                                              */
/* ------------------------------------------------------------------ */
/* No counterpart in the reference library.  For callers that are given
 * device buffers but may not allocate device memory themselves (a plugin
 * whose host application owns the GPU memory budget, or a latency-critical
 * loop that cannot take cudaMalloc's implicit synchronisation): the plain
 * AND+popcount product C = A*B with its one scratch buffer (B transposed)
 * held in a fixed 16 MiB array inside the library instead of a caller
 * workspace.  Limit: n * (ceil(k/64) rounded up to even) * 8 bytes must not
 * exceed mela_static_scratch_bytes(); larger products return
 * MELA_ERR_UNSUPPORTED.  The first call on a device looks up the array's
 * device address, so make it before any stream capture.  All calls share the
 * array: calls that overlap on the GPU race, so serialise them. */
size_t mela_static_scratch_bytes(void);
mela_status mela_dev_matmul_plain_static(const uint64_t *dA, int64_t lda, const uint64_t *dB,
                                         int64_t ldb, uint64_t *dC, int64_t ldc, int64_t m,
                                         int64_t k, int64_t n, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MELA_H */
