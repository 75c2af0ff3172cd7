// mela_host.h -- host-layer helpers shared by the C-ABI translation units.
#pragma once

#include "mela_common.cuh"

namespace mela {

// Stream-ordered device buffer from the default memory pool, released on
// the same stream when it goes out of scope.
struct DevBuf {
    void *p = nullptr;
    cudaStream_t s = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf();
    mela_status alloc(size_t bytes, cudaStream_t st);
};

// The calling thread's library stream on the current device.
mela_status host_stream(cudaStream_t *s);
// The calling thread's side stream on the current device: work forked from a
// caller's stream (through an event) and joined back to it before returning.
mela_status side_stream(cudaStream_t *s);
// A second side stream of the calling thread, for work forked beside the first.
mela_status aux_stream(cudaStream_t *s);
// The calling thread's stream for capturing launch sequences into CUDA graphs
// (a graph is captured there and launched on the caller's stream).
mela_status capture_stream(cudaStream_t *s);
// Synchronise `s` and turn a device-side wait timeout into MELA_ERR_TIMEOUT.
mela_status finish(cudaStream_t s);

// Row pitch in words, rounded up to an even count (16-byte rows).
i64 even_words(i64 bits);

// A variant argument split into its base variant and tuning fields
// (MELA_TUNE_K / MELA_TUNE_TILE of include/mela.h), defaults filled in.
struct Tuning {
    int base;      // mela_gemm_variant or mela_elim_variant
    int k;         // Four-Russians table width (M4RI forms)
    int row_tile;  // rows per update CTA (blocked elimination)
    int tc_tile;   // tensor-core products: 0 default, 1 single CTAs, 2 CTA pairs
};
// false when a field is out of range for the base variant
bool decode_elim_variant(int32_t v, Tuning *t);
bool decode_gemm_variant(int32_t v, Tuning *t);

// Configurations of an op in the cost model's output order (dispatch.cu).
int config_count(int op);
int32_t config_variant(int op, int index);
// AUTO -> a concrete variant argument: the installed model's choice for the
// input's measured density, else the fixed rule.  Other variants pass through.
int32_t resolve_gemm_variant(int32_t variant, const u64 *A, i64 lda, i64 m, i64 k, i64 n, cudaStream_t s);
int32_t resolve_elim_variant(int32_t variant, const u64 *M, i64 ld, i64 m, i64 n, int rref, cudaStream_t s);
int32_t fixed_gemm_variant(i64 m, i64 k, i64 n);
int32_t fixed_elim_variant(i64 m, i64 n);
// Ones of a packed matrix, stream-ordered, into d_count (device).
mela_status launch_popcount(const u64 *M, i64 ld, i64 m, i64 n, long long *d_count, cudaStream_t s);
// Density of a packed device matrix, read back (waits for s); 0.5 while s is
// being captured or on failure.
double measure_density(const u64 *M, i64 ld, i64 m, i64 n, cudaStream_t s);

// Learned cost model (mlp.cu): configuration index for the request, or -1
// without a model.
bool costmodel_loaded();
// Changes whenever a model is installed or removed (dispatch caches key on it).
unsigned costmodel_generation();
int costmodel_choose(int op, double m, double n, double p, double density, double batch_count,
                     double batch_log2_cells);
// Predicted log2 microseconds of every configuration of the request
// (config_count(op) values); false without a model.
bool costmodel_predict(int op, double m, double n, double p, double density, double batch_count,
                       double batch_log2_cells, float *y);
void costmodel_features(int op, double m, double n, double p, double density, double batch_count,
                        double batch_log2_cells, float *x);
// The predictions at kCostProbes densities dens[] at once; false without a model.
constexpr int kCostProbes = 4;
bool costmodel_predict_densities(int op, double m, double n, double p, const double *dens, double batch_count,
                                 double batch_log2_cells, float (*y)[MELA_MLP_OUT]);
size_t gemm_workspace(int variant, i64 m, i64 k, i64 n);
mela_status gemm_prepare(int variant, const u64 *A, i64 lda, const u64 *B, i64 ldb, i64 m, i64 k,
                         i64 n, void *ws, size_t ws_bytes, cudaStream_t s);
mela_status gemm_run(int variant, const u64 *A, i64 lda, const u64 *B, i64 ldb, u64 *C, i64 ldc,
                     i64 m, i64 k, i64 n, void *ws, size_t ws_bytes, cudaStream_t s);
mela_status gemm_device(int variant, const u64 *A, i64 lda, const u64 *B, i64 ldb, u64 *C, i64 ldc,
                        i64 m, i64 k, i64 n, void *ws, size_t ws_bytes, cudaStream_t s);

// Rank / null-space basis of a packed device matrix (overwritten), shared by
// the dense and sparse host entry points.
mela_status rank_of_packed(u64 *P, i64 ld, i64 m, i64 n, int variant, cudaStream_t s, double *rank);
mela_status null_of_packed(u64 *P, i64 ld, i64 m, i64 n, int variant, mela_alloc_fn alloc, void *ctx,
                           int64_t *nullity, cudaStream_t s);

// Copy a host MATLAB array to the device and pack it into dP (ld words/row).
mela_status upload_and_pack(const mela_host_matrix *M, u64 *dP, i64 ld, cudaStream_t s,
                            DevBuf &staging);

}  // namespace mela
