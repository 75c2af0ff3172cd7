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

int choose_gemm_variant(i64 m, i64 k, i64 n);
// Learned cost model: variant index 0..2 for the request, or -1 without a model.
int costmodel_choose(int op, double m, double n, double p, double density);
void costmodel_features(int op, double m, double n, double p, double density, float *x);
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
