// elim.h -- elimination and null-space launchers (elim.cu).
#pragma once

#include "mela_common.cuh"

namespace mela {

struct ElimLayout {
    size_t state, stamp, ps, rbuf, cand, gb, ysnap, total;
};
struct NullLayout {
    size_t pm, pbase, free, rc, rt, total;
    i64 ldr;
};

ElimLayout elim_layout(i64 m, i64 n);
size_t elim_workspace(i64 m, i64 n);

// Rank (rref = 0) or reduced row echelon form (rref = 1) of the packed m x n
// matrix M, in place.  Writes the rank to d_rank, the pivot columns to d_piv
// and the physical row of each RREF row to d_prow (both min(m,n) entries).
mela_status elim_device(int variant, u64 *M, i64 ld, i64 m, i64 n, int rref, long long *d_rank,
                        long long *d_piv, long long *d_prow, void *ws, size_t ws_bytes,
                        cudaStream_t s);

// Tensor-core form (elim_tc.cu): same contract as elim_device.
size_t elim_tc_workspace(i64 m, i64 n);
mela_status elim_tc_device(u64 *M, i64 ld, i64 m, i64 n, int rref, long long *d_rank, long long *d_piv,
                           long long *d_prow, void *ws, size_t ws_bytes, cudaStream_t s);

NullLayout null_layout(i64 n, i64 rank);
// Null-space basis from an RREF: Zt row i = e_{f_i} + sum_p R_p[f_i] e_{piv[p]},
// free columns f_i ascending (n - rank rows of ldz words).
mela_status null_basis_device(const u64 *M, i64 ld, i64 m, i64 n, i64 rank, const long long *d_piv,
                              const long long *d_prow, u64 *Zt, i64 ldz, void *ws, size_t ws_bytes,
                              cudaStream_t s);

// Packed rows -> row-major bytes (rows x n).
mela_status launch_unpack_rows(const u64 *P, i64 ld, i64 rows, i64 n, unsigned char *out, cudaStream_t s);

}  // namespace mela
