"""Packed, stream-ordered device entry points over torch CUDA tensors.

Torch supplies device memory and the current stream; every operation is a
call into ``libmela_b200.so``.  Packed matrices are int64 tensors of shape
(rows, ld) holding the uint64 words (row-major, bit j of row i in word j//64
at bit j%64).
"""
from __future__ import annotations

import torch

from . import _lib
from ._lib import check, lib


def words(n: int) -> int:
    return (n + 63) // 64


def _ptr(t) -> int:
    return t.data_ptr() if t is not None else 0


def _stream(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def empty_packed(rows: int, cols: int, ld: int | None = None, device="cuda") -> torch.Tensor:
    ld = words(cols) if ld is None else ld
    return torch.empty((rows, ld), dtype=torch.int64, device=device)


def rand_dense(seed: int, stream_id: int, m: int, n: int, ld: int | None = None, out=None,
               stream=None) -> torch.Tensor:
    ld = words(n) if ld is None else ld
    out = empty_packed(m, n, ld) if out is None else out
    check(lib().mela_dev_rand_dense(seed, stream_id, m, n, _ptr(out), ld, _stream(stream)))
    return out


def pack(colmajor: torch.Tensor, m: int, n: int, ld: int | None = None, out=None, stream=None):
    """Column-major logical (uint8/bool) or float64 device array -> packed rows."""
    kind = _lib.KIND_DOUBLE if colmajor.dtype == torch.float64 else _lib.KIND_LOGICAL
    ld = words(n) if ld is None else ld
    out = empty_packed(m, n, ld) if out is None else out
    check(lib().mela_dev_pack(kind, m, n, _ptr(colmajor), _ptr(out), ld, _stream(stream)))
    return out


def unpack(packed: torch.Tensor, m: int, n: int, out=None, stream=None) -> torch.Tensor:
    """Packed rows -> column-major logical bytes (flat uint8 tensor of m*n)."""
    out = torch.empty(m * n, dtype=torch.uint8, device=packed.device) if out is None else out
    check(lib().mela_dev_unpack(_ptr(packed), packed.shape[1], m, n, _ptr(out), _stream(stream)))
    return out


def transpose(packed: torch.Tensor, rows: int, cols: int, out=None, stream=None) -> torch.Tensor:
    out = empty_packed(cols, rows) if out is None else out
    check(lib().mela_dev_transpose(_ptr(packed), packed.shape[1], rows, cols, _ptr(out),
                                   out.shape[1], _stream(stream)))
    return out


def matmul_workspace(variant: str | int, m: int, k: int, n: int) -> int:
    v = _lib.GEMM_VARIANTS[variant] if isinstance(variant, str) else variant
    return int(lib().mela_matmul_workspace_size(v, m, k, n))


def matmul(A: torch.Tensor, B: torch.Tensor, m: int, k: int, n: int, variant: str | int = "auto",
           out=None, workspace=None, stream=None) -> torch.Tensor:
    """Packed C = A*B over GF(2) (A: m x k, B: k x n)."""
    v = _lib.GEMM_VARIANTS[variant] if isinstance(variant, str) else variant
    out = empty_packed(m, n) if out is None else out
    wsb = matmul_workspace(v, m, k, n)
    if workspace is None and wsb:
        workspace = torch.empty(wsb, dtype=torch.uint8, device=A.device)
    check(lib().mela_dev_matmul(v, _ptr(A), A.shape[1], _ptr(B), B.shape[1], _ptr(out),
                                out.shape[1], m, k, n, _ptr(workspace),
                                workspace.numel() if workspace is not None else 0,
                                _stream(stream)))
    return out


def null_verify(A: torch.Tensor, m: int, n: int, Zt: torch.Tensor, f: int, workspace=None,
                stream=None) -> int:
    """Number of rows i of A (packed m x n) with A_i . z != 0 for some row z
    of Zt (packed f x n, a null-space basis as mela_dev_null_basis writes
    it); 0 means A Z = 0.  Computed on the device."""
    dev = A.device if A.numel() else Zt.device
    wsb = int(lib().mela_null_verify_workspace_size(m, f))
    if workspace is None and wsb:
        workspace = torch.empty(wsb, dtype=torch.uint8, device=dev)
    bad = torch.zeros(1, dtype=torch.int64, device=dev)
    lda = A.shape[1] if A.dim() == 2 else words(n)
    ldz = Zt.shape[1] if Zt.dim() == 2 else words(n)
    check(lib().mela_dev_null_verify(_ptr(A), lda, m, n, _ptr(Zt), ldz, f, _ptr(bad), _ptr(workspace),
                                     workspace.numel() if workspace is not None else 0, _stream(stream)))
    return int(bad.item())


def device_error_flags(clear: bool = True) -> int:
    import ctypes as C
    v = C.c_uint32(0)
    check(lib().mela_device_error_flags(C.byref(v), 1 if clear else 0))
    return int(v.value)


class BatchPlan:
    """Batched rank + null space (mela_batch_* entry points).

    ``shapes``: sequence of (m, n).  Inputs are packed back to back in the
    order given (``in_offsets``, words); the null-space bases come back in a
    buffer with room for n rows of ceil(n/64) words per matrix
    (``z_offsets``).
    """

    def __init__(self, shapes, force_class: int = -1, densities=None):
        """force_class: the engine policy -- -1 the size rule, 0/1/2 that
        engine wherever it fits, -2 the installed cost model's choice per
        matrix (from its shape, ``densities`` and the batch mix)."""
        import ctypes as C
        import numpy as np
        self.shapes = np.asarray(shapes, dtype=np.int64).reshape(-1, 2)
        m, n = self.shapes[:, 0], self.shapes[:, 1]
        wc = (n + 63) // 64
        self.wc = wc
        sizes = m * wc
        self.in_offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        zsz = n * wc
        self.z_offsets = np.concatenate([[0], np.cumsum(zsz)[:-1]]).astype(np.int64)
        self.in_words = int(sizes.sum())
        self.z_words = int(zsz.sum())
        self.logical_bytes = int((m * n).sum())
        cnt = len(self.shapes)
        items = (_lib.BatchItem * max(cnt, 1))()
        for i in range(cnt):
            items[i] = _lib.BatchItem(int(m[i]), int(n[i]), int(self.in_offsets[i]), int(self.z_offsets[i]))
        self._plan = C.c_void_p()
        self._items = items
        if densities is None:
            check(lib().mela_batch_plan_create_ex(items, cnt, None, force_class, C.byref(self._plan)))
        else:
            dens = np.ascontiguousarray(densities, dtype=np.float64)
            if dens.shape != (cnt,):
                raise ValueError("one density per matrix")
            check(lib().mela_batch_plan_create_ex(items, cnt, dens.ctypes.data, force_class,
                                                  C.byref(self._plan)))
        self.count = cnt

    def densities(self, d_packed, stream=None):
        """Fraction of ones of every matrix of a packed batch (in_offsets
        layout), counted on the device."""
        import numpy as np
        cnt = torch.zeros(max(self.count, 1), dtype=torch.int64, device=d_packed.device)
        check(lib().mela_batch_popcounts(self._items, self.count, _ptr(d_packed), _ptr(cnt), _stream(stream)))
        ones = cnt[:self.count].cpu().numpy().astype(np.float64)
        cells = (self.shapes[:, 0] * self.shapes[:, 1]).astype(np.float64)
        return np.where(cells > 0, ones / np.maximum(cells, 1), 0.0)

    def stats(self):
        import ctypes as C
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().mela_batch_plan_stats(self._plan, C.byref(a), C.byref(b), C.byref(c)))
        return {"cta": a.value, "group128": b.value, "warp": c.value}

    def outputs(self, device="cuda"):
        ranks = torch.empty(max(self.count, 1), dtype=torch.int64, device=device)
        zt = torch.empty(max(self.z_words, 1), dtype=torch.int64, device=device)
        return ranks, zt

    def run(self, d_in, ranks=None, zt=None, use_graph: bool = True, stream=None):
        if ranks is None:
            ranks, zt = self.outputs(d_in.device)
        check(lib().mela_batch_rank_null(self._plan, _ptr(d_in), _ptr(zt), _ptr(ranks),
                                         1 if use_graph else 0, _stream(stream)))
        return ranks, zt

    def run_logical(self, d_logical, ranks=None, zt=None, use_graph: bool = True, stream=None):
        if ranks is None:
            ranks, zt = self.outputs(d_logical.device)
        check(lib().mela_batch_rank_null_logical(self._plan, _ptr(d_logical), _ptr(zt), _ptr(ranks),
                                                 1 if use_graph else 0, _stream(stream)))
        return ranks, zt

    def pack_logical(self, d_logical, out=None, stream=None):
        """All matrices from logical column-major bytes to packed rows (in_offset layout)."""
        out = torch.zeros(max(self.in_words, 1), dtype=torch.int64, device=d_logical.device) \
            if out is None else out
        check(lib().mela_batch_pack_logical(self._plan, _ptr(d_logical), _ptr(out), _stream(stream)))
        return out

    def unpack_logical(self, d_packed, out=None, stream=None):
        """All matrices from packed rows to their logical column-major bytes."""
        out = torch.empty(max(self.logical_bytes, 1), dtype=torch.uint8, device=d_packed.device) \
            if out is None else out
        check(lib().mela_batch_unpack_logical(self._plan, _ptr(d_packed), _ptr(out), _stream(stream)))
        return out

    def basis(self, zt_host, ranks_host, i):
        """Packed basis of matrix i (nullity x ceil(n/64) uint64) from host copies."""
        n = int(self.shapes[i, 1])
        f = n - int(ranks_host[i])
        wc = int(self.wc[i])
        o = int(self.z_offsets[i])
        return zt_host[o:o + f * wc].reshape(f, wc)

    def close(self):
        if getattr(self, "_plan", None) and self._plan.value:
            lib().mela_batch_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
