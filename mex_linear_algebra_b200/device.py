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


def device_error_flags(clear: bool = True) -> int:
    import ctypes as C
    v = C.c_uint32(0)
    check(lib().mela_device_error_flags(C.byref(v), 1 if clear else 0))
    return int(v.value)
