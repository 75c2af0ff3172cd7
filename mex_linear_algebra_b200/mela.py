"""The six reference functions with MATLAB semantics, on numpy arrays.

``mela_matmul_gf2(A, B)``, ``mela_matmul_m4ri(A, B)``, ``mela_rank_gf2(A)``,
``mela_rank_m4ri(A)``, ``mela_null_gf2(H)``, ``mela_null_m4ri(H)`` behave as
the MEX functions of HCPhy/mex_linear_algebra (src/mela_*.c): inputs are
logical (numpy bool) or double (float64, read as ``((int)x) & 1``) arrays,
products and null-space bases come back as logical arrays (Fortran order,
like MATLAB's column-major storage), ranks as a float.  Argument errors
raise :class:`MexError` with the reference's identifier and message.

Each call goes through ``mela_gateway`` in libmela_b200.so -- the same code
the MATLAB gateways use -- and computes on the GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import lib


class MexError(Exception):
    """A gateway error: ``identifier`` (may be empty) and ``message``."""

    def __init__(self, identifier: str, message: str):
        super().__init__(message)
        self.identifier = identifier
        self.message = message


def _host_matrix(a, keep: list):
    sparse = 0
    if hasattr(a, "toarray") and hasattr(a, "nnz"):  # scipy.sparse
        sparse = 1
        a = a.toarray()
    a = np.asarray(a)
    if a.ndim != 2:
        a = a.reshape((a.shape[0] if a.ndim else 1, -1))
    if a.dtype == np.bool_:
        kind = _lib.KIND_LOGICAL
    elif a.dtype == np.float64:
        kind = _lib.KIND_DOUBLE
    else:
        kind = _lib.KIND_OTHER
    a = np.asfortranarray(a)
    keep.append(a)
    return _lib.HostMatrix(kind, sparse, a.shape[0], a.shape[1],
                           a.ctypes.data if a.size else None)


def _call(fn: int, args, nlhs: int = 1):
    keep: list = []
    n = len(args)
    arr = (_lib.HostMatrix * max(n, 1))()
    for i, a in enumerate(args):
        arr[i] = _host_matrix(a, keep)
    outs: dict = {}

    def alloc(ctx, index, kind, rows, cols):
        if kind == _lib.KIND_DOUBLE:
            o = np.zeros((rows, cols), dtype=np.float64, order="F")
        else:
            o = np.zeros((rows, cols), dtype=np.bool_, order="F")
        outs[index] = o
        return o.ctypes.data if o.size else None

    cb = _lib.GATEWAY_ALLOC_FN(alloc)
    err = _lib.GatewayError()
    rc = lib().mela_gateway(fn, nlhs, n, arr, cb, None, C.byref(err))
    if rc:
        raise MexError(err.id.decode(), err.msg.decode())
    return outs.get(0)


def mela_matmul_gf2(A, B):
    """C = A*B over GF(2) (src/mela_matmul_gf2.c)."""
    return _call(_lib.FN_MATMUL_GF2, (A, B))


def mela_matmul_m4ri(A, B):
    """C = A*B over GF(2), Four-Russians kernel (src/mela_matmul_m4ri.c)."""
    return _call(_lib.FN_MATMUL_M4RI, (A, B))


def mela_rank_gf2(A) -> float:
    """Rank over GF(2) (src/mela_rank_gf2.c)."""
    return float(_call(_lib.FN_RANK_GF2, (A,))[0, 0])


def mela_rank_m4ri(A) -> float:
    """Rank over GF(2), Four-Russians elimination (src/mela_rank_m4ri.c)."""
    return float(_call(_lib.FN_RANK_M4RI, (A,))[0, 0])


def mela_null_gf2(H):
    """n x nullity logical null-space basis (src/mela_null_gf2.c)."""
    return _call(_lib.FN_NULL_GF2, (H,))


def mela_null_m4ri(H):
    """Same basis through the Four-Russians elimination (src/mela_null_m4ri.c)."""
    return _call(_lib.FN_NULL_M4RI, (H,))


# ---------------------------------------------------------------- sparse input
# No counterpart in the reference (its gateways reject sparse arrays): rank and
# null space of a sparse matrix packed on the GPU from its CSC arrays.

def _host_csc(H, keep: list):
    """scipy.sparse matrix, or a tuple (colptr, rowidx, values or None, (rows, cols))."""
    if hasattr(H, "tocsc"):
        H = H.tocsc()
        colptr, rowidx, values, shape = H.indptr, H.indices, H.data, H.shape
    else:
        colptr, rowidx, values, shape = H
    colptr = np.ascontiguousarray(colptr, dtype=np.int64)
    rowidx = np.ascontiguousarray(rowidx, dtype=np.int64)
    kind = _lib.KIND_LOGICAL
    if values is not None:
        values = np.asarray(values)
        if values.dtype == np.bool_:
            values = np.ascontiguousarray(values.view(np.uint8))
        else:
            values = np.ascontiguousarray(values, dtype=np.float64)
            kind = _lib.KIND_DOUBLE
    keep.extend([colptr, rowidx, values])
    return _lib.HostCsc(kind, int(shape[0]), int(shape[1]), colptr.ctypes.data,
                        rowidx.ctypes.data if rowidx.size else None,
                        values.ctypes.data if values is not None and values.size else None)


def rank_csc(H) -> int:
    """Rank over GF(2) of a sparse matrix (scipy.sparse, or (colptr, rowidx,
    values, shape)); entries add mod 2, doubles read as ((int)x) & 1."""
    keep: list = []
    h = _host_csc(H, keep)
    r = C.c_int64(0)
    _lib.check(lib().mela_rank_csc(C.byref(h), C.byref(r)))
    return int(r.value)


def null_csc(H):
    """n x nullity logical null-space basis of a sparse matrix (the basis
    mela_null_gf2 returns for its dense form)."""
    keep: list = []
    h = _host_csc(H, keep)
    out = {}

    def alloc(ctx, rows, cols):
        a = np.zeros((rows, cols), dtype=np.bool_, order="F")
        out["z"] = a
        return a.ctypes.data if a.size else None

    cb = _lib.ALLOC_FN(alloc)
    f = C.c_int64(0)
    _lib.check(lib().mela_null_csc(C.byref(h), cb, None, C.byref(f)))
    return out["z"]


def call(name: str, *args, nlhs: int = 1):
    """Call a gateway by its MATLAB name with explicit argument counts
    (for reproducing argument-count errors)."""
    fn = {"mela_matmul_gf2": _lib.FN_MATMUL_GF2, "mela_matmul_m4ri": _lib.FN_MATMUL_M4RI,
          "mela_rank_gf2": _lib.FN_RANK_GF2, "mela_rank_m4ri": _lib.FN_RANK_M4RI,
          "mela_null_gf2": _lib.FN_NULL_GF2, "mela_null_m4ri": _lib.FN_NULL_M4RI}[name]
    out = _call(fn, args, nlhs=nlhs)
    if fn in (_lib.FN_RANK_GF2, _lib.FN_RANK_M4RI):
        return out
    return out
