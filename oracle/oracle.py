"""TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path.

ctypes front end for two CPU implementations of the reference's GF(2)
algorithms:

* ``liboracle.so`` -- this directory's C restatement (mela_oracle.c), each
  function citing the reference file:line it follows;
* ``_ref/<isa>/mela_*.so`` -- the reference's own MEX gateways
  (HCPhy/mex_linear_algebra src/mela_*.c) compiled unmodified against the
  non-MATLAB MEX host by ``oracle/Makefile``.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module.  The library under test never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")

NAMES = ("mela_matmul_gf2", "mela_matmul_m4ri", "mela_rank_gf2",
         "mela_rank_m4ri", "mela_null_gf2", "mela_null_m4ri")

_lib = None


def lib():
    """Load liboracle.so (built by ``make -C oracle``)."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle not built: {path} missing (run make -C oracle)")
        L = C.CDLL(path)
        i64, u64 = C.c_int64, C.c_uint64
        L.orc_stream_key.argtypes = [u64, u64]
        L.orc_stream_key.restype = u64
        L.orc_rand_word.argtypes = [u64, u64]
        L.orc_rand_word.restype = u64
        L.orc_rand_words.argtypes = [u64, u64, u64, i64, _u64p]
        L.orc_rand_dense.argtypes = [u64, u64, i64, i64, _u64p, i64]
        L.orc_parity_double.argtypes = [C.c_double]
        L.orc_parity_double.restype = C.c_int
        L.orc_pack_colmajor.argtypes = [C.c_int, i64, i64, C.c_void_p, _u64p, i64]
        L.orc_unpack_colmajor.argtypes = [_u64p, i64, i64, i64, _u8p]
        L.orc_matmul.argtypes = [_u64p, i64, _u64p, i64, _u64p, i64, i64, i64, i64]
        L.orc_matmul_m4ri.argtypes = [_u64p, i64, _u64p, i64, _u64p, i64, i64, i64, i64, C.c_int]
        L.orc_rank_ge.argtypes = [_u64p, i64, i64, i64]
        L.orc_rank_ge.restype = i64
        L.orc_rank_m4ri.argtypes = [_u64p, i64, i64, i64, C.c_int]
        L.orc_rank_m4ri.restype = i64
        L.orc_rref.argtypes = [_u64p, i64, i64, i64, _i64p]
        L.orc_rref.restype = i64
        L.orc_echelon_m4ri.argtypes = [_u64p, i64, i64, i64, C.c_int, _i64p]
        L.orc_echelon_m4ri.restype = i64
        L.orc_null_backsub.argtypes = [_u64p, i64, i64, _i64p, i64, _u64p, i64]
        L.orc_null_backsub.restype = i64
        L.orc_pivot_columns.argtypes = [_u64p, i64, i64, i64, _i64p]
        L.orc_pivot_columns.restype = i64
        L.orc_num_threads.restype = C.c_int
        _lib = L
    return _lib


def words(n: int) -> int:
    return (n + 63) // 64


# ---------------------------------------------------------------- generator
def rand_dense(seed: int, stream: int, m: int, n: int, ld: int | None = None) -> np.ndarray:
    ld = words(n) if ld is None else ld
    out = np.zeros((max(m, 0), ld), dtype=np.uint64)
    if m and ld:
        lib().orc_rand_dense(seed, stream, m, n, out, ld)
    return out


# ---------------------------------------------------------------- packing
def pack(a: np.ndarray, ld: int | None = None) -> np.ndarray:
    """Column-major MATLAB-style array (bool/uint8 logical or float64) -> packed rows."""
    a = np.asfortranarray(a)
    m, n = a.shape
    ld = words(n) if ld is None else ld
    out = np.zeros((m, ld), dtype=np.uint64)
    if m == 0 or n == 0:
        return out
    if a.dtype == np.float64:
        kind = 1
    else:
        kind = 0
        a = np.asfortranarray(a.view(np.uint8) if a.dtype == np.bool_ else a.astype(np.uint8))
    lib().orc_pack_colmajor(kind, m, n, a.ctypes.data, out, ld)
    return out


def unpack(p: np.ndarray, m: int, n: int) -> np.ndarray:
    """Packed rows -> column-major logical (numpy bool, Fortran order)."""
    out = np.zeros(m * n, dtype=np.uint8)
    if m and n:
        lib().orc_unpack_colmajor(np.ascontiguousarray(p), p.shape[1], m, n, out)
    return out.reshape((m, n), order="F").view(np.bool_)


# ---------------------------------------------------------------- kernels
def matmul(A: np.ndarray, B: np.ndarray, m: int, k: int, n: int, m4ri_k: int = 0) -> np.ndarray:
    A = np.ascontiguousarray(A)
    B = np.ascontiguousarray(B)
    C_ = np.zeros((m, words(n)), dtype=np.uint64)
    if m and n:
        if k == 0:
            return C_
        if m4ri_k:
            lib().orc_matmul_m4ri(A, A.shape[1], B, B.shape[1], C_, C_.shape[1], m, k, n, m4ri_k)
        else:
            lib().orc_matmul(A, A.shape[1], B, B.shape[1], C_, C_.shape[1], m, k, n)
    return C_


def rank(M: np.ndarray, m: int, n: int, m4ri_k: int = 0) -> int:
    W = np.ascontiguousarray(M).copy()
    if m == 0 or n == 0:
        return 0
    if m4ri_k:
        return int(lib().orc_rank_m4ri(W, W.shape[1], m, n, m4ri_k))
    return int(lib().orc_rank_ge(W, W.shape[1], m, n))


def rref(M: np.ndarray, m: int, n: int):
    """Full RREF (reference gf2_rref_standard): returns (R, pivots)."""
    W = np.ascontiguousarray(M).copy()
    piv = np.zeros(max(min(m, n), 1), dtype=np.int64)
    r = 0
    if m and n:
        r = int(lib().orc_rref(W, W.shape[1], m, n, piv))
    return W, piv[:r].copy()


def echelon_m4ri(M: np.ndarray, m: int, n: int, k: int = 8):
    W = np.ascontiguousarray(M).copy()
    piv = np.zeros(max(min(m, n), 1), dtype=np.int64)
    r = 0
    if m and n:
        r = int(lib().orc_echelon_m4ri(W, W.shape[1], m, n, k, piv))
    return W, piv[:r].copy()


def null_basis_packed(M: np.ndarray, m: int, n: int, method: str = "gf2") -> np.ndarray:
    """Null-space basis Zt (nullity x words(n)) by the reference's steps."""
    if method == "m4ri":
        R, piv = echelon_m4ri(M, m, n, 8)
    else:
        R, piv = rref(M, m, n)
    r = len(piv)
    f = n - r
    Zt = np.zeros((f, words(n)), dtype=np.uint64)
    if f and n:
        Rc = np.ascontiguousarray(R) if R.size else np.zeros((1, words(n)), dtype=np.uint64)
        pv = piv if r else np.zeros(1, dtype=np.int64)
        lib().orc_null_backsub(Rc, Rc.shape[1], n, pv, r, Zt, Zt.shape[1])
    return Zt


def null_logical(H: np.ndarray, method: str = "gf2") -> np.ndarray:
    """n x nullity logical (Fortran order) like the reference gateway output."""
    m, n = H.shape
    P = pack(H)
    Zt = null_basis_packed(P, m, n, method)
    f = Zt.shape[0]
    # column i of Z is row i of Zt
    return unpack(Zt, f, n).T.copy(order="F") if f else np.zeros((n, 0), dtype=np.bool_, order="F")


def num_threads() -> int:
    return int(lib().orc_num_threads())


# ---------------------------------------------------------------- reference gateways
class _MxArray(C.Structure):
    _fields_ = [("classid", C.c_int), ("m", C.c_size_t), ("n", C.c_size_t),
                ("data", C.c_void_p), ("sparse", C.c_int), ("owns_data", C.c_int)]


MX_LOGICAL, MX_DOUBLE, MX_SINGLE, MX_INT32 = 3, 6, 7, 12


def host_isa() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
        if " avx512f" in flags and " avx512bw" in flags and " avx512dq" in flags:
            return "avx512"
    except OSError:
        pass
    return "avx2"


_ref_libs: dict = {}


def ref_available(isa: str | None = None) -> bool:
    isa = isa or host_isa()
    return all(os.path.exists(os.path.join(HERE, "_ref", isa, nm + ".so")) for nm in NAMES)


def _ref(name: str, isa: str | None = None):
    isa = isa or host_isa()
    key = (name, isa)
    if key not in _ref_libs:
        path = os.path.join(HERE, "_ref", isa, name + ".so")
        if not os.path.exists(path):
            raise RuntimeError(f"reference gateway not built: {path}")
        L = C.CDLL(path, mode=os.RTLD_LOCAL if hasattr(os, "RTLD_LOCAL") else 0)
        L.mexhost_call.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.POINTER(_MxArray)), C.c_int,
                                   C.POINTER(C.POINTER(_MxArray)), C.c_char_p, C.c_size_t,
                                   C.c_char_p, C.c_size_t]
        L.mexhost_call.restype = C.c_int
        L.mexhost_wrap.argtypes = [C.c_int, C.c_size_t, C.c_size_t, C.c_void_p, C.c_int]
        L.mexhost_wrap.restype = C.POINTER(_MxArray)
        L.mxDestroyArray.argtypes = [C.POINTER(_MxArray)]
        _ref_libs[key] = L
    return _ref_libs[key]


class MexError(Exception):
    def __init__(self, ident: str, msg: str):
        super().__init__(msg)
        self.ident = ident
        self.msg = msg


def mx_class_of(a: np.ndarray) -> int:
    if a.dtype == np.bool_:
        return MX_LOGICAL
    if a.dtype == np.float64:
        return MX_DOUBLE
    if a.dtype == np.float32:
        return MX_SINGLE
    if a.dtype == np.int32:
        return MX_INT32
    raise TypeError(a.dtype)


def call_gateway(L, args, nlhs: int = 1, sparse=()):
    """Call the gateway `mexFunction` of the loaded library `L` with numpy
    arrays (column-major); returns the list of outputs as numpy arrays or
    raises MexError with the gateway's identifier and message."""
    keep = []
    prhs_t = C.POINTER(_MxArray) * max(len(args), 1)
    prhs = prhs_t()
    for i, a in enumerate(args):
        a = np.asfortranarray(a)
        keep.append(a)
        prhs[i] = L.mexhost_wrap(mx_class_of(a), a.shape[0], a.shape[1], a.ctypes.data,
                                 1 if i in sparse else 0)
    plhs_t = C.POINTER(_MxArray) * max(nlhs, 1)
    plhs = plhs_t()
    eid = C.create_string_buffer(256)
    emsg = C.create_string_buffer(1024)
    fn = C.cast(L.mexFunction, C.c_void_p)
    rc = L.mexhost_call(fn, nlhs, plhs, len(args), prhs, eid, 256, emsg, 1024)
    outs = []
    try:
        if rc != 0:
            raise MexError(eid.value.decode(), emsg.value.decode())
        for i in range(nlhs):
            p = plhs[i]
            if not p:
                outs.append(None)
                continue
            arr = p.contents
            m, n = arr.m, arr.n
            if arr.classid == MX_LOGICAL:
                buf = (C.c_uint8 * max(m * n, 1)).from_address(arr.data)
                o = np.frombuffer(buf, dtype=np.uint8, count=m * n).copy()
                o = o.reshape((m, n), order="F").view(np.bool_)
            else:
                buf = (C.c_double * max(m * n, 1)).from_address(arr.data)
                o = np.frombuffer(buf, dtype=np.float64, count=m * n).copy().reshape((m, n), order="F")
            outs.append(o)
            L.mxDestroyArray(p)
    finally:
        for i in range(len(args)):
            L.mxDestroyArray(prhs[i])
    return outs


def ref_call(name: str, *args, nlhs: int = 1, sparse=(), isa: str | None = None):
    """Run the reference gateway `name` on numpy inputs."""
    return call_gateway(_ref(name, isa), args, nlhs=nlhs, sparse=sparse)
