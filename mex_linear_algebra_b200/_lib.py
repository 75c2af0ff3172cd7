"""ctypes binding of ``libmela_b200.so`` (the C ABI declared in include/mela.h).

The library is loaded from the package directory; if it is missing the
import fails loudly -- there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmela_b200.so")

# mela_status
OK, ERR_INVALID, ERR_SPARSE, ERR_DIM, ERR_TYPE, ERR_NOMEM, ERR_CUDA, ERR_TIMEOUT, \
    ERR_UNSUPPORTED, ERR_NO_DEVICE = range(10)
# mela_kind
KIND_LOGICAL, KIND_DOUBLE, KIND_OTHER = 0, 1, 2
# mela_gemm_variant
GEMM_AUTO, GEMM_PLAIN, GEMM_M4RI, GEMM_TC, GEMM_TC_FP4 = 0, 1, 2, 3, 4
GEMM_VARIANTS = {"auto": GEMM_AUTO, "plain": GEMM_PLAIN, "m4ri": GEMM_M4RI, "tc": GEMM_TC,
                 "tc_fp4": GEMM_TC_FP4}


# mela_function (gateway ids)
FN_MATMUL_GF2, FN_MATMUL_M4RI, FN_RANK_GF2, FN_RANK_M4RI, FN_NULL_GF2, FN_NULL_M4RI = range(6)
# mela_op and the cost model's shape
OP_RANK, OP_NULL, OP_MATMUL, OP_BATCH = 0, 1, 2, 3
MLP_IN, MLP_H1, MLP_H2, MLP_OUT, MLP_PARAMS = 10, 32, 32, 10, 1738


# tuning fields of a variant argument (MELA_TUNE_K / MELA_TUNE_TILE)
def tune(base: int, k: int = 0, tile: int = 0) -> int:
    return base | (k << 8) | (tile << 12)
# mela_elim_variant
ELIM_AUTO, ELIM_PLAIN, ELIM_M4RI, ELIM_M4RI_K4, ELIM_FUSED, ELIM_TC = 0, 1, 2, 3, 4, 5
ELIM_VARIANTS = {"auto": ELIM_AUTO, "plain": ELIM_PLAIN, "m4ri": ELIM_M4RI, "m4ri_k4": ELIM_M4RI_K4,
                 "fused": ELIM_FUSED, "tc": ELIM_TC}


class GatewayError(C.Structure):
    _fields_ = [("id", C.c_char * 64), ("msg", C.c_char * 256)]


ALLOC_FN = C.CFUNCTYPE(C.c_void_p, C.c_void_p, C.c_int64, C.c_int64)
GATEWAY_ALLOC_FN = C.CFUNCTYPE(C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int64, C.c_int64)


class BatchItem(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("in_offset", C.c_int64), ("z_offset", C.c_int64)]


class HostMatrix(C.Structure):
    _fields_ = [("kind", C.c_int32), ("sparse", C.c_int32), ("rows", C.c_int64),
                ("cols", C.c_int64), ("data", C.c_void_p)]


class UploadStats(C.Structure):
    _fields_ = [("blocked_bytes", C.c_int64), ("direct_bytes", C.c_int64), ("blocks", C.c_int64),
                ("host_copy_us", C.c_double), ("slot_wait_us", C.c_double)]


class HostCsc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("rows", C.c_int64), ("cols", C.c_int64),
                ("colptr", C.c_void_p), ("rowidx", C.c_void_p), ("values", C.c_void_p)]


# name -> (restype, argtypes); the list of every exported entry point
_i64, _u64, _i32, _u32, _vp, _sz = C.c_int64, C.c_uint64, C.c_int32, C.c_uint32, C.c_void_p, C.c_size_t
_st = C.c_int
SIGNATURES = {
    "mela_version": (C.c_int, []),
    "mela_status_string": (C.c_char_p, [_st]),
    "mela_last_error": (C.c_char_p, []),
    "mela_device_error_flags": (_st, [C.POINTER(_u32), C.c_int]),
    "mela_diag_wait_timeout": (_st, [_i32, _u64, _vp, _i32, _vp]),
    "mela_upload_stats_get": (None, [C.POINTER(UploadStats), C.c_int]),
    "mela_matmul_gf2": (_st, [C.POINTER(HostMatrix), C.POINTER(HostMatrix), _vp]),
    "mela_matmul_m4ri": (_st, [C.POINTER(HostMatrix), C.POINTER(HostMatrix), _vp]),
    "mela_rank_gf2": (_st, [C.POINTER(HostMatrix), C.POINTER(C.c_double)]),
    "mela_rank_m4ri": (_st, [C.POINTER(HostMatrix), C.POINTER(C.c_double)]),
    "mela_null_gf2": (_st, [C.POINTER(HostMatrix), ALLOC_FN, _vp, C.POINTER(_i64)]),
    "mela_null_m4ri": (_st, [C.POINTER(HostMatrix), ALLOC_FN, _vp, C.POINTER(_i64)]),
    "mela_rank_csc": (_st, [C.POINTER(HostCsc), C.POINTER(_i64)]),
    "mela_null_csc": (_st, [C.POINTER(HostCsc), ALLOC_FN, _vp, C.POINTER(_i64)]),
    "mela_dev_pack_csc": (_st, [_vp, _vp, _vp, _i32, _i64, _i64, _vp, _i64, _vp]),
    "mela_gateway": (C.c_int, [_i32, _i32, _i32, C.POINTER(HostMatrix), GATEWAY_ALLOC_FN, _vp,
                               C.POINTER(GatewayError)]),
    "mela_matmul_packed_host": (_st, [_vp, _i64, _vp, _i64, _vp, _i64, _i64, _i64, _i64, _i32]),
    "mela_dev_rand_dense": (_st, [_u64, _u64, _i64, _i64, _vp, _i64, _vp]),
    "mela_dev_rand_bernoulli": (_st, [_u64, _u64, _i64, _i64, C.c_double, _vp, _i64, _vp]),
    "mela_dev_pack": (_st, [_i32, _i64, _i64, _vp, _vp, _i64, _vp]),
    "mela_dev_unpack": (_st, [_vp, _i64, _i64, _i64, _vp, _vp]),
    "mela_dev_transpose": (_st, [_vp, _i64, _i64, _i64, _vp, _i64, _vp]),
    "mela_matmul_workspace_size": (_sz, [_i32, _i64, _i64, _i64]),
    "mela_dev_matmul": (_st, [_i32, _vp, _i64, _vp, _i64, _vp, _i64, _i64, _i64, _i64, _vp, _sz, _vp]),
    "mela_dev_matmul_prepare": (_st, [_i32, _vp, _i64, _vp, _i64, _i64, _i64, _i64, _vp, _sz, _vp]),
    "mela_dev_matmul_run": (_st, [_i32, _vp, _i64, _vp, _i64, _vp, _i64, _i64, _i64, _i64, _vp, _sz, _vp]),
    "mela_elim_workspace_size": (_sz, [_i64, _i64]),
    "mela_dev_rank": (_st, [_i32, _vp, _i64, _i64, _i64, _vp, _vp, _vp, _vp, _sz, _vp]),
    "mela_dev_rref": (_st, [_i32, _vp, _i64, _i64, _i64, _vp, _vp, _vp, _vp, _sz, _vp]),
    "mela_null_workspace_size": (_sz, [_i64, _i64]),
    "mela_dev_null_basis": (_st, [_vp, _i64, _i64, _i64, _i64, _vp, _vp, _vp, _i64, _vp, _sz, _vp]),
    "mela_null_verify_workspace_size": (C.c_size_t, [_i64, _i64]),
    "mela_dev_null_verify": (_st, [_vp, _i64, _i64, _i64, _vp, _i64, _i64, _vp, _vp, C.c_size_t, _vp]),
    "mela_dev_unpack_rows": (_st, [_vp, _i64, _i64, _i64, _vp, _vp]),
    "mela_batch_plan_create": (_st, [C.POINTER(BatchItem), _i64, _i32, C.POINTER(_vp)]),
    "mela_batch_plan_destroy": (None, [_vp]),
    "mela_batch_plan_stats": (_st, [_vp, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)]),
    "mela_batch_rank_null": (_st, [_vp, _vp, _vp, _vp, _i32, _vp]),
    "mela_batch_rank_null_logical": (_st, [_vp, _vp, _vp, _vp, _i32, _vp]),
    "mela_batch_pack_logical": (_st, [_vp, _vp, _vp, _vp]),
    "mela_batch_unpack_logical": (_st, [_vp, _vp, _vp, _vp]),
    "mela_mlp_forward": (_st, [_vp, _vp, _i64, _vp, _vp]),
    "mela_mlp_gradient": (_st, [_vp, _vp, _vp, _vp, _i64, C.c_float, _vp, _vp, _vp]),
    "mela_mlp_adam_step": (_st, [_vp, _vp, _vp, _vp, _i64, C.c_float, _vp]),
    "mela_costmodel_load": (_st, [_vp]),
    "mela_costmodel_choose": (_i32, [_i32, _i64, _i64, _i64, C.c_double, _i64, C.c_double]),
    "mela_costmodel_features": (None, [_i32, _i64, _i64, _i64, C.c_double, _i64, C.c_double, _vp]),
    "mela_costmodel_config_count": (_i32, [_i32]),
    "mela_dispatch_last": (_i32, [C.POINTER(C.c_double)]),
    "mela_costmodel_plan": (_i32, [_i32, _i64, _i64, _i64, C.POINTER(_i32)]),
    "mela_costmodel_predict": (_i32, [_i32, _i64, _i64, _i64, C.c_double, _i64, C.c_double, _vp]),
    "mela_costmodel_config": (_i32, [_i32, _i32]),
    "mela_dev_popcount": (_st, [_vp, _i64, _i64, _i64, _vp, _vp]),
    "mela_batch_plan_create_ex": (_st, [C.POINTER(BatchItem), _i64, _vp, _i32, C.POINTER(_vp)]),
    "mela_batch_popcounts": (_st, [C.POINTER(BatchItem), _i64, _vp, _vp, _vp]),
    "mela_static_scratch_bytes": (_sz, []),
    "mela_dev_matmul_plain_static": (_st, [_vp, _i64, _vp, _i64, _vp, _i64, _i64, _i64, _i64, _vp]),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build the CUDA library first "
                "(python -m mex_linear_algebra_b200.build); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class MelaError(RuntimeError):
    """A failed library call: ``status`` is the mela_status code."""

    def __init__(self, status: int, detail: str = ""):
        self.status = status
        self.detail = detail
        msg = lib().mela_status_string(status).decode()
        super().__init__(f"{msg}: {detail}" if detail else msg)


def check(status: int) -> None:
    if status != OK:
        raise MelaError(status, lib().mela_last_error().decode())
