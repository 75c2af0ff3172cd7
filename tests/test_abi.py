"""The C-ABI library loads on a machine without a GPU and exports every entry
point include/mela.h declares; argument checks that precede any device work
behave as documented."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "mela.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mela_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "mela_matmul_gf2" in syms and "mela_dev_matmul" in syms
    assert len(syms) >= 10


def test_library_exports_every_declared_symbol():
    from mex_linear_algebra_b200 import lib
    L = lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    from mex_linear_algebra_b200._lib import SIGNATURES
    assert sorted(SIGNATURES) == declared_symbols()


def test_status_strings():
    from mex_linear_algebra_b200 import lib
    L = lib()
    assert L.mela_status_string(0) == b"ok"
    assert L.mela_version() >= 10000


def _hm(kind, rows, cols, sparse=0):
    from mex_linear_algebra_b200._lib import HostMatrix
    return HostMatrix(kind, sparse, rows, cols, None)


@pytest.mark.parametrize("fn", ["mela_matmul_gf2", "mela_matmul_m4ri"])
def test_matmul_validation_order(fn):
    """Sparse, then inner dimensions, then class (src/mela_matmul_gf2.c:78-88);
    all three are decided before any device work."""
    from mex_linear_algebra_b200 import _lib
    f = getattr(_lib.lib(), fn)
    A, B = _hm(0, 3, 4, sparse=1), _hm(0, 5, 2)
    assert f(C.byref(A), C.byref(B), None) == _lib.ERR_SPARSE
    A, B = _hm(2, 3, 4), _hm(0, 5, 2)
    assert f(C.byref(A), C.byref(B), None) == _lib.ERR_DIM
    A, B = _hm(2, 3, 4), _hm(0, 4, 2)
    assert f(C.byref(A), C.byref(B), None) == _lib.ERR_TYPE


def test_dev_entry_points_reject_bad_shapes():
    from mex_linear_algebra_b200 import _lib
    L = _lib.lib()
    assert L.mela_dev_matmul(1, None, 0, None, 0, None, 0, -1, 1, 1, None, 0, None) == _lib.ERR_INVALID
    assert L.mela_dev_matmul(9, None, 1, None, 1, None, 1, 1, 1, 1, None, 0, None) == _lib.ERR_INVALID
    assert L.mela_dev_pack(5, 1, 1, None, None, 1, None) == _lib.ERR_INVALID
    assert L.mela_dev_transpose(None, 0, 2, 70, None, 1, None) == _lib.ERR_INVALID


def test_batch_entry_points_reject_bad_arguments():
    """Null plans and buffers, negative shapes or offsets and a bad item list
    are refused before any device work."""
    from mex_linear_algebra_b200 import _lib
    L = _lib.lib()
    for fn in ("mela_batch_rank_null", "mela_batch_rank_null_logical"):
        assert getattr(L, fn)(None, None, None, None, 1, None) == _lib.ERR_INVALID
    for fn in ("mela_batch_pack_logical", "mela_batch_unpack_logical"):
        assert getattr(L, fn)(None, None, None, None) == _lib.ERR_INVALID
    plan = C.c_void_p()
    items = (_lib.BatchItem * 2)(_lib.BatchItem(3, 5, 0, 0), _lib.BatchItem(-1, 5, 1, 5))
    assert L.mela_batch_plan_create(items, 2, -1, C.byref(plan)) == _lib.ERR_INVALID
    assert b"item 1 has a bad shape or offset" in L.mela_last_error()
    assert not plan.value
    items = (_lib.BatchItem * 1)(_lib.BatchItem(3, 5, -8, 0))
    assert L.mela_batch_plan_create(items, 1, -1, C.byref(plan)) == _lib.ERR_INVALID
    assert L.mela_batch_plan_create(None, 4, -1, C.byref(plan)) == _lib.ERR_INVALID
    assert L.mela_batch_plan_create(items, -1, -1, C.byref(plan)) == _lib.ERR_INVALID
    assert L.mela_batch_plan_create(items, 1, -1, None) == _lib.ERR_INVALID


def test_null_verify_rejects_bad_arguments():
    """Shapes, pitches, the result pointer and the workspace are checked
    before any device work."""
    from mex_linear_algebra_b200 import _lib
    L = _lib.lib()
    assert L.mela_null_verify_workspace_size(100, 70) == 100 * 2 * 8
    assert L.mela_null_verify_workspace_size(0, 70) == 0
    assert L.mela_null_verify_workspace_size(100, 0) == 0
    fake = C.c_void_p(16)  # never dereferenced: every call below fails its checks first
    assert L.mela_dev_null_verify(fake, 1, -1, 64, fake, 1, 1, fake, None, 0, None) == _lib.ERR_INVALID
    assert L.mela_dev_null_verify(fake, 1, 4, 130, fake, 3, 1, fake, None, 0, None) == _lib.ERR_INVALID
    assert L.mela_dev_null_verify(fake, 3, 4, 130, fake, 1, 1, fake, None, 0, None) == _lib.ERR_INVALID
    assert L.mela_dev_null_verify(fake, 3, 4, 130, fake, 3, 1, None, None, 0, None) == _lib.ERR_INVALID
    assert L.mela_dev_null_verify(None, 3, 4, 130, fake, 3, 1, fake, fake, 64, None) == _lib.ERR_INVALID
    assert L.mela_dev_null_verify(fake, 3, 4, 130, fake, 3, 1, fake, fake, 31, None) == _lib.ERR_INVALID
    assert b"workspace of 32 bytes needed" in L.mela_last_error()


def test_workspace_sizes():
    from mex_linear_algebra_b200 import _lib
    L = _lib.lib()
    assert L.mela_matmul_workspace_size(_lib.GEMM_M4RI, 100, 100, 100) == 0
    # INT8 tensor-core form: one byte per bit of both operands, padded to the tile grid
    # (B is expanded straight from its packed rows, so no transposed copy is kept)
    ws = L.mela_matmul_workspace_size(_lib.GEMM_TC, 32768, 32768, 32768)
    assert 2 * 32768 * 32768 <= ws < 2 * 32768 * 32768 + 32768 * 512 * 8
    # FP4 form: half a byte per bit
    ws4 = L.mela_matmul_workspace_size(_lib.GEMM_TC_FP4, 32768, 32768, 32768)
    assert 32768 * 32768 <= ws4 < ws
