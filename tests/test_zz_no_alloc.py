"""The allocation-free product mela_dev_matmul_plain_static.

It exists for callers that receive device buffers but may not allocate
device memory (a host application that owns the GPU memory budget, or a
latency-critical loop that cannot take cudaMalloc's implicit
synchronisation): its scratch lives in a fixed array inside the library.
Its results must equal mela_dev_matmul's, call after call, since every call
reuses the same array.  This file sorts last so that a run stopping at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O


def _lib():
    from mex_linear_algebra_b200 import _lib
    return _lib


def test_limit_reported_and_enforced_without_device_work():
    L = _lib().lib()
    cap = L.mela_static_scratch_bytes()
    assert cap == 16 << 20
    # B transposed would need n * ceil(k/64, even) * 8 bytes > cap: rejected up front
    n, k = 8192, 32768
    st = L.mela_dev_matmul_plain_static(C.c_void_p(16), k // 64, C.c_void_p(16), n // 64,
                                        C.c_void_p(16), n // 64, 64, k, n, None)
    assert st == _lib().ERR_UNSUPPORTED
    assert b"static scratch" in L.mela_last_error()
    # one word pair past the limit: n = 2048 and ceil(k/64) = 1025 -> 1026 words per row
    n, k = 2048, 65536 + 64
    st = L.mela_dev_matmul_plain_static(C.c_void_p(16), 1026, C.c_void_p(16), n // 64,
                                        C.c_void_p(16), n // 64, 64, k, n, None)
    assert st == _lib().ERR_UNSUPPORTED
    # within the array but beyond one launch's grid (k / 256 row blocks > 65535)
    n, k = 1, 1 << 25
    st = L.mela_dev_matmul_plain_static(C.c_void_p(16), k // 64, C.c_void_p(16), 1,
                                        C.c_void_p(16), 1, 64, k, n, None)
    assert st == _lib().ERR_UNSUPPORTED
    assert b"grid" in L.mela_last_error()


@pytest.mark.gpu
def test_static_scratch_product_matches_workspace_product(cuda):
    import torch
    from gpu_util import to_dev, to_host, valid_words
    _l = _lib()
    L = _l.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for (m, k, n, seed) in [(1000, 3000, 2000, 21), (4096, 8192, 4096, 22), (37, 23, 31, 23)]:
        A = to_dev(O.rand_dense(seed, 0, m, k))
        B = to_dev(O.rand_dense(seed, 1, k, n))
        C1 = torch.zeros((m, (n + 63) // 64), dtype=torch.int64, device="cuda")
        C2 = torch.full_like(C1, -1)
        wsb = L.mela_matmul_workspace_size(_l.GEMM_PLAIN, m, k, n)
        ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
        _l.check(L.mela_dev_matmul(_l.GEMM_PLAIN, A.data_ptr(), A.shape[1], B.data_ptr(),
                                   B.shape[1], C1.data_ptr(), C1.shape[1], m, k, n,
                                   ws.data_ptr(), wsb, stream))
        _l.check(L.mela_dev_matmul_plain_static(A.data_ptr(), A.shape[1], B.data_ptr(),
                                                B.shape[1], C2.data_ptr(), C2.shape[1], m, k, n,
                                                stream))
        torch.cuda.synchronize()
        assert torch.equal(C1, C2), (m, k, n)
        if m * n <= 4_000_000:
            want = O.matmul(to_host(A), to_host(B), m, k, n)
            assert np.array_equal(valid_words(to_host(C2), n), want)


def _with_padding_bits(P, cols, seed):
    """P with random bits set past column `cols` in every row's last word."""
    P = P.copy()
    if cols % 64:
        junk = O.rand_dense(seed, 9, P.shape[0], 64)[:, 0]
        P[:, (cols - 1) // 64] |= junk & ~np.uint64((1 << (cols % 64)) - 1)
    return P


@pytest.mark.gpu
def test_static_scratch_at_the_limit_and_with_padding_bits(cuda):
    """A product whose transposed operand fills the array exactly, then one
    whose operands carry set bits past their last column (which must not
    reach the result), each checked against mela_dev_matmul and the oracle."""
    import torch
    from gpu_util import to_dev, to_host, valid_words
    _l = _lib()
    L = _l.lib()
    stream = torch.cuda.current_stream().cuda_stream
    n, k = 2048, 65536
    assert n * 1024 * 8 == L.mela_static_scratch_bytes()
    for (m, k, n, seed, junk) in [(300, k, n, 31, False), (257, 1000, 333, 32, True),
                                  (300, k, n, 33, False)]:
        A0, B0 = O.rand_dense(seed, 0, m, k), O.rand_dense(seed, 1, k, n)
        A = to_dev(_with_padding_bits(A0, k, seed) if junk else A0)
        B = to_dev(_with_padding_bits(B0, n, seed + 100) if junk else B0)
        C1 = torch.zeros((m, (n + 63) // 64), dtype=torch.int64, device="cuda")
        C2 = torch.full_like(C1, -1)
        wsb = L.mela_matmul_workspace_size(_l.GEMM_PLAIN, m, k, n)
        ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
        _l.check(L.mela_dev_matmul(_l.GEMM_PLAIN, A.data_ptr(), A.shape[1], B.data_ptr(),
                                   B.shape[1], C1.data_ptr(), C1.shape[1], m, k, n,
                                   ws.data_ptr(), wsb, stream))
        _l.check(L.mela_dev_matmul_plain_static(A.data_ptr(), A.shape[1], B.data_ptr(),
                                                B.shape[1], C2.data_ptr(), C2.shape[1], m, k, n,
                                                stream))
        torch.cuda.synchronize()
        assert torch.equal(C1, C2), (m, k, n)
        want = O.matmul(A0, B0, m, k, n)
        assert np.array_equal(valid_words(to_host(C2), n), want)
