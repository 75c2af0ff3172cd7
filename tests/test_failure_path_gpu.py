"""The bounded-wait failure path, made to happen without faulting the GPU.

A diagnostic kernel (mela_diag_wait_timeout) waits, with a 1 ms limit, on a
device flag or an mbarrier that nothing will ever signal -- the second with
tensor memory allocated.  The wait must run out, set the timeout bit of the
device error word, free what it holds and return; the synchronous form must
report MELA_ERR_TIMEOUT and clear the bit; and the device must stay usable:
a tensor-core product (which allocates all of an SM's tensor memory) right
after still gives the oracle's result.
"""
import numpy as np
import pytest

import oracle as O
from gpu_util import to_dev, to_host, valid_words

pytestmark = pytest.mark.gpu

LIMIT_NS = 1_000_000  # 1 ms


@pytest.mark.parametrize("kind", [0, 1])
def test_wait_runs_out_and_device_stays_usable(cuda, kind):
    import torch
    from mex_linear_algebra_b200 import _lib, device as D
    L = _lib.lib()
    s = torch.cuda.current_stream().cuda_stream
    assert D.device_error_flags(clear=True) == 0
    out = torch.zeros(2, dtype=torch.int32, device="cuda")
    # stream-ordered: the bit is set and stays set until cleared
    _lib.check(L.mela_diag_wait_timeout(kind, LIMIT_NS, out.data_ptr(), 0, s))
    torch.cuda.synchronize()
    assert int(out[0].item()) == 1
    if kind == 1:
        assert int(out[1].item()) == 1  # tensor memory freed on the timeout path
    assert D.device_error_flags(clear=False) & 1
    assert D.device_error_flags(clear=True) & 1
    assert D.device_error_flags(clear=False) == 0
    # synchronous: MELA_ERR_TIMEOUT, bit cleared
    out.zero_()
    st = L.mela_diag_wait_timeout(kind, LIMIT_NS, out.data_ptr(), 1, s)
    assert st == _lib.ERR_TIMEOUT
    assert b"timed out" in L.mela_last_error()
    assert D.device_error_flags(clear=False) == 0
    # the device still computes correctly
    m, k, n = 300, 700, 500
    A, B = O.rand_dense(81, 0, m, k), O.rand_dense(81, 1, k, n)
    want = O.matmul(A, B, m, k, n)
    for variant in ("tc_fp4", "tc", "plain"):
        got = to_host(D.matmul(to_dev(A), to_dev(B), m, k, n, variant=variant))
        assert np.array_equal(valid_words(got, n), want), variant
    assert D.device_error_flags(clear=False) == 0


def test_argument_checks(cuda):
    import torch
    from mex_linear_algebra_b200 import _lib
    L = _lib.lib()
    out = torch.zeros(2, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    for (kind, lim) in [(2, LIMIT_NS), (0, 10), (1, 5_000_000_000)]:
        assert L.mela_diag_wait_timeout(kind, lim, out.data_ptr(), 1, s) == _lib.ERR_INVALID
