"""GF(2) product on the GPU against the oracle (bit-exact).

Cases follow the reference's own tests: run_ci_tests.m:42-56 (37x23 * 23x31,
zero A 5x7 * 7x3), run_ci_tests.m:92-98 (double inputs), compile_mex.m:144-162
(m4ri vs gf2 at 256x128 * 128x64), plus odd/ragged shapes around the tile
sizes, the plain-method config (2048x2048 * 2048x1024) and the large config
(32768^3) through size-independent checks.
"""
import numpy as np
import pytest

import oracle as O
from gpu_util import to_dev, to_host, valid_words

pytestmark = pytest.mark.gpu

VARIANTS = ("plain", "m4ri", "tc", "tc_fp4")


def _dev():
    from mex_linear_algebra_b200 import device
    return device


def test_generator_matches_oracle(cuda):
    D = _dev()
    for (m, n, seed, st) in [(1, 1, 0, 0), (37, 23, 1, 2), (130, 200, 5, 7), (64, 4096, 9, 1)]:
        g = to_host(D.rand_dense(seed, st, m, n))
        o = O.rand_dense(seed, st, m, n)
        assert np.array_equal(g, o), (m, n)


@pytest.mark.parametrize("kind", ["logical", "double"])
@pytest.mark.parametrize("shape", [(1, 1), (37, 23), (64, 64), (65, 129), (300, 1000), (1, 700)])
def test_pack_unpack(cuda, kind, shape):
    import torch
    D = _dev()
    m, n = shape
    rng = np.random.default_rng(m * 1000 + n)
    if kind == "logical":
        a = rng.random((m, n)) >= 0.5
        dev_in = torch.from_numpy(np.asfortranarray(a).ravel(order="F").view(np.uint8).copy()).cuda()
    else:
        a = rng.integers(-7, 8, size=(m, n)).astype(np.float64)
        a[rng.random((m, n)) < 0.05] = 2.5
        dev_in = torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).cuda()
    p = to_host(D.pack(dev_in, m, n))
    assert np.array_equal(p, O.pack(a))
    u = D.unpack(to_dev(p), m, n).cpu().numpy().reshape((m, n), order="F").view(np.bool_)
    assert np.array_equal(u, O.unpack(O.pack(a), m, n))


def test_pack_special_doubles(cuda):
    import torch
    D = _dev()
    vals = np.array([0.0, 1.0, -1.0, 2.0, -3.0, 3.7, -3.7, 0.5, -0.5, 2147483647.0, 2147483648.0,
                     -2147483648.0, -2147483649.0, 1e300, -1e300, np.inf, -np.inf, np.nan, 5.0,
                     2147483646.9, -2147483647.5], dtype=np.float64)
    a = vals.reshape(-1, 1)
    dev_in = torch.from_numpy(a.ravel().copy()).cuda()
    p = to_host(D.pack(dev_in, a.shape[0], 1))
    want = np.array([O.lib().orc_parity_double(float(v)) for v in vals], dtype=np.uint64)
    assert np.array_equal(p[:, 0], want)


@pytest.mark.parametrize("shape", [(1, 1), (64, 64), (100, 37), (257, 513), (1000, 3000)])
def test_transpose(cuda, shape):
    D = _dev()
    r, c = shape
    a = O.rand_dense(3, 4, r, c)
    t = to_host(D.transpose(to_dev(a), r, c))
    ua = O.unpack(a, r, c)
    assert np.array_equal(t, O.pack(np.asfortranarray(ua.T)))


SHAPES = [(1, 1, 1), (37, 23, 31), (5, 7, 3), (3, 3, 2), (256, 128, 64), (129, 65, 257),
          (128, 128, 256), (300, 500, 700), (1000, 777, 1500), (1025, 4096, 300)]


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("shape", SHAPES)
def test_matmul_vs_oracle(cuda, variant, shape):
    D = _dev()
    m, k, n = shape
    A = O.rand_dense(11, 1, m, k)
    B = O.rand_dense(11, 2, k, n)
    if shape == (5, 7, 3):
        A[:] = 0  # zero A (run_ci_tests.m:50-55)
    want = O.matmul(A, B, m, k, n)
    got = to_host(D.matmul(to_dev(A), to_dev(B), m, k, n, variant=variant))
    assert np.array_equal(valid_words(got, n), want)


@pytest.mark.parametrize("variant", VARIANTS)
def test_matmul_plain_config(cuda, variant):
    """2048x2048 * 2048x1024 from seed 0 -- the plain-method configuration."""
    D = _dev()
    m, k, n = 2048, 2048, 1024
    A = D.rand_dense(0, 0, m, k)
    B = D.rand_dense(0, 1, k, n)
    want = O.matmul(to_host(A), to_host(B), m, k, n)
    got = to_host(D.matmul(A, B, m, k, n, variant=variant))
    assert np.array_equal(got, want)


def test_variants_agree_4096(cuda):
    D = _dev()
    m = k = n = 4096
    A = D.rand_dense(7, 0, m, k)
    B = D.rand_dense(7, 1, k, n)
    c_plain = D.matmul(A, B, m, k, n, variant="plain")
    c_tc = D.matmul(A, B, m, k, n, variant="tc")
    c_m4 = D.matmul(A, B, m, k, n, variant="m4ri")
    import torch
    assert torch.equal(c_plain, c_tc)
    assert torch.equal(c_plain, c_m4)
    # spot-check 64 rows against the oracle
    rows = slice(1000, 1064)
    want = O.matmul(to_host(A)[rows], to_host(B), 64, k, n)
    assert np.array_equal(to_host(c_tc)[rows], want)


def test_large_config_checks(cuda):
    """32768^3 (seed 1): the FP4 and INT8 tensor-core forms and the plain form
    all reproduce the checker's digest of the full product (computed on the
    CPU by the oracle and by the reference's own mela_matmul_gf2,
    tests/golden/make_config_digests.py), row block by row block, and
    (A*B)*X == A*(B*X) for a random 32768 x 64 block X."""
    import hashlib
    import json
    import os
    import torch
    D = _dev()
    g = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                    "config_digests.json")))["product_32768"]
    m = k = n = 32768
    A = D.rand_dense(1, 0, m, k)
    B = D.rand_dense(1, 1, k, n)

    def blocks(C):
        h = C.cpu().numpy()
        rb = g["row_block"]
        return [hashlib.blake2b(h[i:i + rb].tobytes(), digest_size=16).hexdigest() for i in range(0, m, rb)]

    c_fp4 = D.matmul(A, B, m, k, n, variant="tc_fp4")
    assert blocks(c_fp4) == g["block_digests"]
    c_tc = D.matmul(A, B, m, k, n, variant="tc")
    assert torch.equal(c_tc, c_fp4)
    del c_fp4
    c_plain = D.matmul(A, B, m, k, n, variant="plain")
    assert torch.equal(c_tc, c_plain)
    X = D.rand_dense(1, 2, n, 64)
    left = D.matmul(c_tc, X, m, n, 64, variant="plain")
    bx = D.matmul(B, X, k, n, 64, variant="plain")
    right = D.matmul(A, bx, m, k, 64, variant="plain")
    assert torch.equal(left, right)
    # a block of rows against the oracle
    want = O.matmul(to_host(A[:8]), to_host(B), 8, k, n)
    assert np.array_equal(to_host(c_tc[:8]), want)
    del c_plain
    torch.cuda.empty_cache()
    assert D.device_error_flags() == 0


def test_bernoulli_generator_matches_host(cuda):
    import torch
    from mex_linear_algebra_b200 import _lib, gen
    L = _lib.lib()
    for (m, n, d, st) in [(7, 70, 0.1, 1), (100, 300, 0.003, 2), (33, 64, 0.5, 3)]:
        out = torch.empty((m, (n + 63) // 64), dtype=torch.int64, device="cuda")
        _lib.check(L.mela_dev_rand_bernoulli(4, st, m, n, d, out.data_ptr(), out.shape[1],
                                             torch.cuda.current_stream().cuda_stream))
        assert np.array_equal(to_host(out), gen.sparse_packed(4, st, m, n, d))


@pytest.mark.parametrize("k", [1, 63, 255, 257, 32767, 32769, 1048577])
def test_long_sums_exact(cuda, k):
    """All-ones operands: every entry of C is k mod 2, the sum of k ones.
    Checks that the tensor-core forms keep the integer sum exact (the fp4 form
    accumulates in f32; exact, and read by one float add, below 2^23)."""
    import torch
    D = _dev()
    m, n = 256, 256
    wk, wn = (k + 63) // 64, (n + 63) // 64
    A = torch.zeros((m, wk), dtype=torch.int64, device="cuda")
    B = torch.zeros((k, wn), dtype=torch.int64, device="cuda")
    A[:] = -1
    B[:] = -1
    if k % 64:
        A[:, -1] = (1 << (k % 64)) - 1
    want = np.uint64(0xFFFFFFFFFFFFFFFF) if (k & 1) else np.uint64(0)
    for variant in ("tc", "tc_fp4", "plain"):
        C = to_host(D.matmul(A, B, m, k, n, variant=variant))
        assert (C == want).all(), (variant, k)


def test_fp4_variants_agree_large(cuda):
    import torch
    D = _dev()
    m, k, n = 8192, 16384, 8192
    A = D.rand_dense(13, 0, m, k)
    B = D.rand_dense(13, 1, k, n)
    assert torch.equal(D.matmul(A, B, m, k, n, variant="tc_fp4"), D.matmul(A, B, m, k, n, variant="tc"))


@pytest.mark.parametrize("variant", ["tc", "tc_fp4", "plain"])
@pytest.mark.parametrize("shape", [(9000, 1000, 9000), (8192, 64, 8192), (20000, 300, 8300), (9000, 1000, 700)])
def test_packed_host_product(cuda, variant, shape):
    """The host-buffer product (for the tensor-core forms once m and n reach
    8192, transfers overlapped in row blocks of A and column blocks of B) equals
    the device product of the oracle's inputs, with ragged last blocks (a
    partial word of columns included) and page-locked and pageable buffers."""
    import torch
    from mex_linear_algebra_b200 import _lib
    m, k, n = shape
    A = O.rand_dense(61, m + k, m, k)
    B = O.rand_dense(61, k + n, k, n)
    wk, wn = (k + 63) // 64, (n + 63) // 64
    want = to_host(_dev().matmul(to_dev(A), to_dev(B), m, k, n, variant="plain"))
    for pinned in (True, False):
        hA = torch.from_numpy(np.ascontiguousarray(A[:, :wk]).view(np.int64))
        hB = torch.from_numpy(np.ascontiguousarray(B[:, :wn]).view(np.int64))
        hC = torch.zeros((m, wn), dtype=torch.int64)
        if pinned:
            hA, hB, hC = hA.pin_memory(), hB.pin_memory(), hC.pin_memory()
        _lib.check(_lib.lib().mela_matmul_packed_host(hA.data_ptr(), wk, hB.data_ptr(), wn, hC.data_ptr(), wn,
                                                      m, k, n, _lib.GEMM_VARIANTS[variant]))
        got = hC.numpy().view(np.uint64)
        assert np.array_equal(valid_words(got, n), valid_words(want, n)), (variant, pinned)


@pytest.mark.parametrize("shape", [(1, 1, 1), (300, 77, 513), (129, 1000, 300), (64, 256, 256), (200, 5000, 700)])
def test_tensor_core_forms_odd_shapes(cuda, shape):
    """Both tensor-core forms (B prepared by the transposing expansion) on
    shapes that leave partial words, partial 256-column tiles and partial
    K steps."""
    D = _dev()
    m, k, n = shape
    A = O.rand_dense(71, m + k, m, k)
    B = O.rand_dense(71, k + n, k, n)
    want = O.matmul(A, B, m, k, n)
    for variant in ("tc", "tc_fp4"):
        got = to_host(D.matmul(to_dev(A), to_dev(B), m, k, n, variant=variant))
        assert np.array_equal(valid_words(got, n), valid_words(want, n)), variant


@pytest.mark.parametrize("tile", [1, 2])
@pytest.mark.parametrize("pad", [0, 1])
@pytest.mark.parametrize("shape", [(37, 23, 31), (129, 65, 257), (513, 1000, 2049), (1000, 777, 1500),
                                   (600, 4100, 4096)])
def test_m4ri_tiles_and_row_pitches(cuda, tile, pad, shape):
    """The Four-Russians product on 16 warps of 32 rows (tile 2, the default)
    and 8 warps of 64 rows (tile 1), with B's rows staged by TMA (row pitch a
    multiple of 16 bytes) or read with plain loads (odd pitch: pad changes
    which), against the oracle."""
    import torch
    from mex_linear_algebra_b200 import _lib
    D = _dev()
    m, k, n = shape
    A = O.rand_dense(17, m, m, k)
    B = O.rand_dense(17, n, k, n)
    wn = (n + 63) // 64
    ldb = wn + pad
    Bp = np.zeros((k, ldb), dtype=np.uint64)
    Bp[:, :wn] = B
    got = to_host(D.matmul(to_dev(A), to_dev(Bp), m, k, n, variant=_lib.tune(_lib.GEMM_M4RI, 0, tile)))
    assert np.array_equal(valid_words(got, n), O.matmul(A, B, m, k, n))
