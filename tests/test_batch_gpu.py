"""Batched rank + null space against the oracle, per matrix (bit-exact).

Covers the parity-check generator (6 ones per row, n about 2m), dense random
matrices of mixed shapes (including ones too large for shared memory), every
engine (forced CTA / 128-thread / warp classes give identical results), the
logical-input path and graph versus direct launch.
"""
import numpy as np
import pytest

import oracle as O
from gpu_util import to_host

pytestmark = pytest.mark.gpu


def _check(plan, ranks, zt, mats):
    rk = to_host(ranks)
    z = to_host(zt)
    for i, (m, n, P) in enumerate(mats):
        R, piv = O.rref(P, m, n)
        assert rk[i] == len(piv), (i, m, n)
        want = O.null_basis_packed(P, m, n)
        got = plan.basis(z, rk, i)
        assert np.array_equal(got, want), (i, m, n)


def _pack_buffer(plan, mats):
    import torch
    buf = np.zeros(max(plan.in_words, 1), dtype=np.uint64)
    for i, (m, n, P) in enumerate(mats):
        o = int(plan.in_offsets[i])
        buf[o:o + P.size] = P.ravel()
    return torch.from_numpy(buf.view(np.int64)).cuda()


def ldpc_mats(count, seed=3):
    from mex_linear_algebra_b200 import gen
    out = []
    for b in range(count):
        m, n, P = gen.ldpc_packed(seed, b)
        out.append((m, n, P))
    return out


def mixed_mats():
    shapes = [(1, 1), (5, 3), (64, 130), (100, 90), (200, 420), (300, 300), (700, 1500),
              (1024, 2300), (1100, 2000), (40, 3000), (3, 5000), (512, 512)]
    return [(m, n, O.rand_dense(77, i, m, n)) for i, (m, n) in enumerate(shapes)]


@pytest.mark.parametrize("force", [-1, 0, 1, 2])
def test_ldpc_batch_all_engines(cuda, force):
    from mex_linear_algebra_b200 import device as D
    mats = ldpc_mats(40)
    plan = D.BatchPlan([(m, n) for (m, n, _) in mats], force_class=force)
    ranks, zt = plan.run(_pack_buffer(plan, mats))
    _check(plan, ranks, zt, mats)
    plan.close()


@pytest.mark.parametrize("use_graph", [True, False])
def test_mixed_dense_batch(cuda, use_graph):
    from mex_linear_algebra_b200 import device as D
    mats = mixed_mats()
    plan = D.BatchPlan([(m, n) for (m, n, _) in mats])
    d_in = _pack_buffer(plan, mats)
    for _ in range(2):  # a replayed graph gives the same answer
        ranks, zt = plan.run(d_in, use_graph=use_graph)
        _check(plan, ranks, zt, mats)
    plan.close()


def test_logical_input(cuda):
    import torch
    from mex_linear_algebra_b200 import device as D
    mats = ldpc_mats(12, seed=5) + mixed_mats()[:6]
    plan = D.BatchPlan([(m, n) for (m, n, _) in mats])
    chunks = [np.asfortranarray(O.unpack(P, m, n)).ravel(order="F").view(np.uint8) for (m, n, P) in mats]
    d_log = torch.from_numpy(np.concatenate(chunks)).cuda()
    # the batched unpack produces the same logical bytes from the packed form
    assert torch.equal(plan.unpack_logical(_pack_buffer(plan, mats)), d_log)
    ranks, zt = plan.run_logical(d_log)
    _check(plan, ranks, zt, mats)
    plan.close()


def _logical_bytes(mats, rng=None):
    """Column-major logical bytes of every matrix; with rng, the nonzero bytes
    of every other matrix become random values in 1..255."""
    out = []
    for i, (m, n, P) in enumerate(mats):
        L = np.asfortranarray(O.unpack(P, m, n)).ravel(order="F").view(np.uint8).copy()
        if rng is not None and i % 2:
            nz = L != 0
            L[nz] = rng.integers(1, 256, size=int(nz.sum()), dtype=np.uint8)
        out.append(L)
    return np.concatenate(out)


@pytest.mark.parametrize("shift", [0, 3, 13])
@pytest.mark.parametrize("dirty", [False, True])
def test_pack_logical_exact(cuda, shift, dirty):
    """The batched packing equals the oracle's packing word for word, from a
    base pointer at any alignment, with nonzero bytes other than 1 read as 1."""
    import torch
    from mex_linear_algebra_b200 import device as D
    shapes = [(1, 1), (7, 200), (16, 64), (17, 63), (511, 65), (512, 128), (513, 130),
              (1000, 700), (1025, 64), (3, 1), (200, 9)]
    mats = [(m, n, O.rand_dense(31, i, m, n)) for i, (m, n) in enumerate(shapes)] + ldpc_mats(5, seed=9)
    plan = D.BatchPlan([(m, n) for (m, n, _) in mats])
    host = _logical_bytes(mats, np.random.default_rng(shift) if dirty else None)
    buf = torch.zeros(shift + host.size, dtype=torch.uint8, device="cuda")
    buf[shift:] = torch.from_numpy(host).cuda()
    got = plan.pack_logical(buf[shift:])
    want = _pack_buffer(plan, mats)
    assert torch.equal(got, want)
    ranks, zt = plan.run_logical(buf[shift:])
    _check(plan, ranks, zt, mats)
    plan.close()


@pytest.mark.parametrize("logical", [False, True])
def test_empty_matrices_in_batch(cuda, logical):
    """0 x n, m x 0 and 0 x 0 items beside ordinary ones: rank 0, null basis
    I_n for m = 0, nothing for n = 0, and the other items unaffected."""
    import torch
    from mex_linear_algebra_b200 import device as D
    shapes = [(0, 5), (33, 70), (7, 0), (0, 0), (0, 70), (300, 640), (1, 0), (0, 1), (64, 64)]
    mats = [(m, n, O.rand_dense(41, i, m, n)) for i, (m, n) in enumerate(shapes)]
    plan = D.BatchPlan([(m, n) for (m, n, _) in mats])
    if logical:
        host = _logical_bytes(mats)
        d_log = torch.from_numpy(host).cuda() if host.size else torch.zeros(1, dtype=torch.uint8, device="cuda")
        assert torch.equal(plan.pack_logical(d_log), _pack_buffer(plan, mats))
        ranks, zt = plan.run_logical(d_log)
    else:
        ranks, zt = plan.run(_pack_buffer(plan, mats))
    _check(plan, ranks, zt, mats)
    plan.close()


def test_large_batch_ranks(cuda):
    """2000 parity-check matrices: ranks equal the per-matrix oracle on a sample."""
    from mex_linear_algebra_b200 import device as D, gen
    shapes, offsets, buf = gen.ldpc_batch(2000)
    plan = D.BatchPlan(shapes)
    import torch
    assert np.array_equal(plan.in_offsets, offsets)
    ranks, zt = plan.run(torch.from_numpy(buf.view(np.int64)).cuda())
    rk = to_host(ranks)
    z = to_host(zt)
    for i in range(0, 2000, 97):
        m, n = shapes[i]
        P = buf[offsets[i]:offsets[i] + m * ((n + 63) // 64)].reshape(m, -1)
        assert rk[i] == O.rank(P, m, n, 10)
        assert np.array_equal(plan.basis(z, rk, i), O.null_basis_packed(P, m, n))
    plan.close()
