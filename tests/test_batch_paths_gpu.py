"""The big-matrix engine's selection and look-ahead paths against the oracle.

A panel's pivots are chosen by one warp among its candidate rows (unused
rows with a nonzero panel word) when there are at most 384 of them, else by
the per-bit eight-warp register panel (m <= 1024) or the per-bit slot search
(larger m); the next panel's pivots are selected while the current panel's
update runs whenever that panel's candidates fit the warp.  The matrices here
are built so that each path and each switch between them runs: a first panel
with exactly 384 and 385 candidates, sparse panels followed by dense ones,
rank-deficient matrices (panels without pivots, early ends), more than 1024
rows, and the single-matrix fused form over the same engine.  Every result
(rank, null basis; for the fused form the RREF rows and pivots) must equal the
oracle's bit for bit.
"""
import numpy as np
import pytest

import oracle as O
from gpu_util import to_host

pytestmark = pytest.mark.gpu


def _pack(bits):
    """(m, n) 0/1 array -> packed uint64 rows (bit j of row i at word j // 64)."""
    m, n = bits.shape
    wc = (n + 63) // 64
    pad = np.zeros((m, wc * 64), dtype=np.uint8)
    pad[:, :n] = bits
    by = np.packbits(pad.reshape(m, wc, 64)[:, :, ::-1], axis=2)  # big-endian bytes of each word
    return by.reshape(m, wc, 8)[:, :, ::-1].copy().view(np.uint64).reshape(m, wc)


def sparse(rng, m, n, k=6):
    a = np.zeros((m, n), dtype=np.uint8)
    for i in range(m):
        a[i, rng.choice(n, size=min(k, n), replace=False)] = 1
    return a


def first_panel_candidates(rng, m, n, c):
    """Rows 0 .. c-1 carry random nonzero words in columns 0..63, the others
    none there; six more ones per row beyond column 63."""
    a = sparse(rng, m, n - 64, 6)
    a = np.concatenate([np.zeros((m, 64), dtype=np.uint8), a], axis=1)
    for i in range(c):
        w = rng.integers(0, 2, size=64, dtype=np.uint8)
        w[rng.integers(0, 64)] = 1
        a[i, :64] = w
    return a


def sparse_then_dense(rng, m, n, split):
    a = sparse(rng, m, n, 4)
    a[:, split:] = rng.integers(0, 2, size=(m, n - split), dtype=np.uint8)
    return a


def low_rank(rng, m, n):
    a = sparse(rng, m, n, 6)
    half = m // 2
    for i in range(half, m):  # each lower row the sum of two upper ones
        a[i] = a[i - half] ^ a[(i - half + 7) % half]
    return a


def _cases():
    rng = np.random.default_rng(20261204)
    return [
        ("cand384", first_panel_candidates(rng, 700, 1400, 384)),
        ("cand385", first_panel_candidates(rng, 700, 1400, 385)),
        ("cand1", first_panel_candidates(rng, 300, 640, 1)),
        ("sparse_then_dense", sparse_then_dense(rng, 900, 1800, 640)),
        ("dense_then_sparse", np.concatenate(
            [rng.integers(0, 2, size=(800, 300), dtype=np.uint8), sparse(rng, 800, 1300, 5)], axis=1)),
        ("low_rank", low_rank(rng, 960, 1900)),
        ("tall_sparse", sparse(rng, 1500, 1200, 6)),
        ("big_m_sparse", sparse(rng, 1400, 2900, 6)),
        ("big_m_dense", rng.integers(0, 2, size=(1100, 1300), dtype=np.uint8)),
        ("zero_panel_gap", np.concatenate(
            [sparse(rng, 600, 700, 5), np.zeros((600, 200), dtype=np.uint8), sparse(rng, 600, 500, 3)], axis=1)),
    ]


CASES = _cases()


def test_packing_helper():
    bits = np.zeros((2, 130), dtype=np.uint8)
    bits[0, 0] = bits[0, 64] = bits[1, 129] = 1
    P = _pack(bits)
    assert P[0, 0] == 1 and P[0, 1] == 1 and P[1, 2] == 2


def test_batch_paths(cuda):
    import torch
    from mex_linear_algebra_b200 import device as D
    mats = [(b.shape[0], b.shape[1], _pack(b)) for _, b in CASES]
    plan = D.BatchPlan([(m, n) for (m, n, _) in mats], force_class=0)  # every matrix on the CTA engine
    buf = np.zeros(max(plan.in_words, 1), dtype=np.uint64)
    for i, (m, n, P) in enumerate(mats):
        o = int(plan.in_offsets[i])
        buf[o:o + P.size] = P.ravel()
    ranks, zt = plan.run(torch.from_numpy(buf.view(np.int64)).cuda())
    rk = to_host(ranks)
    z = to_host(zt)
    for i, ((name, _), (m, n, P)) in enumerate(zip(CASES, mats)):
        R, piv = O.rref(P, m, n)
        assert rk[i] == len(piv), name
        assert np.array_equal(plan.basis(z, rk, i), O.null_basis_packed(P, m, n)), name
    plan.close()


@pytest.mark.parametrize("name", ["big_m_sparse", "sparse_then_dense", "low_rank"])
def test_fused_form_paths(cuda, name):
    """The single-matrix fused form runs the same engine (512 threads) on
    matrices too large for its shared memory."""
    from test_elim_gpu import check_all
    bits = dict(CASES)[name]
    if name != "big_m_sparse":  # make it larger than the fused form's 220 KB of shared memory
        bits = np.concatenate([bits, bits[:, ::-1]], axis=0)
    m, n = bits.shape
    assert m * ((n + 63) // 64) * 8 > 220 * 1024
    check_all(_pack(bits), m, n, "fused")
