"""The batched engine's pivot choice leaves the results unchanged (CPU).

Per 64-column panel the GPU engine takes its pivots among the candidate rows
(unused rows with a nonzero panel word) in the order one warp sees them:
candidate c sits in lane c % 32, slot c // 32, and for each bit the first
lane (then its first slot) holding the bit wins -- not the lowest row, which
the reference's elimination takes.  The reduced row echelon form of a matrix
is unique, so rank, pivot columns, RREF rows and the null basis read off it
do not depend on that choice.  This test replays the panel-blocked
Gauss-Jordan elimination with the warp's choice in numpy and compares every
output with the oracle's.
"""
import numpy as np
import pytest

import oracle as O


def _bits(P, m, n):
    wc = P.shape[1]
    b = np.unpackbits(P.view(np.uint8).reshape(m, wc * 8), axis=1, bitorder="little")
    return b[:, :n].astype(np.uint8)


def _eliminate_warp_order(B, warp_order=True):
    """RREF of the 0/1 matrix B by 64-column panels with the warp's pivot choice
    (or, warp_order=False, the lowest row); returns (rref rows in pivot order,
    pivot columns, physical pivot rows)."""
    A = B.copy()
    m, n = A.shape
    used = np.zeros(m, bool)
    pivots = []  # (column, row)
    for c0 in range(0, n, 64):
        cols = range(c0, min(c0 + 64, n))
        cand = [j for j in range(m) if not used[j] and A[j, c0:c0 + 64].any()]
        # warp order: lane-major, then slot
        order = sorted(range(len(cand)), key=(lambda c: (c % 32, c // 32)) if warp_order else (lambda c: c))
        panel_used = set()
        for col in cols:
            hold = [cand[c] for c in order if cand[c] not in panel_used and A[cand[c], col]]
            if not hold:
                continue
            p = hold[0]
            panel_used.add(p)
            others = np.nonzero(A[:, col])[0]
            for j in others:
                if j != p:
                    A[j] ^= A[p]
            pivots.append((col, p))
        for p in panel_used:
            used[p] = True
    piv = np.array([c for c, _ in pivots], dtype=np.int64)
    rows = np.array([A[p] for _, p in pivots], dtype=np.uint8).reshape(len(pivots), n)
    return rows, piv, [p for _, p in pivots]


@pytest.mark.parametrize("seed,m,n,density", [(1, 40, 150, 0.5), (2, 90, 200, 0.05), (3, 130, 70, 0.3),
                                              (4, 70, 260, 0.02), (5, 100, 100, 0.5)])
def test_warp_pivot_order_gives_the_reference_rref(seed, m, n, density):
    rng = np.random.default_rng(seed)
    B = (rng.random((m, n)) < density).astype(np.uint8)
    B[m // 3] = B[1] ^ B[2]  # a dependent row
    wc = (n + 63) // 64
    pad = np.zeros((m, wc * 64), dtype=np.uint8)
    pad[:, :n] = B
    P = np.packbits(pad, axis=1, bitorder="little").view(np.uint64).reshape(m, wc)
    want_R, want_piv = O.rref(P, m, n)
    rows, piv, prow = _eliminate_warp_order(B)
    assert np.array_equal(piv, want_piv)
    assert np.array_equal(rows, _bits(want_R[:len(want_piv)], len(want_piv), n))
    if m > 64 and density >= 0.3:  # enough candidates for the two orders to pick other rows
        assert prow != _eliminate_warp_order(B, warp_order=False)[2]
