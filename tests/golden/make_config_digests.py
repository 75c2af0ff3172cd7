"""Digests of the benchmark configurations' exact results, from the checker.

The full-size configurations are too large to keep their results as
fixtures, so this script stores digests of them (BLAKE2b, 16 bytes, over the
packed words), computed on the CPU by the oracle (oracle/mela_oracle.c) and,
where it finishes in reasonable time, also by the reference's own gateways
compiled into oracle/_ref (both must agree before anything is written):

* product_32768: C = A*B, A and B 32768 x 32768 from seed 1 (streams 0 and
  1 of the shared generator), packed.  Digest of all of C and of each block
  of 1024 rows.  Oracle: orc_matmul (the reference's XOR-row loop).  With
  --reference-product the reference's mela_matmul_gf2 also runs at full size
  on logical input (about ten minutes on 8 cores, 3 GiB of host memory).
* matmul_gateway_2048: the drop-in call mela_matmul_gf2(A, B) with A
  2048 x 2048 and B 2048 x 1024 double 0/1 from seed 0: digest of the packed
  logical output, from the reference gateway and the oracle.
* dense_16384x32768: the rank-12000 matrix of make_dense_rank.py.  Pivot
  columns, RREF rows (in pivot order) and the null-space basis Zt (row i =
  basis vector i, free columns ascending).  The RREF comes from orc_rref;
  the basis follows from it (Zt row i has bit f_i and, at pivot column c_p,
  bit RREF(p, f_i) -- the unique solution the reference's back-substitution
  computes; tests/test_oracle_pins.py checks that identity on small inputs).
* ldpc_20000 (ldpc_20000.npz): for every matrix of the parity-check batch
  (seed 3), its rank and the digest of its null-space basis Zt from
  oracle.null_basis_packed; a spread sample is also run through the
  reference gateways mela_rank_gf2 / mela_null_gf2.

    python tests/golden/make_config_digests.py [--reference-product] [--only NAME]
"""
import argparse
import hashlib
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import numpy as np  # noqa: E402

OUT_JSON = os.path.join(HERE, "config_digests.json")
OUT_LDPC = os.path.join(HERE, "ldpc_20000.npz")


def digest(words: np.ndarray) -> str:
    """BLAKE2b-128 of a packed array's bytes (row-major uint64 words)."""
    return hashlib.blake2b(np.ascontiguousarray(words, dtype=np.uint64).tobytes(), digest_size=16).hexdigest()


def null_from_rref(R: np.ndarray, piv: np.ndarray, n: int) -> np.ndarray:
    """Zt (f x words(n)) of the null space from RREF rows R (r x words) and
    ascending pivot columns: row i = e_{f_i} + sum_p R[p, f_i] e_{piv[p]}."""
    r = len(piv)
    free = np.setdiff1d(np.arange(n), piv)
    f = len(free)
    wc = (n + 63) // 64
    Rb = np.unpackbits(np.ascontiguousarray(R[:r]).view(np.uint8).reshape(r, wc * 8), axis=1,
                       bitorder="little")[:, :n]  # r x n
    Z = np.zeros((f, wc * 64), dtype=np.uint8)
    Z[np.arange(f), free] = 1
    Z[:, piv] = Rb[:, free].T
    del Rb
    out = np.packbits(Z, axis=1, bitorder="little").view(np.uint64).reshape(f, wc)
    return out


def product_32768(reference: bool):
    import oracle as O
    n = 32768
    A = O.rand_dense(1, 0, n, n)
    B = O.rand_dense(1, 1, n, n)
    t0 = time.time()
    Cp = O.matmul(A, B, n, n, n)
    t1 = time.time()
    rec = {"shape": [n, n, n], "seed": 1, "digest": digest(Cp),
           "row_block": 1024, "block_digests": [digest(Cp[i:i + 1024]) for i in range(0, n, 1024)],
           "oracle_seconds": round(t1 - t0, 1), "reference_checked": False}
    if reference:
        Al = O.unpack(A, n, n)
        Bl = O.unpack(B, n, n)
        t2 = time.time()
        (Cl,) = O.ref_call("mela_matmul_gf2", Al, Bl)
        rec["reference_seconds"] = round(time.time() - t2, 1)
        del Al, Bl
        Cr = O.pack(Cl)
        del Cl
        assert np.array_equal(Cr, Cp), "reference and oracle disagree on the 32768^3 product"
        rec["reference_checked"] = True
    return rec


def matmul_gateway_2048():
    import oracle as O
    m, k, n = 2048, 2048, 1024
    A = O.unpack(O.rand_dense(0, 0, m, k), m, k).astype(np.float64)
    B = O.unpack(O.rand_dense(0, 1, k, n), k, n).astype(np.float64)
    (Cl,) = O.ref_call("mela_matmul_gf2", A, B)
    Cp = O.pack(Cl)
    want = O.matmul(O.rand_dense(0, 0, m, k), O.rand_dense(0, 1, k, n), m, k, n)
    assert np.array_equal(Cp, want), "reference and oracle disagree on the 2048 product"
    return {"shape": [m, k, n], "seed": 0, "input": "double 0/1, column-major",
            "digest": digest(Cp), "ones": int(np.asfortranarray(Cl).sum()), "reference_checked": True}


def dense_16384x32768():
    import oracle as O
    import make_dense_rank as MD
    A = MD.build()
    m, n = MD.M, MD.N
    t0 = time.time()
    R, piv = O.rref(A, m, n)
    t1 = time.time()
    r = len(piv)
    Zt = null_from_rref(R, piv, n)
    return {"m": m, "n": n, "rank": r, "pivots_digest": digest(piv.astype(np.uint64)),
            "rref_rows_digest": digest(R[:r]), "null_digest": digest(Zt), "nullity": int(Zt.shape[0]),
            "oracle_rref_seconds": round(t1 - t0, 1)}


def _ldpc_one(b):
    import oracle as O
    from mex_linear_algebra_b200 import gen
    m, n, P = gen.ldpc_packed(3, b)
    Zt = O.null_basis_packed(P, m, n)
    return b, n - Zt.shape[0], digest(Zt)


def _ldpc_ref(b):
    import oracle as O
    from mex_linear_algebra_b200 import gen
    m, n, P = gen.ldpc_packed(3, b)
    H = O.unpack(P, m, n)
    (rk,) = O.ref_call("mela_rank_gf2", H)
    (Z,) = O.ref_call("mela_null_gf2", H)
    Zt = O.pack(np.asfortranarray(Z.T)) if Z.shape[1] else np.zeros((0, (n + 63) // 64), np.uint64)
    return b, int(rk[0, 0]), digest(Zt)


def ldpc_20000(count=20000, ref_sample=200):
    os.environ["OMP_NUM_THREADS"] = "1"
    ctx = mp.get_context("spawn")
    with ctx.Pool(os.cpu_count()) as pool:
        res = pool.map(_ldpc_one, range(count), chunksize=64)
        sample = np.linspace(0, count - 1, ref_sample).astype(np.int64).tolist()
        ref = pool.map(_ldpc_ref, sample, chunksize=4)
    ranks = np.array([r for (_, r, _) in res], dtype=np.int32)
    digs = [bytes.fromhex(d) for (_, _, d) in res]
    for (b, rk, d) in ref:
        assert rk == ranks[b] and bytes.fromhex(d) == digs[b], f"reference disagrees on matrix {b}"
    dig_arr = np.frombuffer(b"".join(digs), dtype=np.uint8).reshape(count, 16)
    np.savez_compressed(OUT_LDPC, ranks=ranks, null_digests=dig_arr,
                        reference_checked=np.array(sample, dtype=np.int64))
    return {"count": count, "seed": 3, "file": os.path.basename(OUT_LDPC),
            "rank_sum": int(ranks.sum()), "reference_checked": len(sample)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-product", action="store_true")
    ap.add_argument("--only", choices=["product_32768", "matmul_gateway_2048", "dense_16384x32768",
                                       "ldpc_20000"])
    a = ap.parse_args()
    sys.path.insert(0, HERE)
    out = json.load(open(OUT_JSON)) if os.path.exists(OUT_JSON) else {}
    jobs = {"matmul_gateway_2048": matmul_gateway_2048, "dense_16384x32768": dense_16384x32768,
            "ldpc_20000": ldpc_20000, "product_32768": lambda: product_32768(a.reference_product)}
    for name, fn in jobs.items():
        if a.only and name != a.only:
            continue
        t0 = time.time()
        out[name] = fn()
        print(name, round(time.time() - t0, 1), "s", flush=True)
        with open(OUT_JSON, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
