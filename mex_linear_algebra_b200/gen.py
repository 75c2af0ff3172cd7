"""Seeded inputs of the benchmark configurations (numpy, host side).

All randomness is a counter-based splitmix64 stream: word i of stream
(seed, stream_id) is ``mix64(key + (i + 1) * GOLDEN)`` with
``key = mix64(seed * GOLDEN + C1) ^ mix64(stream_id + C2)``.  The device
generator ``mela_dev_rand_dense`` produces the same words, so the host and
the GPU build bit-identical inputs.

Configurations (seeds as in the benchmark definitions):

* dense products  -- ``dense_packed(seed, stream, m, n)``: word w of row i is
  stream word i*ceil(n/64)+w, bits past column n cleared.
* dense rank      -- ``rank_config``: A = L*R mod 2 (L m x r, R r x n from
  seed 2, streams 0 and 1), then ``rows_to_replace`` rows replaced, in order,
  by the XOR of two other rows (triples from stream 2).
* parity-check batch -- ``ldpc_batch``: matrix b of the batch takes its shape
  from words 0-2 of stream b (m uniform in [64, 1024]; n = 2m +/- uniform
  [0, m/4]) and the 6 distinct ones of each row by Floyd's sampling from
  words 3.. of the same stream.
* mixed request stream -- ``mixed_stream``: m, n, p log-uniform in
  [32, 8192], density log-uniform in [0.001, 0.5], aspect ratio <= 8:1.
* batch requests -- ``batch_requests``: homogeneous batches for timing the
  batched engines: m log-uniform in [32, 1024], n = m * [1, 3], density
  log-uniform in [0.002, 0.5], 64 to 4096 matrices.
"""
from __future__ import annotations

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_C1 = np.uint64(0x632BE59BD9B4E019)
_C2 = np.uint64(0xD1B54A32D192ED03)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def mix64(z):
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def stream_key(seed: int, stream: int) -> np.uint64:
    with np.errstate(over="ignore"):
        a = mix64(np.uint64(seed) * GOLDEN + _C1)
        b = mix64(np.uint64(stream) + _C2)
    return np.uint64(a ^ b)


def words(seed: int, stream: int, start: int, count: int) -> np.ndarray:
    key = stream_key(seed, stream)
    idx = np.arange(start + 1, start + 1 + count, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return mix64(key + idx * GOLDEN)


def dense_packed(seed: int, stream: int, m: int, n: int) -> np.ndarray:
    wc = (n + 63) // 64
    out = words(seed, stream, 0, m * wc).reshape(m, wc)
    if n % 64 and wc:
        out[:, -1] &= np.uint64((1 << (n % 64)) - 1)
    return out


def uniform_int(w: np.ndarray, lo: int, hi: int) -> np.ndarray:
    """Map words to integers in [lo, hi] (inclusive), by modulo."""
    return lo + (w % np.uint64(hi - lo + 1)).astype(np.int64)


# ------------------------------------------------------------------ dense rank
def replacement_triples(m: int, count: int, seed: int = 2, stream: int = 2):
    """`count` triples (i, a, b) of distinct rows: row i := row a ^ row b,
    applied in order.  Triple t uses words 3t..3t+2 of the stream; a word
    pair that collides is redrawn from the next unused words."""
    out = []
    pos = 0
    for _ in range(count):
        while True:
            w = words(seed, stream, pos, 3)
            pos += 3
            i, a, b = (int(x) for x in (w % np.uint64(m)))
            if len({i, a, b}) == 3:
                out.append((i, a, b))
                break
    return out


# ------------------------------------------------------------------ parity-check batch
def ldpc_shape(seed: int, b: int):
    w = words(seed, b, 0, 3)
    m = int(uniform_int(w[0:1], 64, 1024)[0])
    d = int(w[1] % np.uint64(m // 4 + 1))
    n = 2 * m + d if (int(w[2]) & 1) else 2 * m - d
    return m, n


def ldpc_rows(seed: int, b: int, m: int, n: int, k: int = 6) -> np.ndarray:
    """(m, k) column indices, distinct per row, by Floyd's algorithm: for
    j = n-k .. n-1, t = word % (j + 1); take t unless already taken, else j."""
    w = words(seed, b, 3, m * k).reshape(m, k)
    cols = np.empty((m, k), dtype=np.int64)
    for s in range(k):
        j = n - k + s
        t = (w[:, s] % np.uint64(j + 1)).astype(np.int64)
        taken = (cols[:, :s] == t[:, None]).any(axis=1) if s else np.zeros(m, bool)
        cols[:, s] = np.where(taken, j, t)
    return cols


def ldpc_packed(seed: int, b: int):
    """Matrix b of the batch, packed (m x ceil(n/64) uint64)."""
    m, n = ldpc_shape(seed, b)
    cols = ldpc_rows(seed, b, m, n)
    wc = (n + 63) // 64
    P = np.zeros((m, wc), dtype=np.uint64)
    rows = np.repeat(np.arange(m), cols.shape[1])
    flat = cols.ravel()
    np.add.at(P, (rows, flat >> 6), np.left_shift(np.uint64(1), (flat & 63).astype(np.uint64)))
    return m, n, P


def ldpc_batch(count: int = 20000, seed: int = 3):
    """The whole batch packed back to back.  Returns (shapes (count, 2) int64,
    word offsets (count,) int64, buffer uint64)."""
    shapes = np.array([ldpc_shape(seed, b) for b in range(count)], dtype=np.int64)
    wcs = (shapes[:, 1] + 63) // 64
    sizes = shapes[:, 0] * wcs
    offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    buf = np.zeros(int(sizes.sum()), dtype=np.uint64)
    for b in range(count):
        m, n = int(shapes[b, 0]), int(shapes[b, 1])
        cols = ldpc_rows(seed, b, m, n)
        wc = int(wcs[b])
        rows = np.repeat(np.arange(m), cols.shape[1])
        flat = cols.ravel()
        idx = offsets[b] + rows * wc + (flat >> 6)
        np.add.at(buf, idx, np.left_shift(np.uint64(1), (flat & 63).astype(np.uint64)))
    return shapes, offsets, buf


# ------------------------------------------------------------------ mixed request stream
def mixed_stream(count: int = 50000, seed: int = 4):
    """Request list: dicts with op ('rank', 'null', 'matmul'), m, n, p (the
    product's right width) and density.  Word layout per request r: 6 words
    of stream 0 at 6r."""
    w = words(seed, 0, 0, 6 * count).reshape(count, 6).astype(np.float64) / 2.0 ** 64
    lo, hi = np.log(32.0), np.log(8192.0)
    m = np.exp(lo + (hi - lo) * w[:, 0])
    n = np.exp(lo + (hi - lo) * w[:, 1])
    # aspect ratio at most 8:1
    n = np.clip(n, m / 8, m * 8)
    n = np.clip(n, 32, 8192)
    p = np.exp(lo + (hi - lo) * w[:, 2])
    dens = np.exp(np.log(0.001) + (np.log(0.5) - np.log(0.001)) * w[:, 3])
    op = (w[:, 4] * 3).astype(np.int64)
    names = np.array(["rank", "null", "matmul"])[op]
    return [dict(op=str(names[i]), m=int(round(m[i])), n=int(round(n[i])), p=int(round(p[i])),
                 density=float(dens[i]), stream=i) for i in range(count)]


def batch_requests(count: int, seed: int = 4, offset: int = 0):
    """Batch requests: dicts with op 'batch', m, n, density and batch_count
    (the number of m x n matrices in the batch).  Word layout per request r:
    4 words of stream 1 at 4(offset + r).  Batches hold at most 2^30 bits."""
    if count <= 0:
        return []
    w = words(seed, 1, 4 * offset, 4 * count).reshape(count, 4).astype(np.float64) / 2.0 ** 64
    m = np.exp(np.log(32.0) + (np.log(1024.0) - np.log(32.0)) * w[:, 0])
    n = m * (1.0 + 2.0 * w[:, 1])
    dens = np.exp(np.log(0.002) + (np.log(0.5) - np.log(0.002)) * w[:, 2])
    cnt = (64 * 4 ** np.floor(w[:, 3] * 4)).astype(np.int64)  # 64, 256, 1024, 4096
    out = []
    for i in range(count):
        mi, ni = int(round(m[i])), int(round(n[i]))
        c = int(cnt[i])
        while c > 64 and c * mi * ni > (1 << 30):
            c //= 4
        out.append(dict(op="batch", m=mi, n=ni, p=0, density=float(dens[i]), batch_count=c,
                        stream=offset + i))
    return out


def batch_requests_sparse(count: int, seed: int = 4, offset: int = 0):
    """Batch requests shaped like parity-check batches: m log-uniform in
    [48, 600], n = m * [1.5, 2.5], density log-uniform in [0.003, 0.1],
    1024, 4096 or 16384 matrices (fewer when the batch would pass 2^31
    bits).  Word layout per request r: 4 words of stream 2 at 4(offset + r)."""
    if count <= 0:
        return []
    w = words(seed, 2, 4 * offset, 4 * count).reshape(count, 4).astype(np.float64) / 2.0 ** 64
    m = np.exp(np.log(48.0) + (np.log(600.0) - np.log(48.0)) * w[:, 0])
    n = m * (1.5 + w[:, 1])
    dens = np.exp(np.log(0.003) + (np.log(0.1) - np.log(0.003)) * w[:, 2])
    cnt = (1024 * 4 ** np.floor(w[:, 3] * 3)).astype(np.int64)  # 1024, 4096, 16384
    out = []
    for i in range(count):
        mi, ni = int(round(m[i])), int(round(n[i]))
        c = int(cnt[i])
        while c > 1024 and c * mi * ni > (1 << 31):
            c //= 4
        out.append(dict(op="batch", m=mi, n=ni, p=0, density=float(dens[i]), batch_count=c,
                        stream=200000 + offset + i))
    return out


def sparse_packed(seed: int, stream: int, m: int, n: int, density: float) -> np.ndarray:
    """Bernoulli(density) packed matrix: bit set when the 16-bit slice of a
    stream word is below density*65536 (4 entries per word)."""
    k = m * n
    w = words(seed, stream, 0, (k + 3) // 4)
    sl = np.stack([(w >> np.uint64(16 * q)) & np.uint64(0xFFFF) for q in range(4)], axis=1).ravel()[:k]
    bits = (sl < np.uint64(int(density * 65536))).reshape(m, n)
    return _pack_bool(bits)


def _pack_bool(bits: np.ndarray) -> np.ndarray:
    m, n = bits.shape
    wc = (n + 63) // 64
    pad = np.zeros((m, wc * 64), dtype=np.uint8)
    pad[:, :n] = bits
    b8 = np.packbits(pad, axis=1, bitorder="little")  # (m, wc*8) bytes, bit j -> byte j/8 bit j%8
    return b8.view(np.uint64).reshape(m, wc).copy()
