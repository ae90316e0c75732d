"""Seeded synthetic workloads with the shapes of the reference's experiments.

The reference generates its datasets as text files seeded with ``time(0)``
(src/generator.h:138-227); these generators are in-memory and seeded, so the
CUDA path, the oracle and the reference harness all see the same arrays.
Seeds are ``0xF17C0001 + workload index``.
"""
from __future__ import annotations

import numpy as np

SEED_BASE = 0xF17C0001


def rng_for(index: int, salt: int = 0) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(SEED_BASE + index + (salt << 8)))


def distinct_pool(rng: np.random.Generator, count: int, bits: int) -> np.ndarray:
    """`count` distinct values drawn uniformly from [0, 2^bits)."""
    return rng.choice(np.uint64(1) << np.uint64(bits), size=count, replace=False).astype(np.uint64)


def cols_17b33(n: int = 16_777_216, seed_index: int = 1):
    """Two columns: col0 holds 17-bit codes drawn i.i.d. from a pool of 8,192
    distinct values (uint32); col1 holds uniform 33-bit codes (uint64)."""
    rng = rng_for(seed_index)
    pool = distinct_pool(rng, 8192, 17).astype(np.uint32)
    col0 = pool[rng.integers(0, pool.shape[0], size=n)]
    col1 = rng.integers(0, 1 << 33, size=n, dtype=np.uint64)
    return [col0, col1], [17, 33]


def cols_zipf(n: int = 67_108_864, seed_index: int = 3, ranks_bits: int = 20, s: float = 1.0):
    """col0 = perm(rank), rank ~ Zipf(s) over 2^ranks_bits ranks by inverse CDF
    (20-bit codes, uint32); col1 uniform 24-bit (uint32); col2 uniform 40-bit
    (uint64)."""
    rng = rng_for(seed_index)
    nr = 1 << ranks_bits
    w = 1.0 / np.power(np.arange(1, nr + 1, dtype=np.float64), s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    u = rng.random(n)
    rank = np.searchsorted(cdf, u, side="right").astype(np.uint32)
    rank = np.minimum(rank, nr - 1)
    perm = rng.permutation(nr).astype(np.uint32)
    col0 = perm[rank]
    col1 = rng.integers(0, 1 << 24, size=n, dtype=np.uint32)
    col2 = rng.integers(0, 1 << 40, size=n, dtype=np.uint64)
    return [col0, col1, col2], [ranks_bits, 24, 40]


def cols_uniform(n: int, widths, seed_index: int = 9, distinct=None):
    """Independent uniform columns of the given widths, stored at the reference's
    width->type mapping (src/generator.h:88-94: <=16 bits u16, <=32 u32, else
    u64).  distinct[c], when given, draws column c from a pool of that many
    distinct values."""
    rng = rng_for(seed_index)
    cols = []
    for c, w in enumerate(widths):
        dt = np.uint16 if w <= 16 else (np.uint32 if w <= 32 else np.uint64)
        if distinct is not None and distinct[c]:
            k = min(int(distinct[c]), 1 << w)
            pool = distinct_pool(rng, k, w).astype(dt)
            cols.append(pool[rng.integers(0, k, size=n)])
        elif w == 64:
            cols.append(rng.integers(0, np.iinfo(np.uint64).max, size=n, dtype=np.uint64, endpoint=True))
        else:
            cols.append(rng.integers(0, 1 << w, size=n, dtype=np.uint64).astype(dt))
    return cols, list(widths)


def split_for_k(k: int, w0: int = 17, w1: int = 33):
    """Bit-borrowing split [w0-k, w1+k] (TwoRoundsExhaustive,
    src/stitch_composer.cpp:4197-4258); k = w0 gives the single bank [w0+w1]."""
    a, b = w0 - k, w1 + k
    return [x for x in (a, b) if x > 0]
