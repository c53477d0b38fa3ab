"""The reference's seeded initial vectors on the host (Executor::create_random_vector /
create_random_multivector, src/core/Executor.cpp:20-62): ``std::mt19937(seed)`` with
``std::uniform_real_distribution<double>(-1, 1)``, whose libstdc++
``generate_canonical<double, 53>`` draws two 32-bit words per value (low word first),
filled column-major. NumPy's MT19937 with legacy seeding produces the same word stream.
Used by the multi-GPU driver, whose shards take row ranges of the same global block."""
from __future__ import annotations

import numpy as np


def _stream(seed: int):
    bg = np.random.MT19937(0)
    bg._legacy_seeding(int(seed) & 0xFFFFFFFF)
    return bg


def _canonical(raw: np.ndarray) -> np.ndarray:
    # lo + hi * 2^32 formed exactly as a 64-bit integer, rounded once to double, as the
    # double sum of generate_canonical rounds it; values at 1 are moved below 1.
    v = ((raw[1::2] << np.uint64(32)) | raw[0::2]).astype(np.float64)
    v *= 1.0 / 18446744073709551616.0
    np.minimum(v, np.nextafter(1.0, 0.0), out=v)
    return 2.0 * v - 1.0


def random_vector(n: int, seed: int) -> np.ndarray:
    return _canonical(_stream(seed).random_raw(2 * n))


def random_block_rows(n: int, cols: int, seed: int, r0: int, r1: int) -> np.ndarray:
    """Rows r0..r1 of the column-major n x cols block, as a row-major array."""
    bg = _stream(seed)
    out = np.empty((r1 - r0, cols))
    for j in range(cols):
        if r0 > 0:
            bg.random_raw(2 * r0)
        out[:, j] = _canonical(bg.random_raw(2 * (r1 - r0)))
        if n - r1 > 0:
            bg.random_raw(2 * (n - r1))
    return out
