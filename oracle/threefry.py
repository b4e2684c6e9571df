"""NumPy restatement of JAX's default PRNG stream (oracle; test only).

The reference's golden test values (``tests/test_mesh.py:186-213``) are computed
from ``jax.random`` streams.  jax / jaxlib are third-party, unpinned in the
reference (``pyproject.toml:14``) and absent here, so their published algorithm
is restated:

- Threefry-2x32 with 20 rounds (Salmon et al., "Parallel random numbers: as easy
  as 1, 2, 3", SC 2011): key schedule ``ks2 = k0 ^ k1 ^ 0x1BD11BDA``, rotation
  constants (13, 15, 26, 6) / (17, 29, 16, 24), key injection every 4 rounds;
- ``random.key(seed)``: key words ``[seed >> 32, seed & 0xFFFFFFFF]``;
- ``random_bits`` in both JAX layouts: the original one (counter ``iota(n)``
  split in two halves, outputs concatenated) and the ``jax_threefry_partitionable``
  one (counter = 64-bit flat index as (hi, lo), output ``y0 ^ y1``), the default
  since JAX 0.5;
- ``random.uniform`` for float32: ``bitcast((bits >> 9) | 0x3F800000) - 1``, and
  for float64: ``bitcast((bits64 >> 12) | 0x3FF0...) - 1``.

Checked against the Random123 / JAX known-answer vectors in
``tests/test_oracle_golden.py``.
"""
import numpy as np

_ROT = (13, 15, 26, 6, 17, 29, 16, 24)


def _rotl(x, r):
    return ((x << np.uint32(r)) | (x >> np.uint32(32 - r))).astype(np.uint32)


def threefry2x32(key, x0, x1):
    """Threefry-2x32-20 of counters (x0, x1) (uint32 arrays) under key (k0, k1)."""
    k0 = np.asarray(key[0], dtype=np.uint32)
    k1 = np.asarray(key[1], dtype=np.uint32)
    k2 = (k0 ^ k1 ^ np.uint32(0x1BD11BDA)).astype(np.uint32)
    ks = (k0, k1, k2)
    shape = np.broadcast_shapes(np.shape(x0), np.shape(x1), k0.shape, k1.shape)
    x0 = np.broadcast_to(np.asarray(x0, dtype=np.uint32), shape).copy()
    x1 = np.broadcast_to(np.asarray(x1, dtype=np.uint32), shape).copy()
    with np.errstate(over='ignore'):
        x0 += ks[0]
        x1 += ks[1]
        for block in range(5):
            rots = _ROT[:4] if block % 2 == 0 else _ROT[4:]
            for r in rots:
                x0 += x1
                x1 = _rotl(x1, r)
                x1 ^= x0
            x0 += ks[(block + 1) % 3]
            x1 += (ks[(block + 2) % 3] + np.uint32(block + 1)).astype(np.uint32)
    return x0, x1


def fold_in(key, data):
    """``jax.random.fold_in(key, uint32 data)``: threefry2x32(key, (0, data)) (vectorised over data)."""
    data = np.asarray(data, dtype=np.uint32)
    return threefry2x32(key, np.zeros_like(data), data)


def fold_in_index(key, ids):
    """``_fold_in`` of the reference (``mesh.py:215-233``) for int64 ids: fold low then high word."""
    ids = np.asarray(ids, dtype=np.uint64)
    lo = (ids & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    hi = (ids >> np.uint64(32)).astype(np.uint32)
    return fold_in(fold_in(key, lo), hi)


def uniform_per_key(keys, m, dtype=np.float64):
    """``vmap(lambda k: uniform(k, (m,), dtype))(keys)`` (partitionable layout): (n, m) array."""
    k0, k1 = keys
    k0 = np.asarray(k0, np.uint32)[:, None]
    k1 = np.asarray(k1, np.uint32)[:, None]
    j = np.arange(m, dtype=np.uint32)[None, :]
    y0, y1 = threefry2x32((k0, k1), np.zeros_like(j), j)
    if np.dtype(dtype) == np.float32:
        bits = y0 ^ y1
        return ((bits >> np.uint32(9)) | np.uint32(0x3F800000)).view(np.float32) - np.float32(1.)
    bits = (y0.astype(np.uint64) << np.uint64(32)) | y1.astype(np.uint64)
    return ((bits >> np.uint64(12)) | np.uint64(0x3FF0000000000000)).view(np.float64) - 1.


def seed_key(seed):
    seed = int(seed)
    return (np.uint32((seed >> 32) & 0xFFFFFFFF), np.uint32(seed & 0xFFFFFFFF))


def random_bits32(key, n, partitionable=True):
    """``_random_bits(key, 32, (n,))`` in either JAX layout."""
    if partitionable:
        idx = np.arange(n, dtype=np.uint64)
        hi = (idx >> np.uint64(32)).astype(np.uint32)
        lo = (idx & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        y0, y1 = threefry2x32(key, hi, lo)
        return y0 ^ y1
    count = np.arange(n, dtype=np.uint32)
    odd = n % 2
    if odd:
        count = np.concatenate([count, np.zeros(1, np.uint32)])
    half = count.size // 2
    y0, y1 = threefry2x32(key, count[:half], count[half:])
    out = np.concatenate([y0, y1])
    return out[:-1] if odd else out


def random_bits64(key, n, partitionable=True):
    if partitionable:
        idx = np.arange(n, dtype=np.uint64)
        hi = (idx >> np.uint64(32)).astype(np.uint32)
        lo = (idx & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        y0, y1 = threefry2x32(key, hi, lo)
        return (y0.astype(np.uint64) << np.uint64(32)) | y1.astype(np.uint64)
    bits = random_bits32(key, 2 * n, partitionable=False)
    a, b = bits[:n].astype(np.uint64), bits[n:].astype(np.uint64)
    return (a << np.uint64(32)) | b


def uniform(key, shape, dtype=np.float32, partitionable=True):
    """``jax.random.uniform(key, shape, dtype)`` on [0, 1)."""
    n = int(np.prod(shape))
    if np.dtype(dtype) == np.float32:
        bits = random_bits32(key, n, partitionable)
        f = ((bits >> np.uint32(9)) | np.uint32(0x3F800000)).view(np.float32) - np.float32(1.)
    else:
        bits = random_bits64(key, n, partitionable)
        f = ((bits >> np.uint64(12)) | np.uint64(0x3FF0000000000000)).view(np.float64) - 1.
    return np.maximum(np.asarray(0., dtype), f.reshape(shape))
