"""Regenerate the reference tests' input catalogs from the restated JAX PRNG.

The reference's golden values (``reference_goldens.json``) are computed on
``jax.random`` catalogs; ``oracle.threefry`` restates that stream, so the inputs
are rebuilt here instead of being stored.

- ``paint_jit_positions``: ``random.uniform(random.key(64), (1000000, 3))`` in
  float64 (``tests/test_mesh.py:189``);
- ``uniform_particles``: ``generate_uniform_particles(mattrs, size, seed=(seed, 'index'))``
  (``mock.py:180-207`` with ``mesh.py:237-329``): per particle, key =
  ``fold_in(fold_in(key(seed), id_lo), id_hi)``, 3 float64 uniforms.
"""
import numpy as np

from oracle.threefry import fold_in_index, seed_key, uniform, uniform_per_key


def paint_jit_positions(seed=64, n=1000000):
    return uniform(seed_key(seed), (n, 3), np.float64, partitionable=True)


def uniform_particles(seed, size, boxsize, boxcenter):
    keys = fold_in_index(seed_key(seed), np.arange(size))
    u = uniform_per_key(keys, 3, np.float64)
    boxsize = np.broadcast_to(np.asarray(boxsize, 'f8'), (3,))
    boxcenter = np.broadcast_to(np.asarray(boxcenter, 'f8'), (3,))
    return boxsize * u - boxsize / 2. + boxcenter
