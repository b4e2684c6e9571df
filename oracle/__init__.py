"""CPU oracle for the mesh power-spectrum path (TEST INFRASTRUCTURE ONLY).

This package restates, in NumPy/SciPy, the arithmetic of jax-power's
single-GPU power-spectrum estimator:

- ``resamplers.py:57-125``  resampler kernels, paint (scatter) and read (gather)
- ``resamplers.py:16-26``   compensation window
- ``mesh.py:360-403``       fftfreq coordinates (k / position grids)
- ``mesh.py:1559-1636``     cellsize, kfun, knyq, rcoords / kcoords
- ``mesh.py:2673-2754``     ``_paint``: normalisation, interlacing, compensation
- ``mesh.py:2812-2910``     Hermitian weights, digitize, bincount
- ``mesh2.py:25-119``       k edges, nmodes, xavg
- ``mesh2.py:253-374``      global and first-point estimators
- ``utils.py:190-360``      real Y_lm and Legendre polynomials
- ``mesh.py:2913-2999``, ``mesh2.py:508-621``  FKP field, normalisation, shot noise
- ``mesh.py:2226-2381``     ``get_mesh_attrs`` / ``next_fft_size``

It exists only to check the CUDA library.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm
may import it, and only as the checker or the timed CPU baseline.  The
product package never imports it.

Parity status.  The reference (JAX) cannot run on the build or GPU machines
(no jax / jaxlib).  The restatement is pinned by:

- the reference's own invariants (mass conservation ``tests/test_mesh.py:119,231``,
  Gaussian-mesh P0 recovery ``tests/test_mesh2.py:60``, shot-noise identities
  ``tests/test_mesh2.py:86-91``, Y_lm vs SciPy ``tests/test_mesh2.py:467``);
- the reference's golden value ``tests/test_mesh.py:211``
  (``mesh.std() == 0.6890684579054714`` for TSC, interlacing 3, compensate,
  1e6 ``jax.random`` positions on a 256x128x64 mesh), reproduced through a
  NumPy restatement of JAX's Threefry-2x32 stream (``threefry.py``) — see
  ``tests/test_oracle_golden.py`` for which stream variant matches.

Two arithmetic modes:

- ``dtype=np.float32``: "reference order" — the float32 operation order of the
  reference (serial scatter-add in particle order, float32 bincounts);
- ``dtype=np.float64``: the same algorithm in float64, used to report errors.
"""
