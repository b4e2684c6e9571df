"""jaxpower_b200: B200-native (sm_100a) drop-in for jax-power's mesh power-spectrum path.

Public API mirrors ``jaxpower`` for the single-GPU power-spectrum estimator:
``MeshAttrs``, ``RealMeshField``, ``ComplexMeshField``, ``ParticleField``, ``FKPField``,
``get_mesh_attrs``, ``BinMesh2SpectrumPoles``, ``compute_mesh2_spectrum``,
``compute_fkp2_normalization``, ``compute_fkp2_shotnoise``, ``compute_box2_normalization``,
``BinMesh2CorrelationPoles`` (separation bins with mode oversampling, or the spherical-Bessel
basis), ``compute_mesh2_correlation``, ``compute_mesh2_spectrum_window`` /
``compute_mesh2_spectrum_mean`` (``WindowMatrix``; global, first-point and end-point lines of
sight, 'firstpoint' and 'local' theory, wide-angle orders, 'smooth' and 'infinite' flags),
``compute_smooth2_spectrum_window`` and the ``resamplers`` namespaces; differentiable paint and
spectrum in ``jaxpower_b200.autodiff``.  All computation runs in the CUDA library
``libjaxpower_b200.so`` through its C ABI (``include/jaxpower_b200.h``).
"""
from . import resamplers
from .mesh import (MeshAttrs, BaseMeshField, RealMeshField, ComplexMeshField, ParticleField, FKPField,
                   get_mesh_attrs, next_fft_size, r2c, c2r, apply, read, paint, split_particles)
from .mesh2 import (BinMesh2SpectrumPoles, BinMesh2CorrelationPoles, compute_mesh2_spectrum,
                    compute_mesh2_correlation, compute_mesh2, compute_fkp2_normalization,
                    compute_fkp2_shotnoise, compute_box2_normalization, compute_normalization,
                    compute_box_normalization, compute_mesh2_spectrum_window,
                    compute_mesh2_spectrum_mean, compute_smooth2_spectrum_window)
from .types import (Mesh2SpectrumPole, Mesh2SpectrumPoles, Mesh2CorrelationPole, Mesh2CorrelationPoles, WindowMatrix,
                    read, write)
from ._lib import load as load_library, LIBRARY_PATH

__version__ = '0.1.0'
