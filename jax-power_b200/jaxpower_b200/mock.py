"""Synthetic catalogs on the GPU: Gaussian and lognormal mocks, Poisson-sampled.

- ``generate_gaussian_mesh`` follows ``mock.py:15-47`` of jax-power: unit white
  noise on the mesh, r2c, multiply by sqrt(P(k) / V_cell) (optionally fixing the
  amplitude to 1, ``unitary_amplitude``), c2r.
- ``lognormal_particles`` (not in the reference; used for the benchmark, batched
  and learned-correction catalogs): delta_LN = exp(delta_G - sigma^2 / 2) - 1, then
  Poisson counts with mean nbar V_cell (1 + delta_LN) per cell, positions uniform
  within each cell.
- ``generate_uniform_particles`` (``mock.py:180-207``): uniform positions in the box.

Random streams are torch's CUDA Philox generator, seeded; they are not
jax.random streams.
"""
import numpy as np
import torch

from .mesh import MeshAttrs, RealMeshField, ParticleField, _r2c, _c2r, _device

__all__ = ['power_law_pk', 'generate_gaussian_mesh', 'lognormal_particles', 'generate_uniform_particles']


def power_law_pk(amplitude=2e4, k0=0.1, index=-1.5, kcut=0.5):
    """P(k) = A (k / k0)^index exp(-(k / kcut)^2), P(0) = 0 (the benchmark spectrum)."""

    def pk(k):
        safe = torch.where(k > 0, k, torch.ones_like(k))
        p = amplitude * (safe / k0)**index * torch.exp(-(safe / kcut)**2)
        return torch.where(k > 0, p, torch.zeros_like(p))

    return pk


def _generator(seed):
    g = torch.Generator(device=_device())
    g.manual_seed(int(seed))
    return g


def generate_gaussian_mesh(mattrs, power, seed=42, unitary_amplitude=False):
    """Gaussian random field with power spectrum ``power(|k|)`` (``mock.py:15-47``)."""
    g = _generator(seed)
    shape = tuple(int(n) for n in mattrs.meshsize)
    noise = torch.randn(shape, generator=g, device=_device(), dtype=torch.float32)
    c = _r2c(noise, mattrs.meshsize)
    del noise
    kx, ky, kz = mattrs.kcoords(sparse=True)
    k = torch.sqrt((kx * kx + ky * ky) + kz * kz)
    ker = torch.sqrt(power(k) / float(np.prod(mattrs.cellsize.astype('f8'))))
    if unitary_amplitude:
        ker = ker * float(np.sqrt(np.prod(mattrs.meshsize.astype('f8')))) / c.abs().clamp_min(1e-30)
    c = c * ker
    return RealMeshField(_c2r(c, mattrs.meshsize, destroy_input=True), attrs=mattrs)


def lognormal_particles(mattrs, power, nbar, seed=42, return_mesh=False):
    """Poisson-sampled lognormal catalog; returns float32 positions (N, 3) on the device."""
    delta = generate_gaussian_mesh(mattrs, power, seed=seed).value
    sigma2 = float(delta.double().pow(2).mean())
    lam = torch.exp(delta - 0.5 * sigma2)  # 1 + delta_LN
    del delta
    vcell = float(np.prod(mattrs.cellsize.astype('f8')))
    lam.mul_(nbar * vcell)
    g = _generator(seed + 1)
    counts = torch.poisson(lam, generator=g).to(torch.int64).reshape(-1)
    del lam
    cells = torch.repeat_interleave(torch.arange(counts.numel(), device=counts.device), counts)
    del counts
    n1, n2 = int(mattrs.meshsize[1]), int(mattrs.meshsize[2])
    ijk = torch.stack([cells // (n1 * n2), (cells // n2) % n1, cells % n2], dim=1).to(torch.float32)
    del cells
    u = torch.rand(ijk.shape, generator=g, device=ijk.device, dtype=torch.float32)
    cell = torch.as_tensor(mattrs.cellsize, device=ijk.device)
    origin = torch.as_tensor(mattrs.boxcenter - mattrs.boxsize / 2., device=ijk.device)
    positions = ((ijk + u) * cell + origin).to(torch.float32).contiguous()
    if return_mesh:
        return positions, sigma2
    return positions


def generate_uniform_particles(mattrs, size, seed=42, exchange=False, **kwargs):
    """Uniform particles in the box (``mock.py:180-207``) as a ParticleField."""
    g = _generator(seed)
    u = torch.rand((int(size), 3), generator=g, device=_device(), dtype=torch.float32)
    box = torch.as_tensor(mattrs.boxsize, device=u.device)
    center = torch.as_tensor(mattrs.boxcenter, device=u.device)
    positions = box * u - box / 2. + center
    return ParticleField(positions, attrs=mattrs, **kwargs)
