"""Synthetic catalogs on the GPU: Gaussian and lognormal mocks, Poisson-sampled.

- ``generate_gaussian_mesh`` follows ``mock.py:15-47`` of jax-power: unit white
  noise on the mesh, r2c, multiply by sqrt(P(k) / V_cell) (optionally fixing the
  amplitude to 1, ``unitary_amplitude``), c2r.
- ``lognormal_particles`` (not in the reference; used for the benchmark, batched
  and learned-correction catalogs): delta_LN = exp(delta_G - sigma^2 / 2) - 1, then
  Poisson counts with mean nbar V_cell (1 + delta_LN) per cell, positions uniform
  within each cell.
- ``generate_uniform_particles`` (``mock.py:180-207``): uniform positions in the box.
- ``cutsky_particles`` (not in the reference; the cut-sky FKP benchmark catalog): data
  and randoms in a spherical shell within a cap around +z seen from the origin, with a
  Gaussian radial density n(r); data clustered by a lognormal field, FKP weights
  1 / (1 + n(r) P0).

Random streams are torch's CUDA Philox generator, seeded; they are not
jax.random streams.
"""
import numpy as np
import torch

from .mesh import MeshAttrs, RealMeshField, ParticleField, _r2c, _c2r, _device

__all__ = ['power_law_pk', 'generate_gaussian_mesh', 'lognormal_particles', 'generate_uniform_particles',
           'cutsky_particles']


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


def _radial_profile(rmin, rmax, rmean, rsigma, ndata, solid_angle, ngrid=4096):
    """n(r) = A exp(-(r - rmean)^2 / (2 rsigma^2)) normalised to ndata objects in the shell;
    returns (n(r) as a torch function, (r grid, CDF of r^2 n(r)) for inverse sampling)."""
    r = np.linspace(rmin, rmax, ngrid)
    shape = np.exp(-0.5 * ((r - rmean) / rsigma)**2)
    dens = shape * r**2
    cdf = np.concatenate([[0.], np.cumsum(0.5 * (dens[1:] + dens[:-1]) * np.diff(r))])
    amplitude = ndata / (solid_angle * cdf[-1])

    def nofr(x):
        return amplitude * torch.exp(-0.5 * ((x - rmean) / rsigma)**2)

    return nofr, (r, cdf / cdf[-1])


def cutsky_particles(ndata=2e6, nrandoms=2e7, rmin=1000., rmax=2000., half_angle=60., rmean=1500., rsigma=250.,
                     power=None, fkp_p0=1e4, gen_meshsize=256, seed=42):
    """Cut-sky data and randoms seen from the origin (float32 device tensors).

    Randoms: exactly ``nrandoms`` points, cos(theta) uniform in [cos(half_angle), 1],
    phi uniform, r drawn from r^2 n(r) on [rmin, rmax].  Data: Poisson counts with mean
    n(r_c) V_cell (1 + delta_LN) in the cells of a ``gen_meshsize`` lognormal field over the
    survey's bounding cube, positions uniform in each cell, then cut to the shell and cap
    (about ``ndata`` objects).  Returns (data, randoms, data_weights, randoms_weights) with
    FKP weights 1 / (1 + n(r) fkp_p0).
    """
    dev = _device()
    power = power or power_law_pk()
    cosmin = float(np.cos(np.radians(half_angle)))
    solid = 2. * np.pi * (1. - cosmin)
    nofr, (rgrid, cdf) = _radial_profile(rmin, rmax, rmean, rsigma, float(ndata), solid)
    g = _generator(seed)

    def sample_r(u):
        return torch.as_tensor(np.interp(u.cpu().numpy(), cdf, rgrid), dtype=torch.float32, device=dev)

    def to_cartesian(r, mu, phi):
        st = torch.sqrt(torch.clamp(1. - mu * mu, min=0.))
        return torch.stack([r * st * torch.cos(phi), r * st * torch.sin(phi), r * mu], dim=1).to(torch.float32)

    nr = int(nrandoms)
    u = torch.rand((nr, 3), generator=g, device=dev, dtype=torch.float64)
    randoms = to_cartesian(sample_r(u[:, 0]).double(), cosmin + (1. - cosmin) * u[:, 1], 2. * np.pi * u[:, 2])
    # lognormal field over the bounding cube of the survey
    smax = rmax * np.sin(np.radians(half_angle)) if half_angle < 90. else rmax
    lo = np.array([-smax, -smax, min(rmin * cosmin, rmax * cosmin)])
    hi = np.array([smax, smax, rmax])
    box = float((hi - lo).max())
    center = 0.5 * (lo + hi)
    attrs = MeshAttrs(meshsize=gen_meshsize, boxsize=box, boxcenter=center)
    delta = generate_gaussian_mesh(attrs, power, seed=seed + 1).value
    sigma2 = float(delta.double().pow(2).mean())
    lam = torch.exp(delta - 0.5 * sigma2)
    del delta
    cell = float(box / gen_meshsize)
    idx = torch.arange(gen_meshsize, device=dev, dtype=torch.float32)
    cx = (idx + 0.5) * cell + float(center[0] - box / 2)
    cy = (idx + 0.5) * cell + float(center[1] - box / 2)
    cz = (idx + 0.5) * cell + float(center[2] - box / 2)
    rc = torch.sqrt(cx[:, None, None]**2 + cy[None, :, None]**2 + cz[None, None, :]**2)
    lam.mul_(nofr(rc) * cell**3)
    del rc
    counts = torch.poisson(lam, generator=_generator(seed + 2)).to(torch.int64).reshape(-1)
    del lam
    cells = torch.repeat_interleave(torch.arange(counts.numel(), device=dev), counts)
    del counts
    n = gen_meshsize
    ijk = torch.stack([cells // (n * n), (cells // n) % n, cells % n], dim=1).to(torch.float32)
    del cells
    ud = torch.rand(ijk.shape, generator=g, device=dev, dtype=torch.float32)
    origin = torch.as_tensor(center - box / 2., dtype=torch.float32, device=dev)
    data = (ijk + ud) * cell + origin
    del ijk, ud
    r = torch.linalg.norm(data.double(), dim=1)
    keep = (r >= rmin) & (r <= rmax) & (data[:, 2].double() >= cosmin * r)
    data = data[keep].contiguous()
    wd = (1. / (1. + nofr(torch.linalg.norm(data.double(), dim=1)) * fkp_p0)).to(torch.float32)
    wr = (1. / (1. + nofr(torch.linalg.norm(randoms.double(), dim=1)) * fkp_p0)).to(torch.float32)
    return data, randoms.contiguous(), wd, wr
