"""Paint / read parity: the CUDA path (through the C ABI) against the CPU oracle.

The oracle restates ``resamplers.py:57-125`` and ``mesh.py:2673-2754`` in the
reference's float32 operation order.  Cell assignment must be bit-exact; mesh
values agree to float32 rounding of the (order-dependent) cell sums.
"""
import numpy as np
import pytest
import torch

from oracle.coords import Geometry
from oracle import paint as opaint

pytestmark = pytest.mark.gpu

RESAMPLERS = {'ngp': 1, 'cic': 2, 'tsc': 3, 'pcs': 4}


def _jp():
    import jaxpower_b200 as jp
    return jp


def _catalog(n, boxsize, boxcenter, seed=0):
    rng = np.random.default_rng(seed)
    pos = (rng.uniform(-0.5, 0.5, (n, 3)) * np.asarray(boxsize) + np.asarray(boxcenter)).astype('f4')
    w = rng.uniform(0.5, 1.5, n).astype('f4')
    return pos, w


@pytest.mark.parametrize('meshsize', [(16, 16, 16), (17, 12, 10), (4, 4, 4), (32, 40, 36), (12, 20, 68)])
@pytest.mark.parametrize('resampler', list(RESAMPLERS))
def test_paint_shifts_match_oracle(meshsize, resampler):
    jp = _jp()
    from jaxpower_b200.mesh import _paint_shifts
    boxsize, boxcenter = np.array([100., 120., 90.]), np.array([3., -5., 10.])
    pos, w = _catalog(5000, 1.2 * boxsize, boxcenter, seed=1)  # some particles outside: periodic wrap
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=boxcenter)
    order = RESAMPLERS[resampler]
    interlacing = 3
    meshes, status = _paint_shifts(attrs, torch.as_tensor(pos).cuda(), torch.as_tensor(w).cuda(), order, interlacing)
    assert int(status.item()) == 0
    geom = Geometry(meshsize, boxsize, boxcenter)
    u = opaint.normalize_positions(geom, pos)
    for s, shift in enumerate(opaint.interlacing_shifts(interlacing, np.float32)):
        us = (u + shift).astype('f4')
        got = meshes[s].cpu().numpy()
        # the GPU sums the reference's float32 contributions in 64-bit fixed point (resolution
        # n max|w| 2^-62 per contribution) and rounds once: equal to the float64-accumulated
        # oracle up to one float32 ulp plus that resolution
        exact = opaint.paint_mesh(geom.rshape, us, w, order, accum='f64')
        fixed = 5000 * 1.5 * 2.**-62 * 64
        assert np.all(np.abs(got - exact) <= np.spacing(np.abs(exact)) + fixed), s
        # and to the reference's serial float32 order within its accumulated rounding
        serial = opaint.paint_mesh(geom.rshape, us, w, order)
        percell = 5000. * order**3 / np.prod(meshsize)
        scale = np.abs(serial).max()
        assert np.allclose(got, serial, rtol=0, atol=2e-7 * max(1., np.sqrt(percell)) * scale), s
        assert np.isclose(got.sum(dtype='f8'), w.sum(dtype='f8'), rtol=1e-6)


@pytest.mark.parametrize('resampler', list(RESAMPLERS))
def test_cell_assignment_bit_exact(resampler):
    """Dyadic positions on cell edges, half-cell ties (round half to even), box edges and
    outside the box, small-integer weights: the mesh must be bit-identical to the oracle's
    (float32 contributions summed exactly, rounded once), which needs every particle in
    exactly the reference's cells."""
    jp = _jp()
    from jaxpower_b200.mesh import _paint_shifts
    n = 16
    boxsize, boxcenter = 32., 0.  # cellsize 2
    ticks = np.arange(-40, 40) * 0.5  # multiples of a quarter cell, beyond the box on both sides
    rng = np.random.default_rng(3)
    pos = rng.choice(ticks, size=(4000, 3)).astype('f4')
    pos[:8] = [[-16., -16., -16.], [16., 16., 16.], [15., -15., 1.], [-1., 1., 3.],
               [0., 0., 0.], [31., -31., 15.5], [-16.5, 16.5, 0.5], [1.5, 2.5, 3.5]]
    w = rng.integers(1, 4, size=4000).astype('f4')
    attrs = jp.MeshAttrs(meshsize=n, boxsize=boxsize, boxcenter=boxcenter)
    order = RESAMPLERS[resampler]
    meshes, _ = _paint_shifts(attrs, torch.as_tensor(pos).cuda(), torch.as_tensor(w).cuda(), order, 2)
    geom = Geometry(n, boxsize, boxcenter)
    u = opaint.normalize_positions(geom, pos)
    for s, shift in enumerate(opaint.interlacing_shifts(2, np.float32)):
        ref = opaint.paint_mesh(geom.rshape, (u + shift).astype('f4'), w, order, accum='f64')
        assert np.array_equal(meshes[s].cpu().numpy(), ref), s


@pytest.mark.parametrize('resampler', ['cic', 'tsc', 'pcs'])
@pytest.mark.parametrize('interlacing', [0, 2, 3, 5])
@pytest.mark.parametrize('compensate', [False, True])
@pytest.mark.parametrize('out', ['real', 'complex'])
def test_particle_paint_pipeline(resampler, interlacing, compensate, out):
    jp = _jp()
    meshsize, boxsize, boxcenter = (32, 24, 20), np.array([500., 400., 300.]), np.array([0., 10., 20.])
    pos, w = _catalog(20000, boxsize, boxcenter, seed=2)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=boxcenter)
    mesh = jp.ParticleField(pos, w, attrs=attrs).paint(resampler=resampler, interlacing=interlacing,
                                                       compensate=compensate, out=out)
    geom = Geometry(meshsize, boxsize, boxcenter)
    ref = opaint.paint(geom, pos, w, resampler, interlacing, compensate, out)
    got = mesh.value.cpu().numpy()
    assert got.shape == ref.shape
    scale = np.abs(ref).max()
    assert np.allclose(got, ref, rtol=0, atol=2e-5 * scale), np.abs(got - ref).max() / scale
    if out == 'real':  # mass conservation (tests/test_mesh.py:231)
        assert np.isclose(got.sum(dtype='f8'), w.sum(dtype='f8'), rtol=1e-5)


@pytest.mark.parametrize('backend', ['jax', 'jaxdecomp'])
@pytest.mark.parametrize('out', ['real', 'complex'])
def test_interlacing_long_xy_axes(backend, out):
    """Meshes with n0 + n1 > 512 form the interlacing phases and windows per row instead of
    from per-axis tables; the painted, interlaced, compensated mesh matches the oracle, and the
    fused binning of the shifted meshes matches binning the stored one."""
    jp = _jp()
    meshsize, boxsize = (300, 240, 8), np.array([3000., 2400., 80.])
    pos, w = _catalog(200000, boxsize, [0.] * 3, seed=6)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, fft_backend=backend)
    mesh = jp.ParticleField(pos, w, attrs=attrs).paint(resampler='tsc', interlacing=3, compensate=True, out=out)
    if out == 'complex':
        b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.01, 'max': 0.3}, ells=(0, 2, 4))
        fused = jp.compute_mesh2_spectrum(mesh, bin=b, los='x')
        stored = jp.compute_mesh2_spectrum(jp.ComplexMeshField(mesh.value, attrs=attrs), bin=b, los='x')
        scale = np.abs(stored.get(0).num_raw).max()
        for ell in (0, 2, 4):
            assert np.allclose(fused.get(ell).num_raw, stored.get(ell).num_raw, rtol=0, atol=1e-6 * scale), ell
    if out == 'complex' and backend == 'jaxdecomp':
        return  # the oracle's jaxdecomp complex mesh is the full grid; the real mesh is compared
    geom = Geometry(meshsize, boxsize, 0., backend=backend)
    ref = opaint.paint(geom, pos, w, 'tsc', 3, True, out)
    got = mesh.value.cpu().numpy()
    scale = np.abs(ref).max()
    assert np.allclose(got, ref, rtol=0, atol=2e-5 * scale), np.abs(got - ref).max() / scale


@pytest.mark.parametrize('backend', ['jax', 'jaxdecomp'])
def test_paint_backends_real(backend):
    jp = _jp()
    meshsize, boxsize = 32, 200.
    pos, w = _catalog(30000, [boxsize] * 3, [0.] * 3, seed=5)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, fft_backend=backend)
    mesh = jp.ParticleField(pos, w, attrs=attrs).paint(resampler='tsc', interlacing=3, compensate=True)
    geom = Geometry(meshsize, boxsize, 0., backend=backend)
    ref = opaint.paint(geom, pos, w, 'tsc', 3, True, 'real')
    scale = np.abs(ref).max()
    assert np.allclose(mesh.value.cpu().numpy(), ref, rtol=0, atol=2e-5 * scale)


@pytest.mark.parametrize('resampler', list(RESAMPLERS))
def test_read_matches_oracle(resampler):
    jp = _jp()
    meshsize, boxsize = (16, 20, 12), np.array([50., 60., 40.])
    rng = np.random.default_rng(7)
    value = rng.normal(size=meshsize).astype('f4')
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize)
    mesh = jp.RealMeshField(torch.as_tensor(value).cuda(), attrs=attrs)
    pos, _ = _catalog(3000, 1.1 * boxsize, [0.] * 3, seed=8)
    got = mesh.read(pos, resampler=resampler).cpu().numpy()
    geom = Geometry(meshsize, boxsize, 0.)
    ref = opaint.read_mesh(value, opaint.normalize_positions(geom, pos), RESAMPLERS[resampler])
    assert np.allclose(got, ref, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize('order,interlacing', [(1, 2), (2, 3), (3, 3), (4, 4)])
def test_read_interlaced_equals_per_shift_reads(order, interlacing):
    """pk_read_interlaced gives, bit for bit, the sum of pk_read over the shifted meshes
    (accumulated in shift order), for the read values and the position gradient."""
    from jaxpower_b200 import _lib as L
    meshsize, boxsize, boxcenter = (16, 20, 12), np.array([50., 60., 40.], dtype='f4'), np.array([1., -2., 3.], dtype='f4')
    rng = np.random.default_rng(9)
    meshes = torch.as_tensor(rng.normal(size=(interlacing,) + meshsize).astype('f4')).cuda()
    pos, w = _catalog(5000, 1.1 * boxsize, boxcenter, seed=10)
    pos = torch.as_tensor(pos).cuda().contiguous()
    w = torch.as_tensor(w).cuda().contiguous()
    n = pos.shape[0]
    cellsize = (boxsize / np.asarray(meshsize)).astype('f4')
    geo = (L.i32(meshsize), L.f32(boxsize), L.f32(boxcenter), L.f32(cellsize), order)
    out_a = torch.zeros(n, device='cuda')
    grad_a = torch.zeros((n, 3), device='cuda')
    for s in range(interlacing):
        shift = float(np.float32(s) / np.float32(interlacing))
        L.call('pk_read', L.stream_handle(), L.ptr(meshes[s]), L.ptr(pos), L.ptr(w), n, *geo, shift, 0.5,
               L.ptr(out_a), L.ptr(grad_a), 1)
    out_b = torch.full((n,), 3., device='cuda')
    grad_b = torch.full((n, 3), 3., device='cuda')
    L.call('pk_read_interlaced', L.stream_handle(), L.ptr(meshes), interlacing, L.ptr(pos), L.ptr(w), n, *geo, 0.5,
           L.ptr(out_b), L.ptr(grad_b), 0)
    assert torch.equal(out_a, out_b)
    assert torch.equal(grad_a, grad_b)


# (64, 48, 32): last axis below 64, every configuration takes the all-shifts kernel;
# (40, 36, 100) and (16, 24, 64): configurations 8 to 10 take the per-shift kernel (partial
# tiles along every axis, an axis that is not a multiple of 8, dense tiles)
@pytest.mark.parametrize('meshsize', [(64, 48, 32), (40, 36, 100), (16, 24, 64)])
@pytest.mark.parametrize('resampler', ['ngp', 'cic', 'tsc', 'pcs'])
def test_paint_same_bits_for_every_tile_config(resampler, meshsize):
    """The fixed-point scale depends on the catalog only: all tile configurations (and so the
    autotuner's choice) paint identical meshes."""
    from jaxpower_b200 import _lib as L
    from jaxpower_b200.mesh import _paint_call
    from jaxpower_b200.autotune import NUM_TILE_CONFIGS
    jp = _jp()
    pos, w = _catalog(300000, [500.] * 3, [0.] * 3, seed=12)
    pos[:1000] = pos[0]  # a dense clump (many particles on a few cells)
    pos[1000:1100] = [249.99998, -250., 0.5]  # on the box faces: periodic wrap of the stencil
    w[::7] *= -0.5
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=500.)
    order = RESAMPLERS[resampler]
    pos = torch.as_tensor(pos).cuda()
    w = torch.as_tensor(w).cuda()
    status = torch.zeros(1, dtype=torch.int32, device='cuda')
    outs = []
    assert NUM_TILE_CONFIGS == 11
    for config in range(NUM_TILE_CONFIGS):
        out = torch.empty((3,) + tuple(attrs.meshsize), dtype=torch.float32, device='cuda')
        _paint_call(attrs, pos, w, order, 3, 0, 3, out, status, config)
        outs.append(out)
    for out in outs[1:]:
        assert torch.equal(out, outs[0])
    assert int(status.item()) == 0


def test_paint_deterministic():
    jp = _jp()
    pos, w = _catalog(200000, [1000.] * 3, [0.] * 3, seed=11)
    attrs = jp.MeshAttrs(meshsize=64, boxsize=1000.)
    p = jp.ParticleField(pos, w, attrs=attrs)
    a = p.paint(resampler='tsc', interlacing=3, compensate=True, out='complex').value
    b = p.paint(resampler='tsc', interlacing=3, compensate=True, out='complex').value
    assert torch.equal(a, b)
    # particle order does not change the mesh (fixed-point accumulation)
    perm = np.random.default_rng(0).permutation(len(pos))
    c = jp.ParticleField(pos[perm], w[perm], attrs=attrs).paint(resampler='tsc', interlacing=3, compensate=True,
                                                                out='complex').value
    assert torch.equal(a, c)


def test_paint_empty_and_status():
    jp = _jp()
    attrs = jp.MeshAttrs(meshsize=8, boxsize=10.)
    mesh = jp.ParticleField(np.zeros((0, 3), 'f4'), attrs=attrs).paint(resampler='cic')
    assert float(mesh.value.abs().sum()) == 0.
    pos = np.array([[0., 0., 0.], [np.nan, 0., 0.], [1., 1., 1.]], dtype='f4')
    with pytest.raises(ValueError):
        from jaxpower_b200.mesh import _paint
        _paint(attrs, pos, None, resampler='cic', check=True)


@pytest.mark.parametrize('wscale', [1e-20, 1e-38, 1e30])
def test_paint_tiny_and_huge_weights(wscale):
    """The 64-bit fixed-point scale 2^e (e = 62 - log2 max|w| - log2 n) leaves float32's range
    for tiny weights (e up to 187): it is applied as two exact power-of-two factors, so the
    mesh still equals the float64-accumulated oracle to one ulp (plus the fixed-point step)."""
    jp = _jp()
    from jaxpower_b200.mesh import _paint_shifts
    meshsize, boxsize = 16, 100.
    pos, w = _catalog(3000, boxsize, 0., seed=9)
    w = (w.astype('f8') * wscale).astype('f4')
    assert np.all(np.isfinite(w)) and np.all(w != 0.)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize)
    meshes, status = _paint_shifts(attrs, torch.as_tensor(pos).cuda(), torch.as_tensor(w).cuda(), 3, 1)
    assert int(status.item()) == 0
    got = meshes[0].cpu().numpy()
    assert np.all(np.isfinite(got))
    geom = Geometry(meshsize, boxsize, 0.)
    exact = opaint.paint_mesh(geom.rshape, opaint.normalize_positions(geom, pos), w, 3, accum='f64')
    fixed = 3000 * np.abs(w).max(initial=0.).astype('f8') * 2.**-62 * 64
    tiny = np.finfo(np.float32).smallest_subnormal * 64  # products below the normal range round differently
    assert np.all(np.abs(got - exact) <= np.spacing(np.abs(exact)) + fixed + tiny)
