"""Whole-ell first-point kernels against the general term-list kernels.

The first-point entry points (Y_lm premultiply, binning, its adjoint, the Y_lm
accumulation of the backward pass) have compiled forms for term lists made of whole
ells in canonical order (every m of each ell, ell ascending).  The same terms in any
other order take the general kernels; both must give the same values term for term
(the arithmetic per mode is the same, only FMA contraction of the polynomials may
differ: 1e-6 relative).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

RTOL = 1e-6


def _lib():
    from jaxpower_b200 import _lib
    return _lib


def _terms(ells, reverse):
    terms = [(ell, m) for ell in sorted(ells) if ell > 0 for m in range(-ell, ell + 1)]
    return terms[::-1] if reverse else terms


def _close(a, b, rtol=RTOL):
    a, b = np.asarray(a, dtype='f8'), np.asarray(b, dtype='f8')
    scale = max(np.abs(b).max(), 1e-30)
    return np.abs(a - b).max() <= rtol * scale, np.abs(a - b).max() / scale


def _premultiply(L, rho, meshsize, cellsize, offset, terms):
    out = torch.empty((len(terms),) + tuple(meshsize), dtype=torch.float32, device='cuda')
    L.call('pk_ylm_premultiply', L.stream_handle(), L.ptr(rho), L.i32(meshsize), L.f32(cellsize), L.f32(offset),
           len(terms), L.i32([t[0] for t in terms]), L.i32([t[1] for t in terms]), L.ptr(out))
    return out


CASES = [((32, 24, 20), (0, 2, 4)), ((33, 17, 15), (0, 1, 2, 3, 4)), ((16, 16, 16), (0, 2, 4, 6)),
         ((24, 20, 8), (2,)), ((20, 20, 36), (0, 3))]


@pytest.mark.parametrize('meshsize,ells', CASES)
@pytest.mark.parametrize('cross', [False, True])
def test_firstpoint_blocks_match_general(meshsize, ells, cross):
    import jaxpower_b200 as jp
    L = _lib()
    rng = np.random.default_rng(7)
    boxsize = np.array([400., 350., 300.], dtype='f4')
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=(300., -100., 450.))
    rho = torch.as_tensor(rng.normal(size=meshsize).astype('f4')).cuda()
    rho2 = torch.as_tensor(rng.normal(size=meshsize).astype('f4')).cuda()
    cellsize = attrs.cellsize
    offset = (attrs.boxcenter - (attrs.boxsize / np.float32(2.)).astype('f4')).astype('f4')
    canon, other = _terms(ells, False), _terms(ells, True)
    order = [other.index(t) for t in canon]  # other[order[q]] == canon[q]

    # Y_lm premultiply
    real_c = _premultiply(L, rho, meshsize, cellsize, offset, canon)
    real_o = _premultiply(L, rho, meshsize, cellsize, offset, other)
    ok, err = _close(real_c.cpu().numpy(), real_o[order].cpu().numpy())
    assert ok, ('premultiply', err)

    # binning: the same F in canonical and general order
    A0 = torch.fft.rfftn(rho).contiguous()
    B0 = torch.fft.rfftn(rho2).contiguous() if cross else None
    F_c = torch.fft.rfftn(real_c, dim=(-3, -2, -1)).contiguous()
    F_o = F_c[[canon.index(t) for t in other]].contiguous()
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=ells)
    ws = b._workspace()
    nbins = b.nbins

    def bin_sums(F, terms):
        raw = torch.full((len(ells) * nbins,), 7., dtype=torch.float64, device='cuda')
        L.call('pk_bin_firstpoint', L.stream_handle(), L.ptr(A0), L.ptr(B0), L.ptr(F), len(terms),
               L.i32([t[0] for t in terms]), L.i32([t[1] for t in terms]), L.i32(meshsize), L.f32(attrs.kfun),
               L.ptr(b.d_edges), len(b._edges1d), b._step, attrs.backend_code, len(ells), L.i32(ells), 1, 0,
               L.ptr(raw), L.ptr(ws), ws.numel())
        return raw.cpu().numpy().reshape(len(ells), nbins)

    got, ref = bin_sums(F_c, canon), bin_sums(F_o, other)
    for i, ell in enumerate(ells):
        ok, err = _close(got[i], ref[i], rtol=1e-5)
        assert ok, ('bin', ell, err)

    # adjoint (for_c2r) and the Y_lm accumulation of the backward pass
    wsa = torch.empty(1 << 16, dtype=torch.uint8, device='cuda')
    coef = torch.as_tensor(rng.normal(size=(len(ells), nbins)).astype('f4')).cuda()
    edge0 = float(b._edges1d[0])

    def adjoint(F, terms):
        ga0 = torch.zeros_like(A0)
        gf = torch.empty_like(F)
        L.call('pk_bin_firstpoint_adjoint', L.stream_handle(), L.ptr(A0), L.ptr(F), len(terms),
               L.i32([t[0] for t in terms]), L.i32([t[1] for t in terms]), L.i32(meshsize), L.f32(attrs.kfun),
               L.ptr(b.d_edges), len(b._edges1d), b._step, edge0, attrs.backend_code, len(ells), L.i32(ells),
               L.ptr(coef), 1, L.ptr(ga0), 1, L.ptr(gf), L.ptr(wsa), wsa.numel())
        return ga0, gf

    ga0_c, gf_c = adjoint(F_c, canon)
    ga0_o, gf_o = adjoint(F_o, other)
    ok, err = _close(torch.view_as_real(ga0_c).cpu().numpy(), torch.view_as_real(ga0_o).cpu().numpy(), rtol=1e-5)
    assert ok, ('adjoint A0', err)
    ok, err = _close(torch.view_as_real(gf_c).cpu().numpy(), torch.view_as_real(gf_o[order]).cpu().numpy())
    assert ok, ('adjoint F', err)

    def accumulate(r, terms):
        out = rho2.clone()
        L.call('pk_ylm_accumulate', L.stream_handle(), L.ptr(r), L.i32(meshsize), L.f32(cellsize), L.f32(offset),
               len(terms), L.i32([t[0] for t in terms]), L.i32([t[1] for t in terms]), L.ptr(out))
        return out.cpu().numpy()

    ok, err = _close(accumulate(real_c, canon), accumulate(real_o, other), rtol=1e-5)
    assert ok, ('accumulate', err)
