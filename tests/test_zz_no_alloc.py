"""The allocation-free binning entry point against the workspace one.

``pk_bin_global_noalloc`` exists for callers that cannot allocate device memory when
they call into the library (a host callback, a foreign runtime that owns the
allocator): it takes its scratch from a fixed static device array instead of a caller
workspace.  Both entry points launch the same deterministic kernels with the same grid,
so it must give bit-identical multipoles to ``pk_bin_global`` on the same inputs, on two
calls in a row (the second call reuses the array the first one left behind).

This file is collected last on purpose, so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _call_both(delta, attrs, bins, ells, los):
    from jaxpower_b200 import _lib
    lib = _lib.load()
    nbins = bins.nbins
    stream = _lib.stream_handle()
    args = (_lib.ptr(delta), None, _lib.i32(attrs.meshsize), _lib.f32(attrs.kfun), _lib.f32(los),
            _lib.ptr(bins.d_edges), len(bins._edges1d), bins._step, attrs.backend_code, len(ells),
            _lib.i32(ells))
    ref = torch.empty(len(ells) * nbins, dtype=torch.float64, device='cuda')
    ws = bins._workspace()
    _lib.call('pk_bin_global', stream, *args, _lib.ptr(ref), _lib.ptr(ws), ws.numel())
    outs = []
    for _ in range(2):
        out = torch.full((len(ells) * nbins,), np.nan, dtype=torch.float64, device='cuda')
        _lib.call('pk_bin_global_noalloc', stream, *args, _lib.ptr(out))
        outs.append(out.cpu().numpy())
    torch.cuda.synchronize()
    return ref.cpu().numpy(), outs


@pytest.mark.parametrize('meshsize,step', [(64, 0.01), ((48, 40, 36), 0.02)])
def test_noalloc_matches_workspace_entry_point(meshsize, step):
    import jaxpower_b200 as jp
    rng = np.random.default_rng(5)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=1000.)
    shape = tuple(attrs.meshsize[:2]) + (int(attrs.meshsize[2]) // 2 + 1,)
    delta = torch.as_tensor((rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype('c8')).cuda()
    ells = (0, 2, 4)
    bins = jp.BinMesh2SpectrumPoles(attrs, edges={'step': step}, ells=ells)
    ref, outs = _call_both(delta, attrs, bins, ells, (0., 0., 1.))
    for out in outs:
        assert np.all(np.isfinite(out))
        assert np.array_equal(out, ref)


def test_noalloc_rejects_oversized_request():
    import jaxpower_b200 as jp
    from jaxpower_b200 import _lib
    attrs = jp.MeshAttrs(meshsize=256, boxsize=1000.)
    edges = torch.linspace(0., 0.8, 4001, device='cuda', dtype=torch.float32)
    delta = torch.zeros((256, 256, 129), dtype=torch.complex64, device='cuda')
    out = torch.empty(9 * 4000, dtype=torch.float64, device='cuda')
    ells = list(range(9))
    status = _lib.load().pk_bin_global_noalloc(_lib.stream_handle(), _lib.ptr(delta), None,
                                               _lib.i32(attrs.meshsize), _lib.f32(attrs.kfun),
                                               _lib.f32((0., 0., 1.)), _lib.ptr(edges), 4001, 0.0002,
                                               0, 9, _lib.i32(ells), _lib.ptr(out))
    assert status != 0
    assert b'scratch' in _lib.load().pk_last_error() or b'bins' in _lib.load().pk_last_error()
