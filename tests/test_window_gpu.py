"""Window matrices (compute_mesh2_spectrum_window) and mean spectra (compute_mesh2_spectrum_mean)
against the CPU oracle: global, first-point and end-point lines of sight; input power on the mesh
and the 'smooth' / 'infinite' flags; 'firstpoint' and 'local' theory lines of sight; wide-angle
theory orders; periodic boxes and auto / cross selection functions.  Float32 modes and FFTs,
float64 bin sums: 2e-5 of the largest entry."""
import numpy as np
import pytest
import torch

from oracle.coords import Geometry
from oracle.spectrum import Bins, compute_mesh2_spectrum_window as owindow

pytestmark = pytest.mark.gpu

TOL = 2e-5


def _check(got, ref):
    assert got.shape == ref.shape
    fin = np.isfinite(ref)
    assert np.array_equal(fin, np.isfinite(got))
    scale = max(np.abs(ref[fin]).max(), 1e-30)
    err = np.abs(got[fin] - ref[fin]).max() / scale
    assert err <= TOL, err


@pytest.mark.parametrize('meshsize', [(16, 12, 10), (24, 20, 16)])
@pytest.mark.parametrize('los', ['z', [0.6, 0., 0.8]])
@pytest.mark.parametrize('ells', [(0, 2, 4), (0, 1, 2)])
@pytest.mark.parametrize('kind', ['common', 'disjoint', 'overlapping'])
def test_periodic_window_matches_oracle(meshsize, los, ells, kind):
    """Input edges equal to the output bins (diagonal fill), disjoint input bins with gaps and
    a range past the output bins (one pass on the merged edges), overlapping input bins (one
    pass per column)."""
    import jaxpower_b200 as jp
    boxsize = np.array([400., 300., 250.])
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=ells)
    ob = Bins(Geometry(meshsize, boxsize), step=0.02, ells=ells)
    if kind == 'common':
        edgesin = b._edges1d
    elif kind == 'disjoint':
        a = np.arange(0.004, 0.5, 0.013)
        edgesin = np.column_stack([a[:-1], a[:-1] + 0.009])
    else:
        a = np.arange(0., 0.3, 0.013)
        edgesin = np.column_stack([a[:-2], a[2:]])
    w = jp.compute_mesh2_spectrum_window(attrs, edgesin=edgesin, ellsin=(0, 2, 4), bin=b, los=los)
    ref = owindow(ob, edgesin, (0, 2, 4), los=los)
    _check(w.value, ref)
    assert w.observable.ells == tuple(ells) and w.theory.ells == (0, 2, 4)


@pytest.mark.parametrize('meshsize', [(16, 12, 10), (20, 16, 12), (10, 8, 182)])
@pytest.mark.parametrize('los', ['x', [0., 0.6, 0.8]])
@pytest.mark.parametrize('cross', [False, True])
def test_selection_window_matches_oracle(meshsize, los, cross):
    """Short last axes take the flat chunk walk of the fused binning pass, (10, 8, 182) its
    row-run walk."""
    import jaxpower_b200 as jp
    boxsize = np.array([500., 400., 300.])
    rng = np.random.default_rng(3)
    sel = [rng.uniform(0.5, 1.5, meshsize).astype('f4') for _ in range(2)]
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 2, 4))
    ob = Bins(Geometry(meshsize, boxsize), step=0.02, ells=(0, 2, 4))
    edgesin = np.arange(0., 0.25, 0.012)  # 20 input bins: batches of 6 leave a ragged last one
    meshes = [attrs.create(kind='real', fill=torch.as_tensor(s)) for s in (sel if cross else sel[:1])]
    ells = (0, 1, 2, 4) if cross else (0, 2, 4)
    if cross:
        b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=ells)
        ob = Bins(Geometry(meshsize, boxsize), step=0.02, ells=ells)
    w = jp.compute_mesh2_spectrum_window(*meshes, edgesin=edgesin, ellsin=(0, 2), bin=b, los=los, batch_size=6)
    ref = owindow(ob, edgesin, (0, 2), los=los, meshes=(sel if cross else sel[:1]))
    _check(w.value, ref)


def test_window_norm_and_io(tmp_path):
    import jaxpower_b200 as jp
    attrs = jp.MeshAttrs(meshsize=(16, 16, 16), boxsize=400.)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 2))
    w1 = jp.compute_mesh2_spectrum_window(attrs, edgesin=b._edges1d, ellsin=(0, 2), bin=b)
    w2 = jp.compute_mesh2_spectrum_window(attrs, edgesin=b._edges1d, ellsin=(0, 2), bin=b, norm=2. * 64.)
    default = np.float32(16 ** 3) / np.float32((400. / 16) ** 3)
    fin = np.isfinite(w1.value)
    assert np.allclose(w2.value[fin], w1.value[fin] * default / np.float32(128.), rtol=1e-6)
    assert np.allclose(w2.observable.get(0).norm, 128.)
    # input edges and multipoles taken from a multipole container (mesh2.py:996-998)
    w3 = jp.compute_mesh2_spectrum_window(attrs, edgesin=w1.observable, bin=b)
    assert w3.theory.ells == (0, 2) and np.array_equal(w3.value, w1.value, equal_nan=True)
    fn = tmp_path / 'window.npz'
    w1.write(str(fn))
    back = jp.read(str(fn))
    assert np.array_equal(back.value, w1.value, equal_nan=True)
    assert back.observable.ells == (0, 2) and back.theory.ells == (0, 2)
    assert np.array_equal(back.theory.get(0).k_edges, w1.theory.get(0).k_edges)


def _pk0(k):
    return 1e4 * (k + 0.02) ** -1.5


def _pk2(k):
    return 3e3 * (k + 0.03) ** -1.2


@pytest.mark.parametrize('los', ['z', [0.6, 0., 0.8]])
@pytest.mark.parametrize('selection', [None, 'auto', 'cross'])
@pytest.mark.parametrize('meshsize', [(16, 12, 10), (10, 8, 182)])
def test_mean_spectrum_matches_oracle(los, selection, meshsize):
    """compute_mesh2_spectrum_mean with theory multipoles (callables of |k|): periodic box and
    selection functions; k = 0 kept, odd ell 0."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_spectrum_mean as omean
    boxsize = np.array([500., 400., 300.])
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize)
    ells = (0, 1, 2, 4)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=ells)
    ob = Bins(Geometry(meshsize, boxsize), step=0.02, ells=ells)
    rng = np.random.default_rng(5)
    sel = [rng.uniform(0.5, 1.5, meshsize).astype('f4') for _ in range(2)]
    theory = {0: _pk0, 2: _pk2}
    if selection is None:
        got = jp.compute_mesh2_spectrum_mean(attrs, theory=theory, bin=b, los=los)
        ref = omean(ob, theory, los=los)
    else:
        use = sel if selection == 'cross' else sel[:1]
        meshes = [attrs.create(kind='real', fill=torch.as_tensor(s)) for s in use]
        got = jp.compute_mesh2_spectrum_mean(*meshes, theory=theory, bin=b, los=los)
        ref = omean(ob, theory, los=los, meshes=use)
    num = np.array([p.num_raw for p in got])
    _check(num, ref['num_raw'])
    assert np.allclose(got.get(0).norm, ref['norm'], rtol=1e-6)
    assert np.all(got.get(1).num_raw == 0.)


def test_mean_spectrum_theory_forms():
    """A callable of the k vector, array poles on input edges, and the periodic identity
    mean(P = const) = const."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_spectrum_mean as omean
    meshsize, boxsize = (16, 16, 16), np.array([400., 400., 400.])
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 2))
    ob = Bins(Geometry(meshsize, boxsize), step=0.02, ells=(0, 2))

    def pkvec(kvec):
        k2 = kvec[0] ** 2 + kvec[1] ** 2 + kvec[2] ** 2
        return 5e3 / (1. + 100. * k2) * (1. + 0.5 * kvec[2] ** 2 / (k2 + 1e-6))

    got = jp.compute_mesh2_spectrum_mean(attrs, theory=pkvec, bin=b, los='z')
    ref = omean(ob, pkvec, los='z')
    _check(np.array([p.num_raw for p in got]), ref['num_raw'])
    # array poles on edges: a constant monopole over the whole k range gives value() = 1
    kin = np.array([0., 1.])
    const = jp.compute_mesh2_spectrum_mean(attrs, theory=(kin, {0: np.array([1.])}), bin=b, los='z')
    v = const.get(0).value()
    assert np.allclose(v[np.isfinite(v)], 1., rtol=1e-6)
    # a multipole container as the theory: its values read per mode from its k bins
    poles = jp.Mesh2SpectrumPoles([jp.Mesh2SpectrumPole(k=b.xavg, k_edges=b.edges, nmodes=b.nmodes,
                                                        num_raw=np.full(b.nbins, 2.), ell=ell) for ell in (0, 2)])
    both = jp.compute_mesh2_spectrum_mean(attrs, theory=poles, bin=b, los='z')
    v = both.get(0).value()
    assert np.allclose(v[np.isfinite(v)][1:], 2., rtol=1e-5)


@pytest.mark.parametrize('selection', [None, 'auto', 'cross'])
@pytest.mark.parametrize('los', ['firstpoint', 'endpoint'])
def test_firstpoint_mean_spectrum_matches_oracle(selection, los):
    """First-point / end-point mean spectrum (theory multipoles 0 and 2) against the oracle."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_spectrum_mean_firstpoint as omean_fp
    meshsize, boxsize = (16, 12, 10), np.array([500., 400., 300.])
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=(900., -200., 300.))
    ells = (0, 1, 2)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=ells)
    ob = Bins(Geometry(meshsize, boxsize, (900., -200., 300.)), step=0.02, ells=ells)
    rng = np.random.default_rng(9)
    sel = [rng.uniform(0.5, 1.5, meshsize).astype('f4') for _ in range(2)]
    theory = {0: _pk0, 2: _pk2}
    if selection is None:
        got = jp.compute_mesh2_spectrum_mean(attrs, theory=theory, bin=b, los=los)
        ref = omean_fp(ob, theory, swap=los == 'endpoint')
    else:
        use = sel if selection == 'cross' else sel[:1]
        meshes = [attrs.create(kind='real', fill=torch.as_tensor(s)) for s in use]
        got = jp.compute_mesh2_spectrum_mean(*meshes, theory=theory, bin=b, los=los)
        ref = omean_fp(ob, theory, meshes=use, swap=los == 'endpoint')
    _check(np.array([p.num_raw for p in got]), ref)
    if selection is None and los == 'firstpoint':
        tagged = jp.compute_mesh2_spectrum_mean(attrs, theory=(theory, 'firstpoint'), bin=b, los=los)
        assert np.array_equal(np.array([p.num_raw for p in tagged]), np.array([p.num_raw for p in got]))
        with pytest.raises(NotImplementedError):
            jp.compute_mesh2_spectrum_mean(attrs, theory=(theory, 'other'), bin=b, los=los)


@pytest.mark.parametrize('selection', [None, 'auto', 'cross'])
def test_local_theory_mean_spectrum_matches_oracle(selection):
    """Mean spectrum with the 'local' theory line of sight (theory multipoles 0, 2, 4)."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_spectrum_mean_firstpoint as omean_fp
    meshsize, boxsize, center = (12, 10, 8), np.array([500., 400., 300.]), (900., -200., 300.)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=center)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 2))
    ob = Bins(Geometry(meshsize, boxsize, center), step=0.02, ells=(0, 2))
    rng = np.random.default_rng(11)
    sel = [rng.uniform(0.5, 1.5, meshsize).astype('f4') for _ in range(2)]
    theory = {0: _pk0, 2: _pk2, 4: lambda k: 1e3 * (k + 0.05) ** -1.}
    if selection is None:
        got = jp.compute_mesh2_spectrum_mean(attrs, theory=(theory, 'local'), bin=b, los='firstpoint')
        ref = omean_fp(ob, theory, theory_los='local')
    else:
        use = sel if selection == 'cross' else sel[:1]
        meshes = [attrs.create(kind='real', fill=torch.as_tensor(s)) for s in use]
        got = jp.compute_mesh2_spectrum_mean(*meshes, theory=(theory, 'local'), bin=b, los='firstpoint')
        ref = omean_fp(ob, theory, meshes=use, theory_los='local')
    _check(np.array([p.num_raw for p in got]), ref)


@pytest.mark.parametrize('selection', [None, 'auto', 'cross'])
@pytest.mark.parametrize('los', ['firstpoint', 'endpoint'])
def test_firstpoint_window_matches_oracle(selection, los):
    """First-point / end-point window matrix (input power on the mesh) against the oracle."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_spectrum_window_firstpoint as owin_fp
    meshsize, boxsize, center = (12, 10, 8), np.array([500., 400., 300.]), (900., -200., 300.)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=center)
    ells = (0, 2) if selection != 'cross' else (1, 2)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=ells)
    ob = Bins(Geometry(meshsize, boxsize, center), step=0.02, ells=ells)
    rng = np.random.default_rng(13)
    sel = [rng.uniform(0.5, 1.5, meshsize).astype('f4') for _ in range(2)]
    edgesin = np.arange(0., 0.06, 0.015)
    if selection is None:
        w = jp.compute_mesh2_spectrum_window(attrs, edgesin=edgesin, ellsin=((0, 2), 'firstpoint'), bin=b, los=los)
        ref = owin_fp(ob, edgesin, (0, 2), swap=los == 'endpoint')
    else:
        use = sel if selection == 'cross' else sel[:1]
        meshes = [attrs.create(kind='real', fill=torch.as_tensor(s)) for s in use]
        w = jp.compute_mesh2_spectrum_window(*meshes, edgesin=edgesin, ellsin=(0, 2), bin=b, los=los)
        ref = owin_fp(ob, edgesin, (0, 2), meshes=use, swap=los == 'endpoint')
    _check(w.value, ref)
    assert w.theory.ells == (0, 2)


@pytest.mark.parametrize('selection', [None, 'cross'])
def test_local_theory_window_matches_oracle(selection):
    """Window matrix with the 'local' theory line of sight against the oracle."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_spectrum_window_firstpoint as owin_fp
    meshsize, boxsize, center = (10, 8, 8), np.array([500., 400., 400.]), (900., -200., 300.)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=center)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 2))
    ob = Bins(Geometry(meshsize, boxsize, center), step=0.02, ells=(0, 2))
    rng = np.random.default_rng(17)
    sel = [rng.uniform(0.5, 1.5, meshsize).astype('f4') for _ in range(2)]
    edgesin = np.arange(0., 0.05, 0.02)
    if selection is None:
        w = jp.compute_mesh2_spectrum_window(attrs, edgesin=edgesin, ellsin=((0, 2, 4), 'local'), bin=b,
                                             los='firstpoint')
        ref = owin_fp(ob, edgesin, (0, 2, 4), theory_los='local')
    else:
        meshes = [attrs.create(kind='real', fill=torch.as_tensor(s)) for s in sel]
        w = jp.compute_mesh2_spectrum_window(*meshes, edgesin=edgesin, ellsin=((0, 2, 4), 'local'), bin=b,
                                             los='firstpoint')
        ref = owin_fp(ob, edgesin, (0, 2, 4), meshes=sel, theory_los='local')
    _check(w.value, ref)


@pytest.mark.parametrize('selection', [None, 'auto'])
@pytest.mark.parametrize('los', ['z', [0.6, 0., 0.8]])
def test_smooth_window_matches_oracle(selection, los):
    """'smooth' window (global line of sight): correlation-space Legendre products binned on the
    GPU, Bessel transforms on the host, against the oracle (direct products, adaptive
    quadrature)."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_spectrum_window_smooth as owin_smooth
    meshsize, boxsize = (12, 10, 8), np.array([500., 400., 300.])
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 2, 4))
    ob = Bins(Geometry(meshsize, boxsize), step=0.02, ells=(0, 2, 4))
    sedges = jp.BinMesh2CorrelationPoles(attrs)._edges1d
    rng = np.random.default_rng(19)
    sel = rng.uniform(0.5, 1.5, meshsize).astype('f4')
    edgesin = np.arange(0., 0.08, 0.02)
    if selection is None:
        w = jp.compute_mesh2_spectrum_window(attrs, edgesin=edgesin, ellsin=(0, 2), bin=b, los=los, flags=('smooth',))
        ref = owin_smooth(ob, sedges, edgesin, (0, 2), los=los)
    else:
        mesh = attrs.create(kind='real', fill=torch.as_tensor(sel))
        w = jp.compute_mesh2_spectrum_window(mesh, edgesin=edgesin, ellsin=(0, 2), bin=b, los=los, flags=('smooth',))
        ref = owin_smooth(ob, sedges, edgesin, (0, 2), los=los, meshes=[sel])
    _check(w.value, ref)


@pytest.mark.parametrize('selection', [None, 'auto'])
def test_infinite_window_matches_oracle(selection):
    """'infinite' window (global line of sight): tophat theory correlation function on the
    separation grid, batched R2C and the fused linear binning pass, against the oracle."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_spectrum_window_infinite as owin_inf
    meshsize, boxsize = (12, 10, 8), np.array([500., 400., 300.])
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 1, 2))
    ob = Bins(Geometry(meshsize, boxsize), step=0.02, ells=(0, 1, 2))
    rng = np.random.default_rng(23)
    sel = rng.uniform(0.5, 1.5, meshsize).astype('f4')
    edgesin = np.arange(0.01, 0.08, 0.02)
    if selection is None:
        w = jp.compute_mesh2_spectrum_window(attrs, edgesin=edgesin, ellsin=(0, 2), bin=b, los='y',
                                             flags=('infinite',), batch_size=2)
        ref = owin_inf(ob, edgesin, (0, 2), los='y')
    else:
        mesh = attrs.create(kind='real', fill=torch.as_tensor(sel))
        w = jp.compute_mesh2_spectrum_window(mesh, edgesin=edgesin, ellsin=(0, 2), bin=b, los='y',
                                             flags=('infinite',), batch_size=2)
        ref = owin_inf(ob, edgesin, (0, 2), los='y', meshes=[sel])
    _check(w.value, ref)


@pytest.mark.parametrize('selection', [None, 'cross'])
@pytest.mark.parametrize('los', ['firstpoint', 'endpoint'])
def test_firstpoint_smooth_window_matches_oracle(selection, los):
    """'smooth' window with the first-point / end-point line of sight against the oracle."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_spectrum_window_firstpoint_smooth as owin
    meshsize, boxsize, center = (10, 8, 8), np.array([500., 400., 400.]), (900., -200., 300.)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=center)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 2))
    ob = Bins(Geometry(meshsize, boxsize, center), step=0.02, ells=(0, 2))
    sedges = jp.BinMesh2CorrelationPoles(attrs)._edges1d
    rng = np.random.default_rng(29)
    sel = [rng.uniform(0.5, 1.5, meshsize).astype('f4') for _ in range(2)]
    edgesin = np.arange(0.005, 0.06, 0.02)
    if selection is None:
        w = jp.compute_mesh2_spectrum_window(attrs, edgesin=edgesin, ellsin=((0, 2), 'firstpoint'), bin=b, los=los,
                                             flags=('smooth',))
        ref = owin(ob, sedges, edgesin, (0, 2), swap=los == 'endpoint')
    else:
        meshes = [attrs.create(kind='real', fill=torch.as_tensor(s)) for s in sel]
        w = jp.compute_mesh2_spectrum_window(*meshes, edgesin=edgesin, ellsin=(0, 2), bin=b, los=los,
                                             flags=('smooth',))
        ref = owin(ob, sedges, edgesin, (0, 2), meshes=sel, swap=los == 'endpoint')
    _check(w.value, ref)


@pytest.mark.parametrize('selection', [None, 'cross'])
def test_firstpoint_infinite_window_matches_oracle(selection):
    """'infinite' window with the first-point line of sight against the oracle."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_spectrum_window_firstpoint_infinite as owin
    meshsize, boxsize, center = (10, 8, 8), np.array([500., 400., 400.]), (900., -200., 300.)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=center)
    ells = (0, 2) if selection is None else (1, 2)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=ells)
    ob = Bins(Geometry(meshsize, boxsize, center), step=0.02, ells=ells)
    rng = np.random.default_rng(31)
    sel = [rng.uniform(0.5, 1.5, meshsize).astype('f4') for _ in range(2)]
    edgesin = np.arange(0.005, 0.06, 0.02)
    if selection is None:
        w = jp.compute_mesh2_spectrum_window(attrs, edgesin=edgesin, ellsin=(0, 2), bin=b, los='firstpoint',
                                             flags=('infinite',))
        ref = owin(ob, edgesin, (0, 2))
    else:
        meshes = [attrs.create(kind='real', fill=torch.as_tensor(s)) for s in sel]
        w = jp.compute_mesh2_spectrum_window(*meshes, edgesin=edgesin, ellsin=(0, 2), bin=b, los='endpoint',
                                             flags=('infinite',))
        ref = owin(ob, edgesin, (0, 2), meshes=sel, swap=True)
    _check(w.value, ref)


@pytest.mark.parametrize('selection', [None, 'cross'])
def test_local_smooth_window_matches_oracle(selection):
    """'smooth' window with the 'local' theory line of sight against the oracle (direct sums,
    its own real Gaunt coefficients)."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_spectrum_window_local_smooth as owin
    meshsize, boxsize, center = (8, 8, 6), np.array([500., 400., 400.]), (900., -200., 300.)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=center)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 2))
    ob = Bins(Geometry(meshsize, boxsize, center), step=0.02, ells=(0, 2))
    sedges = jp.BinMesh2CorrelationPoles(attrs)._edges1d
    rng = np.random.default_rng(37)
    sel = [rng.uniform(0.5, 1.5, meshsize).astype('f4') for _ in range(2)]
    edgesin = np.arange(0.005, 0.05, 0.02)
    if selection is None:
        w = jp.compute_mesh2_spectrum_window(attrs, edgesin=edgesin, ellsin=((0, 2, 4), 'local'), bin=b,
                                             los='firstpoint', flags=('smooth',))
        ref = owin(ob, sedges, edgesin, (0, 2, 4))
    else:
        meshes = [attrs.create(kind='real', fill=torch.as_tensor(s)) for s in sel]
        w = jp.compute_mesh2_spectrum_window(*meshes, edgesin=edgesin, ellsin=((0, 2, 4), 'local'), bin=b,
                                             los='firstpoint', flags=('smooth',))
        ref = owin(ob, sedges, edgesin, (0, 2, 4), meshes=sel)
    _check(w.value, ref)


@pytest.mark.parametrize('selection', [None, 'cross'])
def test_local_infinite_window_matches_oracle(selection):
    """'infinite' window with the 'local' theory line of sight against the oracle."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_spectrum_window_local_infinite as owin
    meshsize, boxsize, center = (8, 8, 6), np.array([500., 400., 400.]), (900., -200., 300.)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=center)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 2))
    ob = Bins(Geometry(meshsize, boxsize, center), step=0.02, ells=(0, 2))
    rng = np.random.default_rng(41)
    sel = [rng.uniform(0.5, 1.5, meshsize).astype('f4') for _ in range(2)]
    edgesin = np.arange(0.005, 0.05, 0.02)
    if selection is None:
        w = jp.compute_mesh2_spectrum_window(attrs, edgesin=edgesin, ellsin=((0, 2, 4), 'local'), bin=b,
                                             los='firstpoint', flags=('infinite',))
        ref = owin(ob, edgesin, (0, 2, 4))
    else:
        meshes = [attrs.create(kind='real', fill=torch.as_tensor(s)) for s in sel]
        w = jp.compute_mesh2_spectrum_window(*meshes, edgesin=edgesin, ellsin=((0, 2, 4), 'local'), bin=b,
                                             los='firstpoint', flags=('infinite',))
        ref = owin(ob, edgesin, (0, 2, 4), meshes=sel)
    _check(w.value, ref)


@pytest.mark.parametrize('selection', [None, 'auto'])
def test_wide_angle_mean_spectrum_matches_oracle(selection):
    """First-point mean spectrum with a wide-angle order 1 theory term ((ell, 1) keys):
    xi |s|, W1 |x|^-1 (mesh2.py:1641-1645)."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_spectrum_mean_firstpoint as omean_fp
    meshsize, boxsize, center = (12, 10, 8), np.array([500., 400., 300.]), (900., -200., 300.)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=center)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 1, 2))
    ob = Bins(Geometry(meshsize, boxsize, center), step=0.02, ells=(0, 1, 2))
    rng = np.random.default_rng(43)
    sel = rng.uniform(0.5, 1.5, meshsize).astype('f4')
    theory = {(0, 0): _pk0, (2, 0): _pk2, (1, 1): lambda k: 50. * (k + 0.05) ** -1.}
    if selection is None:
        got = jp.compute_mesh2_spectrum_mean(attrs, theory=theory, bin=b, los='firstpoint')
        ref = omean_fp(ob, theory)
    else:
        got = jp.compute_mesh2_spectrum_mean(attrs.create(kind='real', fill=torch.as_tensor(sel)), theory=theory, bin=b,
                                             los='firstpoint')
        ref = omean_fp(ob, theory, meshes=[sel])
    _check(np.array([p.num_raw for p in got]), ref)


@pytest.mark.parametrize('flag', [None, 'smooth', 'infinite'])
@pytest.mark.parametrize('los', ['firstpoint', 'endpoint'])
def test_firstpoint_window_wide_angle_matches_oracle(flag, los):
    """First-point window matrices with wide-angle theory orders (ell_in, wa): the selection
    mesh times |x|^-wa and the real-space products times |s|^wa (mesh2.py:1214, 1249, 1273)."""
    import jaxpower_b200 as jp
    from oracle import spectrum as ospec
    meshsize, boxsize, center = (10, 8, 8), np.array([500., 400., 400.]), (900., -200., 300.)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=center)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 2))
    ob = Bins(Geometry(meshsize, boxsize, center), step=0.02, ells=(0, 2))
    sel = np.random.default_rng(37).uniform(0.5, 1.5, meshsize).astype('f4')
    mesh = attrs.create(kind='real', fill=torch.as_tensor(sel))
    ellsin = [(0, 0), (0, 1), (2, 1), (1, 2)]
    edgesin = np.arange(0.005, 0.06, 0.02)
    w = jp.compute_mesh2_spectrum_window(mesh, edgesin=edgesin, ellsin=(ellsin, 'firstpoint'), bin=b, los=los,
                                         flags=(flag,) if flag else ())
    swap = los == 'endpoint'
    if flag is None:
        ref = ospec.compute_mesh2_spectrum_window_firstpoint(ob, edgesin, ellsin, meshes=[sel], swap=swap)
    elif flag == 'smooth':
        sedges = jp.BinMesh2CorrelationPoles(attrs)._edges1d
        ref = ospec.compute_mesh2_spectrum_window_firstpoint_smooth(ob, sedges, edgesin, ellsin, meshes=[sel],
                                                                    swap=swap)
    else:
        ref = ospec.compute_mesh2_spectrum_window_firstpoint_infinite(ob, edgesin, ellsin, meshes=[sel], swap=swap)
    _check(w.value, ref)
    assert w.theory.ells == (0, 0, 2, 1) and w.theory.wa_orders == (0, 1, 1, 2)
    assert w.theory.get(0, wa_orders=1) is w.theory.poles[1]
    # the wide-angle columns differ from the order-0 ones (the |x|^-wa |s|^wa factors act)
    n = len(edgesin)
    assert not np.allclose(w.value[:, :n], w.value[:, n:2 * n])


def test_wide_angle_needs_local_line_of_sight():
    import jaxpower_b200 as jp
    attrs = jp.MeshAttrs(meshsize=8, boxsize=400.)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.05}, ells=(0,))
    with pytest.raises(ValueError):
        jp.compute_mesh2_spectrum_window(attrs, edgesin=np.array([0., 0.1]), ellsin=[(0, 1)], bin=b, los='z')
    with pytest.raises(NotImplementedError):
        jp.compute_mesh2_spectrum_window(attrs, edgesin=np.array([0., 0.1]), ellsin=([(0, 1)], 'local'), bin=b,
                                         los='firstpoint')


@pytest.mark.parametrize('flag', [None, 'infinite'])
def test_firstpoint_window_mode_oversampling_matches_oracle(flag):
    """First-point window and mean spectrum with mode_oversampling = 1: the output bins average
    the shifted binnings (mesh2.py:48-61) through bin(...), as the reference's."""
    import jaxpower_b200 as jp
    from oracle import spectrum as ospec
    meshsize, boxsize, center = (10, 8, 8), np.array([500., 400., 400.]), (900., -200., 300.)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=center)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 2), mode_oversampling=1)
    ob = Bins(Geometry(meshsize, boxsize, center), step=0.02, ells=(0, 2), mode_oversampling=1)
    assert np.allclose(b.nmodes, ob.nmodes)
    sel = np.random.default_rng(41).uniform(0.5, 1.5, meshsize).astype('f4')
    mesh = attrs.create(kind='real', fill=torch.as_tensor(sel))
    edgesin = np.arange(0.005, 0.06, 0.02)
    w = jp.compute_mesh2_spectrum_window(mesh, edgesin=edgesin, ellsin=(0, 2), bin=b, los='firstpoint',
                                         flags=(flag,) if flag else ())
    if flag is None:
        ref = ospec.compute_mesh2_spectrum_window_firstpoint(ob, edgesin, (0, 2), meshes=[sel])
    else:
        ref = ospec.compute_mesh2_spectrum_window_firstpoint_infinite(ob, edgesin, (0, 2), meshes=[sel])
    _check(w.value, ref)
    with pytest.raises(NotImplementedError):
        jp.compute_mesh2_spectrum_window(mesh, edgesin=edgesin, ellsin=(0, 2), bin=b, los='z')
