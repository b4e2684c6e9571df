"""Window matrix of the power-spectrum multipoles (global line of sight): the oracle's own
identities, on the CPU.

- A periodic box with input edges equal to the output bins fills the diagonal in one pass
  per input multipole (mesh2.py:1113-1118); the selection-function path with W = 1
  (Q = c2r(|r2c(1)|^2) / N = 1) walks every input bin through c2r and r2c and must give the
  same matrix.
- The (ell = 0, ell_in = 0) diagonal of the periodic window is 1 in every bin, except the
  first, which loses the k = 0 mode: (nmodes - 1) / nmodes.
"""
import numpy as np
import pytest

from oracle.coords import Geometry
from oracle.spectrum import Bins, compute_mesh2_spectrum_window as owindow


@pytest.mark.parametrize('los', ['z', [0.6, 0., 0.8]])
def test_window_selection_of_ones_is_periodic(los):
    geom = Geometry((16, 12, 10), (400., 300., 250.))
    bins = Bins(geom, step=0.02, ells=(0, 2, 4))
    periodic = owindow(bins, bins.edges, (0, 2, 4), los=los)
    ones = owindow(bins, bins.edges, (0, 2, 4), los=los, meshes=[np.ones(geom.rshape, dtype='f4')])
    nb = bins.nbins
    assert periodic.shape == ones.shape == (3 * nb, 3 * len(bins.edges) - 3)
    fin = np.isfinite(periodic)
    assert np.array_equal(fin, np.isfinite(ones))
    scale = np.abs(periodic[fin]).max()
    assert np.allclose(periodic[fin], ones[fin], atol=2e-5 * scale)
    # periodic: every (ell, ell_in) block diagonal
    block = periodic[:nb, :nb]
    off = block - np.diag(np.diag(block))
    assert np.all(off[np.isfinite(off)] == 0.)
    expect = np.ones(nb)
    expect[0] = (bins.nmodes[0] - 1.) / bins.nmodes[0]
    assert np.allclose(np.diag(block), expect, rtol=1e-6)


def test_window_theory_vector_of_a_constant_power():
    """W @ P_in for a constant monopole P_in = 1 gives 1 in every monopole bin (no k = 0)."""
    geom = Geometry((12, 12, 12), (300., 300., 300.))
    bins = Bins(geom, step=0.03, ells=(0, 2))
    edgesin = np.arange(0., 0.4, 0.01)
    w = owindow(bins, edgesin, (0,), los='x')
    got = w.dot(np.ones(len(edgesin) - 1))
    nb = bins.nbins
    expect = np.ones(nb)
    expect[0] = (bins.nmodes[0] - 1.) / bins.nmodes[0]
    assert np.allclose(got[:nb], expect, rtol=1e-6)
    assert np.allclose(got[nb:], 0., atol=1e-6)  # isotropic input: no quadrupole


def test_smooth2_window_from_correlation_multipoles():
    """compute_smooth2_spectrum_window ('rect'): host sums over the window's separations, against
    plain loops with sympy's Wigner 3j coefficients (no GPU: the output binning is given by its
    attributes)."""
    from types import SimpleNamespace
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_smooth2_spectrum_window as osmooth2
    rng = np.random.default_rng(3)
    s = np.linspace(2.5, 200., 80)
    nmodes = rng.integers(0, 50, s.size).astype('f8')
    windows = {0: np.exp(-s / 80.), 2: 0.3 * np.exp(-s / 60.), 4: 0.1 * np.exp(-s / 40.)}
    poles = jp.Mesh2CorrelationPoles([jp.Mesh2CorrelationPole(s=s, s_edges=np.column_stack([s - 1.25, s + 1.25]),
                                                               nmodes=nmodes, num_raw=windows[q], volume=nmodes, ell=q)
                                      for q in (0, 2, 4)])
    kedges = np.arange(0.01, 0.2, 0.02)
    bin = SimpleNamespace(ells=(0, 2, 4), xavg=(kedges[:-1] + kedges[1:]) / 2.,
                          edges=np.column_stack([kedges[:-1], kedges[1:]]), nmodes=np.ones(kedges.size - 1))
    edgesin = np.arange(0., 0.25, 0.025)
    w = jp.compute_smooth2_spectrum_window(poles, edgesin=edgesin, ellsin=(0, 2, 4), bin=bin)
    ref = osmooth2(s, windows, nmodes, edgesin, (0, 2, 4), (0, 2, 4), bin.xavg)
    assert w.value.shape == ref.shape == (3 * bin.xavg.size, 3 * (edgesin.size - 1))
    assert np.allclose(w.value, ref, rtol=1e-10, atol=1e-12 * np.abs(ref).max())
    assert w.theory.ells == (0, 2, 4)


def test_smooth2_window_wide_angle_orders():
    """compute_smooth2_spectrum_window with wide-angle inputs (ell_in, n): the window multipoles
    labelled with order n times s^n (mesh2.py:845-851, 869); an order n > 0 without labelled
    window multipoles raises ValueError (mesh2.py:850-851)."""
    from types import SimpleNamespace
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_smooth2_spectrum_window as osmooth2
    s = np.linspace(2.5, 200., 60)
    nmodes = np.full(s.size, 3.)
    windows = {(0, 0): np.exp(-s / 80.), (2, 0): 0.3 * np.exp(-s / 60.), (0, 1): 0.01 * np.exp(-s / 50.),
               (2, 1): 0.004 * np.exp(-s / 70.), (1, 1): 0.02 * np.exp(-s / 90.)}
    poles = jp.Mesh2CorrelationPoles([jp.Mesh2CorrelationPole(s=s, s_edges=np.column_stack([s - 1.25, s + 1.25]),
                                                               nmodes=nmodes, num_raw=w, volume=nmodes, ell=q,
                                                               attrs=dict(wa_order=n))
                                      for (q, n), w in windows.items()])
    assert poles.wa_orders == (0, 0, 1, 1, 1)
    kedges = np.arange(0.01, 0.2, 0.02)
    bin = SimpleNamespace(ells=(0, 1, 2), xavg=(kedges[:-1] + kedges[1:]) / 2.,
                          edges=np.column_stack([kedges[:-1], kedges[1:]]), nmodes=np.ones(kedges.size - 1))
    edgesin = np.arange(0., 0.25, 0.025)
    ellsin = [(0, 0), (2, 0), (1, 1), (0, 1)]
    w = jp.compute_smooth2_spectrum_window(poles, edgesin=edgesin, ellsin=ellsin, bin=bin)
    ref = osmooth2(s, windows, nmodes, edgesin, ellsin, (0, 1, 2), bin.xavg)
    assert np.allclose(w.value, ref, rtol=1e-10, atol=1e-12 * np.abs(ref).max())
    assert w.theory.wa_orders == (0, 0, 1, 1)
    plain = jp.Mesh2CorrelationPoles([jp.Mesh2CorrelationPole(s=s, s_edges=np.column_stack([s - 1.25, s + 1.25]),
                                                               nmodes=nmodes, num_raw=windows[q, 0], volume=nmodes,
                                                               ell=q) for q in (0, 2)])
    with pytest.raises(ValueError):
        jp.compute_smooth2_spectrum_window(plain, edgesin=edgesin, ellsin=[(0, 1)], bin=bin)
