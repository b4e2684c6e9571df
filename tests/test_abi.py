"""C ABI boundary checks that need no GPU: the library loads and exports every
entry point ``include/jaxpower_b200.h`` declares; argument validation errors are
reported through status codes without touching the device."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, 'include', 'jaxpower_b200.h')


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(pk_[a-z0-9_]+)\s*\(', text)))


@pytest.fixture(scope='module')
def lib():
    from jaxpower_b200 import _lib
    if not os.path.exists(_lib.LIBRARY_PATH):
        import subprocess, sys
        subprocess.check_call([sys.executable, os.path.join(ROOT, 'jax-power_b200', 'build.py')])
    return _lib.load()


def test_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name


def test_python_binding_covers_header():
    from jaxpower_b200 import _lib
    names = set(declared_symbols()) - {'pk_version', 'pk_last_error'}
    assert names <= set(_lib.SIGNATURES), names - set(_lib.SIGNATURES)


def test_status_codes_without_gpu(lib):
    from jaxpower_b200 import _lib
    nbytes = ctypes.c_size_t()
    assert lib.pk_paint_workspace_size(1000, _lib.i32([64, 64, 64]), 3, 3, ctypes.byref(nbytes)) == 0
    assert nbytes.value > 1000 * 16
    assert lib.pk_paint_workspace_size(1000, _lib.i32([64, 64, 64]), 5, 3, ctypes.byref(nbytes)) == 1
    assert b'order' in lib.pk_last_error()
    assert lib.pk_paint_workspace_size(1000, _lib.i32([0, 64, 64]), 2, 1, ctypes.byref(nbytes)) == 1
    assert lib.pk_bin_workspace_size(_lib.i32([64, 64, 64]), 21, 3, ctypes.byref(nbytes)) in (0, 2)
    assert lib.pk_version().startswith(b'jaxpower_b200')


def test_argument_errors_of_later_entries_without_gpu(lib):
    """Entry points reject bad arguments before any launch (fake, never dereferenced
    pointers stand for device buffers)."""
    from jaxpower_b200 import _lib
    fake = ctypes.c_void_p(4096)
    nbytes = ctypes.c_size_t()
    ms = _lib.i32([32, 32, 32])
    # paint tile configurations 0..10 (4..7 swizzled, 8..10 the per-shift kernel); 11 is out of range
    assert lib.pk_paint_batch_workspace_size(1000, 1, ms, 3, 3, 10, ctypes.byref(nbytes)) == 0
    assert lib.pk_paint_batch_workspace_size(1000, 1, ms, 3, 3, 11, ctypes.byref(nbytes)) == 1
    geo = (ms, _lib.f32([100.] * 3), _lib.f32([0.] * 3), _lib.f32([100. / 32] * 3), 3)
    # interlaced read: interlacing out of range, NULL meshes
    assert lib.pk_read_interlaced(None, fake, 0, fake, None, 10, *geo, 1., fake, fake, 0) == 1
    assert lib.pk_read_interlaced(None, fake, 9, fake, None, 10, *geo, 1., fake, fake, 0) == 1
    assert lib.pk_read_interlaced(None, None, 3, fake, None, 10, *geo, 1., fake, fake, 0) == 1
    assert b'NULL' in lib.pk_last_error() or b'null' in lib.pk_last_error()
    # Y_lm premultiply: no terms, or an (ell, m) outside |m| <= ell <= 8
    cs, off = _lib.f32([1.] * 3), _lib.f32([0.] * 3)
    assert lib.pk_ylm_premultiply(None, fake, ms, cs, off, 0, _lib.i32([2]), _lib.i32([0]), fake) == 1
    assert lib.pk_ylm_premultiply(None, fake, ms, cs, off, 1, _lib.i32([2]), _lib.i32([3]), fake) == 1
    assert lib.pk_ylm_premultiply(None, fake, ms, cs, off, 1, _lib.i32([9]), _lib.i32([0]), fake) == 1
    # first-point binning: too many terms, bad number of multipoles
    kf, ells = _lib.f32([0.01] * 3), _lib.i32([0, 2, 4])
    assert lib.pk_bin_firstpoint(None, fake, None, fake, 33, _lib.i32([2] * 33), _lib.i32([0] * 33), ms, kf, fake,
                                 10, 0.01, 0, 3, ells, 1, 0, fake, fake, 1 << 20) == 1
    assert lib.pk_bin_firstpoint(None, fake, None, fake, 5, _lib.i32([2] * 5), _lib.i32(range(-2, 3)), ms, kf, fake,
                                 10, 0.01, 0, 0, ells, 1, 0, fake, fake, 1 << 20) == 1


def test_window_argument_errors_without_gpu(lib):
    """Window-matrix entry points: column count, multipole range, layout and NULL checks."""
    from jaxpower_b200 import _lib
    fake = ctypes.c_void_p(4096)
    ms, kf, los = _lib.i32([32, 32, 32]), _lib.f32([0.01] * 3), _lib.f32([0., 0., 1.])
    lo, hi = _lib.f32([0.] * 17), _lib.f32([0.1] * 17)
    assert lib.pk_window_fill(None, ms, kf, 0, los, 2, 1., 0, lo, hi, fake) == 1
    assert lib.pk_window_fill(None, ms, kf, 0, los, 2, 1., 17, lo, hi, fake) == 1
    assert lib.pk_window_fill(None, ms, kf, 0, los, 9, 1., 1, lo, hi, fake) == 1
    assert lib.pk_window_fill(None, ms, kf, 1, los, 2, 1., 1, lo, hi, fake) == 1  # jaxdecomp layout
    assert lib.pk_window_fill(None, ms, kf, 0, los, 2, 1., 1, lo, hi, None) == 1
    assert lib.pk_window_multiply(None, fake, 1, ctypes.c_void_p(4100), 64) == 1  # misaligned
    assert lib.pk_window_multiply(None, fake, 0, fake, 64) == 1
    ells = _lib.i32([0, 2, 4])
    assert lib.pk_bin_window(None, None, ms, kf, los, fake, 10, 0.01, 0, 0, ells, 0, 0., 1., 1., fake, fake,
                             1 << 20) == 1
    assert lib.pk_bin_window(None, None, ms, kf, los, fake, 10, 0.01, 0, 3, ells, 10, 0., 1., 1., fake, fake,
                             1 << 20) == 1
    assert lib.pk_bin_window(None, None, ms, kf, los, None, 10, 0.01, 0, 3, ells, 0, 0., 1., 1., fake, fake,
                             1 << 20) == 1
    pe, pi = _lib.i32([0] * 10), _lib.i32([0] * 10)
    assert lib.pk_bin_window_pairs(None, ms, kf, los, fake, 10, 0., 0, 0, pe, pi, 1., fake, fake, 1 << 20) == 1
    assert lib.pk_bin_window_pairs(None, ms, kf, los, fake, 10, 0., 0, 10, pe, pi, 1., fake, fake, 1 << 20) == 1
    assert lib.pk_bin_window_pairs(None, ms, kf, los, fake, 10, 0., 1, 3, pe, pi, 1., fake, fake, 1 << 20) == 1
    ev = _lib.i32([0, 2, 4, 6, 8, 0])
    assert lib.pk_bin_window_batch(None, fake, 1, ms, kf, los, fake, 10, 0.01, 0, 6, ev, 1, fake, fake, 1 << 20) == 1
    assert lib.pk_bin_window_batch(None, fake, 1, ms, kf, los, fake, 10, 0.01, 0, 2, _lib.i32([0, 1]), 1, fake, fake,
                                   1 << 20) == 1
    assert lib.pk_bin_window_batch(None, fake, 0, ms, kf, los, fake, 10, 0.01, 0, 2, ev, 1, fake, fake, 1 << 20) == 1
    assert lib.pk_bin_window_batch(None, None, 1, ms, kf, los, fake, 10, 0.01, 0, 2, ev, 1, fake, fake, 1 << 20) == 1


def test_argument_errors_of_bessel_adjoint_and_shift_entries_without_gpu(lib):
    """The Bessel projection, wide-angle factor, C2R adjoint and shifted (mode oversampling)
    entry points reject bad arguments before any launch."""
    from jaxpower_b200 import _lib
    fake = ctypes.c_void_p(4096)
    nbytes = ctypes.c_size_t()
    ms, kf, cs, off = _lib.i32([32, 32, 32]), _lib.f32([0.01] * 3), _lib.f32([1.] * 3), _lib.f32([0.] * 3)
    los, ells = _lib.f32([0., 0., 1.]), _lib.i32([0, 2, 4])
    # Bessel basis: at most 1024 separation bins and 5 multipoles; terms are first-point inputs
    assert lib.pk_bin_bessel_workspace_size(ms, 2000, 3, ctypes.byref(nbytes)) == 4
    assert lib.pk_bin_bessel_workspace_size(ms, 10, 6, ctypes.byref(nbytes)) == 4
    assert lib.pk_bin_bessel(None, fake, None, None, 0, None, None, ms, kf, 0, los, fake, 2000, None, 3, ells, 1, 0,
                             fake, fake, 1 << 20) == 4
    assert lib.pk_bin_bessel(None, fake, None, fake, 1, _lib.i32([2]), _lib.i32([0]), ms, kf, 0, los, fake, 10, None,
                             3, ells, 1, 0, fake, fake, 1 << 20) == 1
    assert lib.pk_bin_bessel(None, fake, None, None, 0, None, None, ms, kf, 0, los, fake, 10, None, 1,
                             _lib.i32([6]), 1, 0, fake, fake, 1 << 20) == 4
    # wide-angle factors: |power| <= 8, an offset for positions
    assert lib.pk_radial_power(None, fake, 1, ms, cs, off, 0, 9) == 1
    assert lib.pk_radial_power(None, fake, 1, ms, cs, None, 0, 1) == 1
    assert lib.pk_radial_power(None, fake, 0, ms, cs, off, 1, 1) == 1
    # C2R adjoint: NULL buffers
    assert lib.pk_c2r_adjoint(None, None, ms, 0, fake) == 1
    # shifted adjoints: at most 125 shifts, a shift array
    many = _lib.f32([0.] * (3 * 126))
    assert lib.pk_bin_global_adjoint_shifted(None, fake, ms, kf, los, fake, 10, 0.01, 0., 0, 3, ells, fake, 1, 126,
                                             many, fake, fake, 1 << 20) == 4
    assert lib.pk_bin_firstpoint_adjoint_shifted(None, fake, None, 0, None, None, ms, kf, fake, 10, 0.01, 0., 0, 3,
                                                 ells, fake, 1, 27, None, fake, 0, None, fake, 1 << 20) == 1
    # shifted separation bins: a shift vector
    assert lib.pk_bin_separation_modes_shifted(None, ms, cs, None, fake, 10, 10., 0, fake, fake, fake, 1 << 20) == 1
    assert lib.pk_bin_separation_global_shifted(None, fake, ms, cs, None, los, fake, 10, 10., 3, ells, 0, fake, fake,
                                                1 << 20) == 1
