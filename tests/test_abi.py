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
