"""Loader of the oracle's C restatements (TEST INFRASTRUCTURE ONLY).

``paint_c.c`` restates the scatter of ``paint.py:paint_mesh`` (``resamplers.py:57-97``)
in C so that the oracle finishes the 512^3 configurations in seconds.  It is compiled
with gcc into ``oracle/_build/liboracle.so`` by ``build()`` (``__graft_entry__.py``), or
here on first use; float contraction is off, so the float32 arithmetic is the NumPy
restatement's, operation for operation.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = [os.path.join(HERE, 'paint_c.c')]
LIBRARY = os.path.join(HERE, '_build', 'liboracle.so')
_lib = None


def build(force=False):
    """Compile the C restatements (gcc, -O2, no float contraction); return the library path."""
    newest = max(os.path.getmtime(s) for s in SOURCES)
    if not force and os.path.exists(LIBRARY) and os.path.getmtime(LIBRARY) >= newest:
        return LIBRARY
    os.makedirs(os.path.dirname(LIBRARY), exist_ok=True)
    tmp = LIBRARY + '.{}.tmp'.format(os.getpid())
    cmd = ['gcc', '-O2', '-fPIC', '-shared', '-ffp-contract=off', '-fno-fast-math', '-o', tmp] + SOURCES + ['-lm']
    subprocess.run(cmd, check=True, capture_output=True)
    os.replace(tmp, LIBRARY)
    return LIBRARY


def load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(build())
        i64p = ctypes.POINTER(ctypes.c_int64)
        for name in ('oracle_paint_serial', 'oracle_paint_f64', 'oracle_paint_double'):
            fn = getattr(lib, name)
            fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, i64p, ctypes.c_void_p]
            fn.restype = None
        _lib = lib
    return _lib


def paint(shape, u, weights, order, accum):
    """Scatter of ``paint_mesh``: accum 'serial' (float32, np.add.at order), 'f64' (float32
    contributions summed in float64) or 'double' (everything in float64)."""
    lib = load()
    if accum == 'double':
        u = np.ascontiguousarray(u, dtype=np.float64)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        acc = np.zeros(tuple(int(s) for s in shape), dtype=np.float64)
        shp = (ctypes.c_int64 * 3)(*[int(s) for s in shape])
        lib.oracle_paint_double(u.ctypes.data, None if w is None else w.ctypes.data, u.shape[0], int(order), shp,
                                acc.ctypes.data)
        return acc
    u = np.ascontiguousarray(u, dtype=np.float32)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
    shp = (ctypes.c_int64 * 3)(*[int(s) for s in shape])
    n = u.shape[0]
    wptr = None if w is None else w.ctypes.data
    if accum == 'serial':
        mesh = np.zeros(tuple(int(s) for s in shape), dtype=np.float32)
        lib.oracle_paint_serial(u.ctypes.data, wptr, n, int(order), shp, mesh.ctypes.data)
        return mesh
    acc = np.zeros(tuple(int(s) for s in shape), dtype=np.float64)
    lib.oracle_paint_f64(u.ctypes.data, wptr, n, int(order), shp, acc.ctypes.data)
    return acc
