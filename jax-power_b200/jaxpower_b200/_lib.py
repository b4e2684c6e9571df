"""ctypes binding of the C ABI (``include/jaxpower_b200.h``).

This is the same boundary a ``jax.ffi`` / cgo / JNI caller would bind: plain
device pointers, sizes and a CUDA stream.  The library must be built
(``python jax-power_b200/build.py``); there is no CPU fallback — importing a
compute entry point without the library raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, 'libjaxpower_b200.so')

PK_BACKEND_JAX = 0
PK_BACKEND_JAXDECOMP = 1

c_int = ctypes.c_int
c_int64 = ctypes.c_int64
c_float = ctypes.c_float
c_size_t = ctypes.c_size_t
c_void_p = ctypes.c_void_p
c_double_p = ctypes.POINTER(ctypes.c_double)
c_float_p = ctypes.POINTER(ctypes.c_float)
c_int32_p = ctypes.POINTER(ctypes.c_int32)

# name -> (argtypes); every entry point returns an int status except the two strings
SIGNATURES = {
    'pk_paint_workspace_size': [c_int64, c_int32_p, c_int, c_int, ctypes.POINTER(c_size_t)],
    'pk_paint': [c_void_p, c_void_p, c_void_p, c_int64, c_int32_p, c_float_p, c_float_p, c_float_p,
                 c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_size_t, c_void_p],
    'pk_paint_batch_workspace_size': [c_int64, c_int, c_int32_p, c_int, c_int, c_int, ctypes.POINTER(c_size_t)],
    'pk_paint_batch': [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int, c_int32_p, c_float_p, c_float_p,
                       c_float_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_size_t, c_void_p],
    'pk_interlace_compensate_batch': [c_void_p, c_void_p, c_int, c_int, c_int32_p, c_int, c_int, c_int, c_float,
                                      c_void_p],
    'pk_bin_batch_workspace_size': [c_int32_p, c_int, c_int, c_int, ctypes.POINTER(c_size_t)],
    'pk_bin_global_batch': [c_void_p, c_void_p, c_void_p, c_int, c_int32_p, c_float_p, c_float_p, c_void_p,
                            c_int, c_float, c_int, c_int, c_int32_p, c_void_p, c_void_p, c_size_t],
    'pk_read': [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32_p, c_float_p, c_float_p,
                c_float_p, c_int, c_float, c_float, c_void_p, c_void_p, c_int],
    'pk_read_interlaced': [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int64, c_int32_p, c_float_p, c_float_p,
                           c_float_p, c_int, c_float, c_void_p, c_void_p, c_int],
    'pk_fft_plan_create': [c_int32_p, c_int, c_int, ctypes.POINTER(c_void_p)],
    'pk_fft_exec': [c_void_p, c_void_p, c_void_p, c_void_p],
    'pk_fft_plan_destroy': [c_void_p],
    'pk_interlace_compensate': [c_void_p, c_void_p, c_int, c_int32_p, c_int, c_int, c_int, c_float,
                                c_void_p],
    'pk_scale_real': [c_void_p, c_void_p, c_int64, c_float],
    'pk_uniform_ids': [c_void_p, ctypes.c_uint64, c_void_p, c_int64, c_void_p],
    'pk_bin_workspace_size': [c_int32_p, c_int, c_int, ctypes.POINTER(c_size_t)],
    'pk_bin_modes': [c_void_p, c_int32_p, c_float_p, c_void_p, c_int, c_float, c_int, c_void_p,
                     c_void_p, c_void_p, c_size_t],
    'pk_bin_mesh': [c_void_p, c_void_p, c_int32_p, c_float_p, c_void_p, c_int, c_float, c_int, c_int,
                    c_void_p, c_void_p, c_size_t],
    'pk_bin_modes_shifted': [c_void_p, c_int32_p, c_float_p, c_float_p, c_void_p, c_int, c_float, c_int, c_int,
                             c_void_p, c_void_p, c_void_p, c_size_t],
    'pk_bin_mesh_shifted': [c_void_p, c_void_p, c_int32_p, c_float_p, c_float_p, c_void_p, c_int, c_float, c_int,
                            c_int, c_int, c_void_p, c_void_p, c_size_t],
    'pk_bin_global_shifted': [c_void_p, c_void_p, c_void_p, c_int32_p, c_float_p, c_float_p, c_float_p, c_void_p,
                              c_int, c_float, c_int, c_int, c_int32_p, c_int, c_void_p, c_void_p, c_size_t],
    'pk_bin_firstpoint_shifted': [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int32_p, c_int32_p, c_int32_p,
                                  c_float_p, c_float_p, c_void_p, c_int, c_float, c_int, c_int, c_int32_p, c_int,
                                  c_int, c_void_p, c_void_p, c_size_t],
    'pk_bin_global': [c_void_p, c_void_p, c_void_p, c_int32_p, c_float_p, c_float_p, c_void_p,
                      c_int, c_float, c_int, c_int, c_int32_p, c_void_p, c_void_p, c_size_t],
    'pk_bin_separation_workspace_size': [c_int32_p, c_int, c_int, ctypes.POINTER(c_size_t)],
    'pk_bin_separation_modes': [c_void_p, c_int32_p, c_float_p, c_void_p, c_int, c_float, c_void_p, c_void_p,
                                c_void_p, c_size_t],
    'pk_bin_separation_global': [c_void_p, c_void_p, c_int32_p, c_float_p, c_float_p, c_void_p, c_int, c_float,
                                 c_int, c_int32_p, c_void_p, c_void_p, c_size_t],
    'pk_ylm_separation_accumulate': [c_void_p, c_void_p, c_int32_p, c_float_p, c_int, c_int32_p, c_int32_p,
                                     c_void_p],
    'pk_conj_multiply': [c_void_p, c_void_p, c_void_p, c_int, c_int64, c_void_p],
    'pk_window_fill': [c_void_p, c_int32_p, c_float_p, c_int, c_float_p, c_int, c_float, c_int, c_float_p,
                       c_float_p, c_void_p],
    'pk_window_multiply': [c_void_p, c_void_p, c_int, c_void_p, c_int64],
    'pk_bin_window_batch': [c_void_p, c_void_p, c_int, c_int32_p, c_float_p, c_float_p, c_void_p, c_int, c_float,
                            c_int, c_int, c_int32_p, c_int, c_void_p, c_void_p, c_size_t],
    'pk_ylm_kgrid_multiply': [c_void_p, c_void_p, c_int32_p, c_float_p, c_int, c_int32_p, c_int32_p, c_float,
                              c_int, c_void_p],
    'pk_sum_products': [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_float_p, c_int64, c_int],
    'pk_bin_window_pairs': [c_void_p, c_int32_p, c_float_p, c_float_p, c_void_p, c_int, c_float, c_int, c_int,
                            c_int32_p, c_int32_p, c_float, c_void_p, c_void_p, c_size_t],
    'pk_bin_window': [c_void_p, c_void_p, c_int32_p, c_float_p, c_float_p, c_void_p, c_int, c_float, c_int, c_int,
                      c_int32_p, c_int, c_float, c_float, c_float, c_void_p, c_void_p, c_size_t],
    'pk_bin_global_interlaced': [c_void_p, c_void_p, c_int, c_int, c_int, c_int32_p, c_float_p, c_float_p, c_void_p,
                                 c_int, c_float, c_int, c_int, c_int32_p, c_void_p, c_void_p, c_size_t],
    'pk_bin_global_noalloc': [c_void_p, c_void_p, c_void_p, c_int32_p, c_float_p, c_float_p, c_void_p,
                              c_int, c_float, c_int, c_int, c_int32_p, c_void_p],
    'pk_bin_firstpoint': [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int32_p, c_int32_p,
                          c_int32_p, c_float_p, c_void_p, c_int, c_float, c_int, c_int, c_int32_p,
                          c_int, c_int, c_void_p, c_void_p, c_size_t],
    'pk_adjoint_workspace_size': [c_int, ctypes.POINTER(c_size_t)],
    'pk_bin_global_adjoint': [c_void_p, c_void_p, c_int32_p, c_float_p, c_float_p, c_void_p, c_int, c_float,
                              c_float, c_int, c_int, c_int32_p, c_void_p, c_int, c_void_p, c_void_p, c_size_t],
    'pk_bin_firstpoint_adjoint': [c_void_p, c_void_p, c_void_p, c_int, c_int32_p, c_int32_p, c_int32_p,
                                  c_float_p, c_void_p, c_int, c_float, c_float, c_int, c_int, c_int32_p,
                                  c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p, c_size_t],
    'pk_bin_global_adjoint_shifted': [c_void_p, c_void_p, c_int32_p, c_float_p, c_float_p, c_void_p, c_int, c_float,
                                      c_float, c_int, c_int, c_int32_p, c_void_p, c_int, c_int, c_float_p, c_void_p,
                                      c_void_p, c_size_t],
    'pk_bin_firstpoint_adjoint_shifted': [c_void_p, c_void_p, c_void_p, c_int, c_int32_p, c_int32_p, c_int32_p,
                                          c_float_p, c_void_p, c_int, c_float, c_float, c_int, c_int, c_int32_p,
                                          c_void_p, c_int, c_int, c_float_p, c_void_p, c_int, c_void_p, c_void_p,
                                          c_size_t],
    'pk_interlace_adjoint': [c_void_p, c_void_p, c_int, c_int, c_int32_p, c_int, c_int, c_void_p],
    'pk_c2r_adjoint': [c_void_p, c_void_p, c_int32_p, c_int, c_void_p],
    'pk_bin_bessel_workspace_size': [c_int32_p, c_int, c_int, ctypes.POINTER(c_size_t)],
    'pk_bin_bessel': [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int32_p, c_int32_p, c_int32_p, c_float_p,
                      c_int, c_float_p, c_void_p, c_int, c_float_p, c_int, c_int32_p, c_int, c_int, c_void_p,
                      c_void_p, c_size_t],
    'pk_radial_power': [c_void_p, c_void_p, c_int, c_int32_p, c_float_p, c_float_p, c_int, c_int],
    'pk_bin_separation_modes_shifted': [c_void_p, c_int32_p, c_float_p, c_float_p, c_void_p, c_int, c_float, c_int,
                                        c_void_p, c_void_p, c_void_p, c_size_t],
    'pk_bin_separation_global_shifted': [c_void_p, c_void_p, c_int32_p, c_float_p, c_float_p, c_float_p, c_void_p,
                                         c_int, c_float, c_int, c_int32_p, c_int, c_void_p, c_void_p, c_size_t],
    'pk_ylm_accumulate': [c_void_p, c_void_p, c_int32_p, c_float_p, c_float_p, c_int, c_int32_p, c_int32_p,
                          c_void_p],
    'pk_ylm_premultiply': [c_void_p, c_void_p, c_int32_p, c_float_p, c_float_p, c_int, c_int32_p,
                           c_int32_p, c_void_p],
    'pk_mlp_num_params': [],
    'pk_mlp_cast': [c_void_p, c_void_p, c_void_p],
    'pk_mlp_forward': [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
    'pk_mlp_forward_tc': [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                          c_void_p],
    'pk_mlp_mse': [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p],
    'pk_mlp_backward_workspace_size': [c_int, ctypes.POINTER(c_size_t)],
    'pk_mlp_backward': [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                        c_void_p, c_size_t],
    'pk_mlp_backward_tc': [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                           c_void_p, c_size_t, c_void_p],
    'pk_mlp_adam': [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p,
                    c_float, c_float, c_float, c_float],
}

_lib = None


class PKError(RuntimeError):
    """Error status returned by the CUDA library."""


def load():
    """Load the library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBRARY_PATH):
        raise ImportError('jaxpower_b200 CUDA library not found at {}; build it with '
                          '`python jax-power_b200/build.py` (there is no CPU fallback)'.format(LIBRARY_PATH))
    lib = ctypes.CDLL(LIBRARY_PATH)
    lib.pk_version.restype = ctypes.c_char_p
    lib.pk_version.argtypes = []
    lib.pk_last_error.restype = ctypes.c_char_p
    lib.pk_last_error.argtypes = []
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = c_int
    _lib = lib
    return lib


def call(name, *args):
    """Call an entry point; raise PKError with the library's message on failure.

    Inside a ``tracing.Timeline`` the call is bracketed by CUDA events.
    """
    lib = load()
    from .tracing import active
    timeline = active()
    token = timeline.start(name) if timeline is not None else None
    status = getattr(lib, name)(*args)
    if token is not None:
        timeline.stop(token)
    if status != 0:
        msg = lib.pk_last_error().decode()
        raise PKError('{} failed (status {}): {}'.format(name, status, msg))
    return status


def i32(values):
    arr = (ctypes.c_int32 * len(values))(*[int(v) for v in values])
    return arr


def f32(values):
    arr = (ctypes.c_float * len(values))(*[float(np.float32(v)) for v in values])
    return arr


def ptr(tensor):
    """Device pointer of a torch tensor (None -> NULL)."""
    if tensor is None:
        return None
    return ctypes.c_void_p(tensor.data_ptr())


def stream_handle(stream=None):
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)
