"""Reference app drivers restated on the OPS-B200 runtime (C++ drivers in
ops_b200/csrc/apps_*.cpp, reached through the C-ABI)."""
import ctypes

import numpy as np

from ._lib import check, lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def laplace2d(field, iters, warmup=0, return_errors=True):
    """Laplace Jacobi (apps/c/laplace2d_tutorial/step7/laplace2d.cpp:113-124).

    field: (jmax+2, imax+2) float64 full extent (ring = boundary values).
    Returns (final_field, errors_per_iteration, device_seconds)."""
    field = np.ascontiguousarray(field, dtype=np.float64)
    jmax, imax = field.shape[0] - 2, field.shape[1] - 2
    out = np.empty_like(field)
    errs = np.empty(max(warmup + iters, 1), dtype=np.float64) if return_errors else None
    secs = ctypes.c_double(0.0)
    check(lib().ops_b200_app_laplace2d(imax, jmax, warmup, iters, _ptr(field), _ptr(out), _ptr(errs),
                                       ctypes.byref(secs)))
    return out, (errs[:warmup + iters] if errs is not None else None), secs.value
