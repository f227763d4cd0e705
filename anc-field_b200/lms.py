"""LMS impulse-response estimation on the GPU (include/afd_lms.h), with the
reference's signature: EstimateIr(input, output, N, mu=1e-4) of
anc_field_py/ancutil.py:24-37 (16 passes of sample-serial LMS, FP64)."""
import ctypes as C

import numpy as np

from . import afd

EXPORTS = ["afd_lms_estimate", "afd_lms_last_error"]
_bound = False


def _lib():
    global _bound
    L = afd.library()
    if not _bound:
        P = C.POINTER
        L.afd_lms_estimate.restype = C.c_int
        L.afd_lms_estimate.argtypes = [P(C.c_double), C.c_int64, P(C.c_double), C.c_int64, C.c_int32, C.c_double,
                                       C.c_int32, C.c_int32, P(C.c_double)]
        L.afd_lms_last_error.restype = C.c_char_p
        L.afd_lms_last_error.argtypes = []
        _bound = True
    return L


def estimate_ir(x, d, N, mu=1e-4, epochs=16, device=0):
    """Weights [N] (float64) of the LMS estimate of the response from x to d."""
    x = np.ascontiguousarray(x, dtype=np.float64).ravel()
    d = np.ascontiguousarray(d, dtype=np.float64).ravel()
    N = int(N)
    w = np.zeros(max(N, 1), np.float64)
    L = _lib()
    P = C.POINTER(C.c_double)
    st = L.afd_lms_estimate(x.ctypes.data_as(P), x.size, d.ctypes.data_as(P), d.size, N, float(mu), int(epochs),
                            int(device), w.ctypes.data_as(P))
    if st != afd.OK:
        raise afd.AfdError(st, L.afd_lms_last_error().decode())
    return w[:N]


def EstimateIr(input, output, N, mu=1e-4):  # noqa: N802 - the reference's name
    return estimate_ir(input, output, N, mu)
