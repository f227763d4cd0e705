"""afd_check_filters_static: the filter check for callers that may not
allocate device memory (its scratch is a fixed device array inside the
library). Through the C ABI it must return what afd_check_filters returns,
call after call, even though every call reuses the same scratch.

This file is collected last so that a run that stops at the first failure
has already run every other test; it also passes when run alone.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# the FP64 check runs the same kernels on the same data in both entry
# points; results agree to this relative tolerance
RTOL = 1e-12


def _call(lib, name, a, b, n_freq=4096):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    nmat, ncoef = a.shape
    status = np.full(nmat, -1, np.int32)
    min_real = np.full(nmat, np.nan)
    max_root = np.full(nmat, np.nan)
    P = C.POINTER
    rc = getattr(lib, name)(nmat, ncoef, a.ctypes.data_as(P(C.c_double)), b.ctypes.data_as(P(C.c_double)),
                            n_freq, status.ctypes.data_as(P(C.c_int32)), min_real.ctypes.data_as(P(C.c_double)),
                            max_root.ctypes.data_as(P(C.c_double)))
    return rc, status, min_real, max_root


def _filters(seed):
    import ancfield_b200.workloads as W
    a, b = W.passive_filters(5, 4, seed)
    # one unstable filter (pole outside the unit circle) and one active one
    bad_a, bad_b = a[:2].copy(), b[:2].copy()
    bad_b[0] = [1.0, -2.5, 1.2, 0.1]
    bad_a[1] = [-0.3, 0.0, 0.0, 0.0]
    return np.vstack([a, bad_a]), np.vstack([b, bad_b])


def test_static_matches_allocating_check_twice(pkg):
    lib = pkg.afd.library()
    for seed in (11, 12):  # two calls in a row with different inputs
        a, b = _filters(seed)
        rc0, st0, mr0, rt0 = _call(lib, "afd_check_filters", a, b)
        rc1, st1, mr1, rt1 = _call(lib, "afd_check_filters_static", a, b)
        assert rc0 == 0 and rc1 == 0
        assert np.array_equal(st0, st1)
        np.testing.assert_allclose(mr1, mr0, rtol=RTOL, atol=0.0)
        np.testing.assert_allclose(rt1, rt0, rtol=RTOL, atol=0.0)
        assert st1[-2] & 1 and st1[-1] & 2 and not st1[:-2].any()


def test_static_rejects_sizes_beyond_its_scratch(pkg):
    lib = pkg.afd.library()
    a = np.ones((65, 2))
    b = np.ones((65, 2))
    rc, _, _, _ = _call(lib, "afd_check_filters_static", a, b)
    assert rc == pkg.afd.ERR_ARG
    assert b"64 materials" in lib.afd_model_last_error(None)
    # a valid call afterwards still works and leaves nothing behind
    a, b = _filters(13)
    rc0, st0, mr0, _ = _call(lib, "afd_check_filters", a[:3], b[:3])
    rc1, st1, mr1, _ = _call(lib, "afd_check_filters_static", a[:3], b[:3])
    assert rc0 == rc1 == 0
    assert np.array_equal(st0, st1)
    np.testing.assert_allclose(mr1, mr0, rtol=RTOL, atol=0.0)
