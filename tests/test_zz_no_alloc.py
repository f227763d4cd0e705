"""afd_check_filters_static: the filter check for callers that may not
allocate device memory (its scratch is a fixed device array inside the
library). Through the C ABI it must return what afd_check_filters returns,
call after call, even though every call reuses the same scratch; it must
agree with numpy's roots and admittance; and it must work when no device
memory is left to allocate.

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


def test_static_against_independent_restatement(pkg):
    """Stability radius against numpy's polynomial roots and the passivity
    minimum against the numpy admittance on the same frequency grid, on the
    GPU box (the CPU suite checks the host path the same way)."""
    import ancfield_b200.workloads as W
    lib = pkg.afd.library()
    a, b = _filters(14)
    rc, st, mr, rt = _call(lib, "afd_check_filters_static", a, b)
    assert rc == 0
    np.testing.assert_allclose(rt, [np.abs(np.roots(b[m])).max() for m in range(len(b))], rtol=1e-9)
    np.testing.assert_allclose(mr, W.admittance_real_min(a, b), rtol=1e-9)


def test_static_full_layout_and_coefficient_limit(pkg):
    """64 materials x 16 coefficients (the b, root and partial-minimum slots
    at their largest offsets) equals the allocating check; 17 coefficients
    are rejected before anything runs."""
    import ancfield_b200.workloads as W
    lib = pkg.afd.library()
    a, b = W.passive_filters(64, 16, 15)
    rc0, st0, mr0, rt0 = _call(lib, "afd_check_filters", a, b)
    rc1, st1, mr1, rt1 = _call(lib, "afd_check_filters_static", a, b)
    assert rc0 == 0 and rc1 == 0
    assert np.array_equal(st0, st1) and not st1.any()
    np.testing.assert_allclose(mr1, mr0, rtol=RTOL, atol=0.0)
    np.testing.assert_allclose(rt1, rt0, rtol=RTOL, atol=0.0)
    rc, _, _, _ = _call(lib, "afd_check_filters_static", np.ones((4, 17)), np.ones((4, 17)))
    assert rc == pkg.afd.ERR_ARG


def test_static_call_leaves_device_memory_unchanged(pkg):
    """No allocation that outlives the call, and none by the library's own
    allocator during it: the device's free memory is the same before and
    after warmed-up calls (the allocating check's buffers are freed again,
    so this alone does not tell the two apart; the static check's source has
    no allocation call at all, and its kernels use no local memory, which the
    driver would otherwise reserve for the launch)."""
    import torch
    lib = pkg.afd.library()
    a, b = _filters(16)
    rc, st_ref, mr_ref, _ = _call(lib, "afd_check_filters_static", a, b)
    assert rc == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        rc, st, mr, _ = _call(lib, "afd_check_filters_static", a, b)
        assert rc == 0
        assert np.array_equal(st, st_ref)
        np.testing.assert_allclose(mr, mr_ref, rtol=RTOL, atol=0.0)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
