"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module. `simulate(impl=...)`:
  impl="ora"  the restatement afd_oracle.c (_build/liboracle.so)
  impl="ref"  the reference's own kernel sources compiled by
              ref_harness.c (_ref/libref32.so, _ref/libref64.so)
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORA_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIBS = {"f32": os.path.join(HERE, "_ref", "libref32.so"),
            "f64": os.path.join(HERE, "_ref", "libref64.so")}

_loaded = {}
P = C.POINTER
_ARGS = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_int32), C.c_int, C.c_int,
         P(C.c_double), P(C.c_double), C.c_double, C.c_double, C.c_double, C.c_int, C.c_uint,
         P(C.c_float), P(C.c_float), P(C.c_float), C.c_int, P(C.c_int32), P(C.c_int64), P(C.c_int64),
         P(C.c_float), C.c_int, P(C.c_int32), C.c_int, P(C.c_int64), P(C.c_float), P(C.c_float)]


def available(impl="ora", precision="f32"):
    path = ORA_LIB if impl == "ora" else REF_LIBS[precision]
    return os.path.exists(path)


def _fn(impl, precision):
    key = (impl, precision)
    if key in _loaded:
        return _loaded[key]
    if impl == "ora":
        lib = C.CDLL(ORA_LIB)
        fn = getattr(lib, "ora_simulate_" + precision)
    else:
        lib = C.CDLL(REF_LIBS[precision])
        fn = getattr(lib, "ref_simulate_" + precision)
    fn.restype = C.c_int
    fn.argtypes = _ARGS
    _loaded[key] = fn
    return fn


def ref_timing(pml_parallel, precision="f32"):
    """Timing controls of the reference harness (impl "ref"): whether its PML
    NDRange runs over all host threads (as a CPU OpenCL device runs it) and a
    reader of the last call's step-loop wall seconds (set-up excluded)."""
    lib = C.CDLL(REF_LIBS[precision])
    lib.ref_set_pml_parallel.argtypes = [C.c_int]
    lib.ref_set_pml_parallel.restype = None
    lib.ref_last_loop_seconds.argtypes = []
    lib.ref_last_loop_seconds.restype = C.c_double
    lib.ref_set_pml_parallel(1 if pml_parallel else 0)
    return lib.ref_last_loop_seconds


def _p(a, t):
    return a.ctypes.data_as(P(t))


def simulate(grid, vox=None, a=None, b=None, dx=0.02, c=340.0, dt=3.125e-5, mode=0, pml_width=0,
             faces=63, ksi=None, sources=(), receivers=(), steps=100, runs=None, impl="ora",
             precision="f32", want_field=False):
    """One batch member. grid = (nx, ny, nz); vox int32 [mz, my, mx] or None;
    a, b [nmat, K]; sources = [((i, j, k), signal)]; receivers = [(i, j, k)];
    runs = list of consecutive run lengths (default [steps]).
    precision "f16": the FIXED scheme with FP16 storage of the pressure levels.
    Returns (receivers [n, T] float32, field [nz, ny, nx] or None)."""
    nx, ny, nz = grid
    runs = list(runs) if runs is not None else [steps]
    total = int(sum(runs))
    if vox is None:
        mx = my = mz = 0
        vox_a = np.zeros(1, np.int32)
    else:
        vox_a = np.ascontiguousarray(vox, dtype=np.int32)
        mz, my, mx = vox_a.shape
    if a is None:
        a = np.ones((1, 1))
        b = np.ones((1, 1))
    a = np.ascontiguousarray(np.atleast_2d(a), dtype=np.float64)
    b = np.ascontiguousarray(np.atleast_2d(b), dtype=np.float64)
    nmat, K = a.shape
    if ksi is None:
        ksi = (np.zeros(nx), np.zeros(ny), np.zeros(nz))
    kx, ky, kz = [np.ascontiguousarray(k, dtype=np.float32) for k in ksi]
    src_ijk = np.ascontiguousarray([s[0] for s in sources] or [(0, 0, 0)], dtype=np.int32)
    sigs = [np.asarray(s[1], dtype=np.float32).ravel() for s in sources]
    src_len = np.ascontiguousarray([len(s) for s in sigs] or [0], dtype=np.int64)
    src_off = np.ascontiguousarray(np.concatenate([[0], np.cumsum(src_len)[:-1]]) if sigs else [0],
                                   dtype=np.int64)
    src_data = np.ascontiguousarray(np.concatenate(sigs) if sigs and sum(map(len, sigs)) else [0.0],
                                    dtype=np.float32)
    rcv_ijk = np.ascontiguousarray(list(receivers) or [(0, 0, 0)], dtype=np.int32)
    nr = len(receivers)
    out = np.zeros((max(nr, 1), max(total, 1)), np.float32)
    field = np.zeros((nz, ny, nx), np.float32) if want_field else None
    run_arr = np.ascontiguousarray(runs, dtype=np.int64)
    fn = _fn(impl, precision)
    st = fn(mode, nx, ny, nz, mx, my, mz, _p(vox_a, C.c_int32), nmat, K, _p(a, C.c_double),
            _p(b, C.c_double), float(dx), float(c), float(dt), int(pml_width), int(faces),
            _p(kx, C.c_float), _p(ky, C.c_float), _p(kz, C.c_float), len(sources), _p(src_ijk, C.c_int32),
            _p(src_off, C.c_int64), _p(src_len, C.c_int64), _p(src_data, C.c_float), nr,
            _p(rcv_ijk, C.c_int32), len(runs), _p(run_arr, C.c_int64), _p(out, C.c_float),
            _p(field, C.c_float) if want_field else None)
    if st != 0:
        raise RuntimeError("oracle simulate failed with %d" % st)
    return out[:nr, :total], field
