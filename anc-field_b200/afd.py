"""ctypes binding of the C ABI in include/afd.h and a Python mirror of the
reference's Simulation class (anc-field/src/simulation.hpp:83-156).

The library is lib/libafd.so next to this file (built by build.py). There is
no fallback: if the library or a CUDA device is missing the calls fail with
AfdError.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libafd.so")
EXE_PATH = os.path.join(HERE, "bin", "anc-field")

OK = 0
ERR_ARG, ERR_STATE, ERR_IO, ERR_GEOMETRY, ERR_CUDA, ERR_NUMERIC, ERR_FILTER, ERR_ABORTED = (
    -1, -2, -3, -4, -5, -6, -7, -8)
MODE_REF, MODE_FIXED = 0, 1
STORE_FP32, STORE_FP16 = 0, 1
FACE_XM, FACE_XP, FACE_YM, FACE_YP, FACE_ZM, FACE_ZP = 1, 2, 4, 8, 16, 32
NUM_GROUPS = 26
# group names in the numbering of lrs-data.hpp:53-78
GROUP_NAMES = ["X_P", "X_M", "Y_P", "Y_M", "Z_P", "Z_M", "X_P_Y_P", "X_P_Y_M", "X_P_Z_P", "X_P_Z_M",
               "X_M_Y_P", "X_M_Y_M", "X_M_Z_P", "X_M_Z_M", "Y_P_Z_P", "Y_P_Z_M", "Y_M_Z_P", "Y_M_Z_M",
               "X_P_Y_P_Z_P", "X_P_Y_P_Z_M", "X_P_Y_M_Z_P", "X_P_Y_M_Z_M", "X_M_Y_P_Z_P",
               "X_M_Y_P_Z_M", "X_M_Y_M_Z_P", "X_M_Y_M_Z_M"]

# Every entry point include/afd.h declares.
EXPORTS = [
    "afd_default_params", "afd_version", "afd_device_name",
    "afd_model_load_kerkythea", "afd_model_from_voxels", "afd_model_dims", "afd_model_voxels",
    "afd_model_coefs", "afd_model_material_names", "afd_model_classify", "afd_model_group_points",
    "afd_model_load_kerkythea_on", "afd_model_boundary",
    "afd_model_last_error", "afd_model_destroy", "afd_check_filters", "afd_check_filters_static",
    "afd_create", "afd_set_min_size", "afd_load", "afd_set_model", "afd_set_pml",
    "afd_set_pml_profile", "afd_add_source", "afd_add_source_cell", "afd_add_receiver",
    "afd_add_receiver_cell", "afd_run", "afd_prepare", "afd_get_receivers", "afd_update_source",
    "afd_get_receivers_range", "afd_get_field", "afd_get_plane", "afd_set_capture", "afd_get_frames",
    "afd_set_timeline", "afd_get_timeline", "afd_wait_selftest",
    "afd_get_info", "afd_energy", "afd_set_stream", "afd_set_plan", "afd_set_slab", "afd_step_phase", "afd_halo",
    "afd_kernel_stats", "afd_last_error",
    "afd_destroy",
]


class AfdError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (status %d)" % (msg, status))
        self.status = status


class Params(C.Structure):
    _fields_ = [("dx", C.c_float), ("c", C.c_float), ("dt", C.c_float), ("fs", C.c_float),
                ("mode", C.c_int32), ("storage", C.c_int32), ("batch", C.c_int32),
                ("device", C.c_int32), ("watchdog", C.c_int32), ("graphs", C.c_int32),
                ("fused", C.c_int32), ("profile", C.c_int32), ("reserved", C.c_int32 * 4)]


class Info(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("ncoef", C.c_int32),
                ("nmat", C.c_int32), ("batch", C.c_int32), ("steps_done", C.c_int64),
                ("n_sources", C.c_int64), ("n_receivers", C.c_int64), ("n_boundary", C.c_int64),
                ("group_counts", C.c_int64 * NUM_GROUPS), ("n_pml_cells", C.c_int64),
                ("lambda2", C.c_float), ("mode", C.c_int32), ("storage", C.c_int32),
                ("last_run_ms", C.c_double), ("kernel_launches", C.c_int64),
                ("tile_x", C.c_int32), ("tile_y", C.c_int32), ("tile_z", C.c_int32),
                ("stream_blocks", C.c_int32), ("tuned", C.c_int32), ("stream_beside", C.c_int32),
                ("stream_per_sm", C.c_int32), ("stream_tail", C.c_int32), ("reserved", C.c_int32 * 4)]


class Plan(C.Structure):
    _fields_ = [("tile_x", C.c_int32), ("tile_y", C.c_int32), ("per_sm", C.c_int32), ("dz", C.c_int32),
                ("beside", C.c_int32), ("tail", C.c_int32), ("reserved", C.c_int32 * 2)]


PROGRESS_FN = C.CFUNCTYPE(C.c_int, C.c_int64, C.c_int64, C.c_void_p)

_lib = None


def library(path=LIB_PATH):
    """Loads lib/libafd.so once and declares the signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise AfdError(ERR_STATE, "native library %s is missing: run build.py" % path)
    L = C.CDLL(path)
    vp, i32, i64, f32, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_float, C.c_double
    P = C.POINTER
    sig = {
        "afd_default_params": (None, [P(Params)]),
        "afd_version": (C.c_char_p, []),
        "afd_device_name": (C.c_int, [i32, C.c_char_p, i64]),
        "afd_model_load_kerkythea": (C.c_int, [P(vp), C.c_char_p, f32]),
        "afd_model_from_voxels": (C.c_int, [P(vp), i32, i32, i32, P(i32), i32, i32, P(f32), P(f32)]),
        "afd_model_dims": (C.c_int, [vp, P(i32), P(i32), P(i32)]),
        "afd_model_voxels": (C.c_int, [vp, P(i32), i64]),
        "afd_model_coefs": (C.c_int, [vp, P(f32), P(f32), i64]),
        "afd_model_material_names": (C.c_int, [vp, C.c_char_p, i64]),
        "afd_model_classify": (C.c_int, [vp, P(i64)]),
        "afd_model_group_points": (C.c_int, [vp, i32, P(i32), i64, P(i64)]),
        "afd_model_load_kerkythea_on": (C.c_int, [P(vp), C.c_char_p, f32, i32]),
        "afd_model_boundary": (C.c_int, [vp, i32, P(i32), i64, P(i64)]),
        "afd_model_last_error": (C.c_char_p, [vp]),
        "afd_model_destroy": (None, [vp]),
        "afd_check_filters": (C.c_int, [i32, i32, P(f64), P(f64), i32, P(i32), P(f64), P(f64)]),
        "afd_check_filters_static": (C.c_int, [i32, i32, P(f64), P(f64), i32, P(i32), P(f64), P(f64)]),
        "afd_create": (C.c_int, [P(vp), P(Params)]),
        "afd_set_min_size": (C.c_int, [vp, f32, f32, f32]),
        "afd_load": (C.c_int, [vp, C.c_char_p]),
        "afd_set_model": (C.c_int, [vp, vp]),
        "afd_set_pml": (C.c_int, [vp, i32, C.c_uint32, P(f32), P(f32), P(f32)]),
        "afd_set_pml_profile": (C.c_int, [vp, i32, P(f32), i32]),
        "afd_add_source": (C.c_int, [vp, i32, P(f32), P(f32), i64]),
        "afd_add_source_cell": (C.c_int, [vp, i32, P(i32), P(f32), i64]),
        "afd_add_receiver": (C.c_int, [vp, P(f32)]),
        "afd_add_receiver_cell": (C.c_int, [vp, P(i32)]),
        "afd_run": (C.c_int, [vp, i64, PROGRESS_FN, vp]),
        "afd_prepare": (C.c_int, [vp, i64]),
        "afd_get_receivers": (C.c_int, [vp, i32, P(f32), i64]),
        "afd_update_source": (C.c_int, [vp, i64, i64, P(f32), i64]),
        "afd_get_receivers_range": (C.c_int, [vp, i32, i64, i64, P(f32), i64]),
        "afd_get_field": (C.c_int, [vp, i32, P(f32), i64]),
        "afd_get_plane": (C.c_int, [vp, i32, i32, i32, P(f32), i64]),
        "afd_set_capture": (C.c_int, [vp, i32, i32, i32, i32, i32]),
        "afd_get_frames": (C.c_int, [vp, P(f32), i64, P(i64), i64, P(i32)]),
        "afd_set_timeline": (C.c_int, [vp, i64, i32]),
        "afd_wait_selftest": (C.c_int, [i32, i32, i32, P(i32), P(i64)]),
        "afd_get_timeline": (C.c_int, [vp, P(f64), i64, P(i32)]),
        "afd_get_info": (C.c_int, [vp, P(Info)]),
        "afd_energy": (C.c_int, [vp, i32, P(f64)]),
        "afd_set_stream": (C.c_int, [vp, vp]),
        "afd_set_plan": (C.c_int, [vp, P(Plan)]),
        "afd_set_slab": (C.c_int, [vp, i32, i32]),
        "afd_step_phase": (C.c_int, [vp, i32]),
        "afd_halo": (C.c_int, [vp, i32, i32, i32, vp, i64]),
        "afd_kernel_stats": (C.c_int, [vp, i32, C.c_char_p, i64, P(i64), P(f64)]),
        "afd_last_error": (C.c_char_p, [vp]),
        "afd_destroy": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def default_params(**kw):
    p = Params()
    library().afd_default_params(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def device_names():
    L = library()
    out, buf = [], C.create_string_buffer(256)
    while L.afd_device_name(len(out), buf, 256) == OK:
        out.append(buf.value.decode())
    return out


class Model:
    """Host-side geometry (afd_model): Kerkythea loader or caller voxels."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def load_kerkythea(cls, path, res=0.02, device=None):
        """device=None rasterises on the host, an ordinal on that GPU."""
        L = library()
        h = C.c_void_p()
        if device is None:
            st = L.afd_model_load_kerkythea(C.byref(h), path.encode(), res)
        else:
            st = L.afd_model_load_kerkythea_on(C.byref(h), path.encode(), res, device)
        if st != OK:
            raise AfdError(st, L.afd_model_last_error(None).decode())
        return cls(h)

    @classmethod
    def from_voxels(cls, vox, a, b):
        """vox: int32 [nz, ny, nx] (-1 air); a, b: float32 [nmat, ncoef]."""
        L = library()
        vox = np.ascontiguousarray(vox, dtype=np.int32)
        a = np.ascontiguousarray(np.atleast_2d(a), dtype=np.float32)
        b = np.ascontiguousarray(np.atleast_2d(b), dtype=np.float32)
        nz, ny, nx = vox.shape
        h = C.c_void_p()
        st = L.afd_model_from_voxels(C.byref(h), nx, ny, nz, _ptr(vox, C.c_int32), a.shape[0],
                                     a.shape[1], _ptr(a, C.c_float), _ptr(b, C.c_float))
        if st != OK:
            raise AfdError(st, L.afd_model_last_error(None).decode())
        return cls(h)

    def _check(self, st):
        if st != OK:
            raise AfdError(st, library().afd_model_last_error(self._h).decode())

    @property
    def dims(self):
        d = (C.c_int32 * 3)()
        nm, nc = C.c_int32(), C.c_int32()
        self._check(library().afd_model_dims(self._h, d, C.byref(nm), C.byref(nc)))
        return (d[0], d[1], d[2]), nm.value, nc.value

    def voxels(self):
        (nx, ny, nz), _, _ = self.dims
        out = np.empty((nz, ny, nx), np.int32)
        self._check(library().afd_model_voxels(self._h, _ptr(out, C.c_int32), out.size))
        return out

    def coefs(self):
        _, nm, nc = self.dims
        a = np.empty((nm, nc), np.float32)
        b = np.empty((nm, nc), np.float32)
        self._check(library().afd_model_coefs(self._h, _ptr(a, C.c_float), _ptr(b, C.c_float), a.size))
        return a, b

    def material_names(self):
        buf = C.create_string_buffer(1 << 16)
        self._check(library().afd_model_material_names(self._h, buf, 1 << 16))
        s = buf.value.decode()
        return s.split("\n") if s else []

    def classify(self):
        counts = (C.c_int64 * NUM_GROUPS)()
        self._check(library().afd_model_classify(self._h, counts))
        return np.array(counts[:], dtype=np.int64)

    def group_points(self, group):
        n = C.c_int64()
        self._check(library().afd_model_group_points(self._h, group, None, 0, C.byref(n)))
        out = np.empty((max(n.value, 1), 6), np.int32)
        self._check(library().afd_model_group_points(self._h, group, _ptr(out, C.c_int32), out.size,
                                                     C.byref(n)))
        return out[:n.value]

    def boundary(self, device=None):
        """Rows (x, y, z, group, mat0, mat1, mat2) of every boundary cell in
        z-y-x scan order, classified on the host (device=None) or a GPU."""
        dev = -1 if device is None else int(device)
        n = C.c_int64()
        self._check(library().afd_model_boundary(self._h, dev, None, 0, C.byref(n)))
        out = np.empty((max(n.value, 1), 7), np.int32)
        self._check(library().afd_model_boundary(self._h, dev, _ptr(out, C.c_int32), out.size, C.byref(n)))
        return out[:n.value]

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.afd_model_destroy(self._h)
            self._h = None


def wait_selftest(which, complete, device=0):
    """Bounded-wait self-test on the GPU: (gave up, seconds waited) for
    the streaming kernel's wait (which=0) or the GEMM kernels' (which=1)."""
    t, ns = C.c_int32(), C.c_int64()
    s = library().afd_wait_selftest(device, which, 1 if complete else 0, C.byref(t), C.byref(ns))
    if s != OK:
        raise AfdError(s, "wait self-test failed")
    return bool(t.value), ns.value / 1e9


def check_filters(a, b, n_freq=4096):
    """FP64 stability/passivity check; returns (status, min_real, max_root)."""
    a = np.ascontiguousarray(np.atleast_2d(a), dtype=np.float64)
    b = np.ascontiguousarray(np.atleast_2d(b), dtype=np.float64)
    nm, nc = a.shape
    st = np.zeros(nm, np.int32)
    mr = np.zeros(nm)
    rt = np.zeros(nm)
    L = library()
    s = L.afd_check_filters(nm, nc, _ptr(a, C.c_double), _ptr(b, C.c_double), n_freq,
                            _ptr(st, C.c_int32), _ptr(mr, C.c_double), _ptr(rt, C.c_double))
    if s != OK:
        raise AfdError(s, L.afd_model_last_error(None).decode())
    return st, mr, rt


class Simulation:
    """Mirror of the reference Simulation (simulation.hpp:83-156) on one GPU."""

    def __init__(self, params=None, **kw):
        L = library()
        p = params if params is not None else default_params(**kw)
        self.params = p
        h = C.c_void_p()
        st = L.afd_create(C.byref(h), C.byref(p))
        if st != OK:
            raise AfdError(st, L.afd_last_error(None).decode())
        self._h = h
        self._cb = None

    def _check(self, st):
        if st != OK:
            raise AfdError(st, library().afd_last_error(self._h).decode())

    # --- reference-named methods ---------------------------------------
    def Load(self, path):
        self._check(library().afd_load(self._h, path.encode()))

    def SetModel(self, model):
        self._check(library().afd_set_model(self._h, model._h))

    def SetMinSize(self, x, y, z):
        self._check(library().afd_set_min_size(self._h, x, y, z))

    def SetPml(self, width, profile=None, faces=None, ksi=None):
        """Reference form: SetPml(width, profile) builds the ksi arrays as
        SetPml does. FIXED form: SetPml(width, faces=mask, ksi=(kx, ky, kz))."""
        L = library()
        if ksi is not None:
            k = [np.ascontiguousarray(v, dtype=np.float32) for v in ksi]
            self._check(L.afd_set_pml(self._h, width, 63 if faces is None else faces,
                                      _ptr(k[0], C.c_float), _ptr(k[1], C.c_float), _ptr(k[2], C.c_float)))
        else:
            prof = np.ascontiguousarray([] if profile is None else profile, dtype=np.float32)
            self._check(L.afd_set_pml_profile(self._h, width, _ptr(prof, C.c_float), prof.size))

    def AddSource(self, pos, signal, batch=0):
        sig = np.ascontiguousarray(signal, dtype=np.float32).ravel()
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        self._check(library().afd_add_source(self._h, batch, _ptr(pos, C.c_float), _ptr(sig, C.c_float),
                                             sig.size))

    def AddSourceCell(self, ijk, signal, batch=0):
        sig = np.ascontiguousarray(signal, dtype=np.float32).ravel()
        ijk = np.ascontiguousarray(ijk, dtype=np.int32)
        self._check(library().afd_add_source_cell(self._h, batch, _ptr(ijk, C.c_int32),
                                                  _ptr(sig, C.c_float), sig.size))

    def AddMic(self, pos):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        self._check(library().afd_add_receiver(self._h, _ptr(pos, C.c_float)))

    def AddMicCell(self, ijk):
        ijk = np.ascontiguousarray(ijk, dtype=np.int32)
        self._check(library().afd_add_receiver_cell(self._h, _ptr(ijk, C.c_int32)))

    def Run(self, steps, progress=None):
        """progress(i, steps) -> truthy to stop; called at step 0, every 200
        steps and at the end, like the reference's progress lines."""
        if progress is None:
            cb = PROGRESS_FN()
        else:
            def _cb(i, n, _user):
                return 1 if progress(i, n) else 0
            cb = PROGRESS_FN(_cb)
        self._cb = cb
        self._check(library().afd_run(self._h, int(steps), cb, None))

    def prepare(self, steps):
        """Setup work of Run(steps) (buffers, uploads, CUDA graphs) without
        running a step."""
        self._check(library().afd_prepare(self._h, int(steps)))

    def mics(self, batch=0):
        info = self.info()
        out = np.empty((info.n_receivers, info.steps_done), np.float32)
        self._check(library().afd_get_receivers(self._h, batch, _ptr(out, C.c_float), out.size))
        return out

    # --- additions --------------------------------------------------------
    def update_source(self, index, t0, signal):
        sig = np.ascontiguousarray(signal, dtype=np.float32).ravel()
        self._check(library().afd_update_source(self._h, index, t0, _ptr(sig, C.c_float), sig.size))

    def mics_range(self, t0, t1, batch=0, out=None):
        info = self.info()
        if out is None:
            out = np.empty((info.n_receivers, t1 - t0), np.float32)
        self._check(library().afd_get_receivers_range(self._h, batch, t0, t1, _ptr(out, C.c_float), out.size))
        return out

    def info(self):
        i = Info()
        self._check(library().afd_get_info(self._h, C.byref(i)))
        return i

    def field(self, batch=0):
        i = self.info()
        out = np.empty((i.nz, i.ny, i.nx), np.float32)
        self._check(library().afd_get_field(self._h, batch, _ptr(out, C.c_float), out.size))
        return out

    def plane(self, axis, index, batch=0):
        i = self.info()
        shape = {0: (i.nz, i.ny), 1: (i.nz, i.nx), 2: (i.ny, i.nx)}[axis]
        out = np.empty(shape, np.float32)
        self._check(library().afd_get_plane(self._h, batch, axis, index, _ptr(out, C.c_float), out.size))
        return out

    def set_capture(self, axis, index, every, max_frames=64, batch=0):
        """From the next Run on, copy a plane (the plane() layout) after every
        `every`-th step of each run into a ring of max_frames device frames."""
        self._check(library().afd_set_capture(self._h, batch, axis, index, every, max_frames))
        self._cap = (axis, max_frames)

    def frames(self):
        """(frames [n, rows, cols], global step of each frame), oldest first."""
        axis, mx = getattr(self, "_cap", (1, 0))
        i = self.info()
        shape = {0: (i.nz, i.ny), 1: (i.nz, i.nx), 2: (i.ny, i.nx)}[axis]
        out = np.empty((mx,) + shape, np.float32)
        steps = np.empty(max(mx, 1), np.int64)
        n = C.c_int32()
        self._check(library().afd_get_frames(self._h, _ptr(out, C.c_float), out.size, _ptr(steps, C.c_int64),
                                             steps.size, C.byref(n)))
        return out[:n.value], steps[:n.value]

    TIMELINE_KINDS = ("interior_stream", "boundary", "pml_pressure", "pml_aux_x", "pml_aux_y", "pml_aux_z",
                      "source_receiver")

    def set_timeline(self, first, steps):
        """From the next Run on, record the start of the first block and the
        end of the last block of every kernel kind of global steps
        first .. first+steps-1 (device clock)."""
        self._check(library().afd_set_timeline(self._h, first, steps))
        self._tl_steps = max(int(steps), 0)

    def timeline(self):
        """[steps, len(TIMELINE_KINDS), 2] (start, end) in microseconds from
        the earliest recorded start; NaN where a kind did not run."""
        n_max = getattr(self, "_tl_steps", 0)
        out = np.empty((max(n_max, 1), len(self.TIMELINE_KINDS), 2), np.float64)
        n = C.c_int32()
        self._check(library().afd_get_timeline(self._h, _ptr(out, C.c_double), out.size, C.byref(n)))
        t = out[:n.value] / 1e3
        t[out[:n.value] < 0] = np.nan
        return t

    def energy(self, batch=0):
        e = C.c_double()
        self._check(library().afd_energy(self._h, batch, C.byref(e)))
        return e.value

    def set_stream(self, stream_handle):
        self._check(library().afd_set_stream(self._h, C.c_void_p(stream_handle)))

    def set_plan(self, tile=(0, 0), per_sm=0, dz=0, beside=False, tail=False, auto=False):
        """Fixes the streaming kernel's plan (tile in cells, resident blocks
        per SM, z-chunk depth, boundary/PML kernels beside it or in its tail
        warps) and turns the online autotuner off; auto=True gives the
        choice back to it."""
        if auto:
            self._check(library().afd_set_plan(self._h, None))
            return
        p = Plan(tile[0], tile[1], per_sm, dz, 1 if beside else 0, 1 if tail else 0)
        self._check(library().afd_set_plan(self._h, C.byref(p)))

    # --- z-slab decomposition ----------------------------------------
    def set_slab(self, z_offset, nz_global):
        """This grid is global planes z_offset.. of nz_global planes; its end
        planes are halos filled between step phases (nz_global 0: off)."""
        self._check(library().afd_set_slab(self._h, z_offset, nz_global))

    def step_phase(self, phase):
        """Phase 1 (interior, boundary, PML pressure) or phase 2 (PML
        auxiliary fields, sources, receivers) of the next step."""
        self._check(library().afd_step_phase(self._h, phase))

    def halo(self, side, direction, field, dev_ptr, cap):
        """Plane copy between the simulation and a device buffer (afd_halo):
        side 0/1 low/high z, direction 0 read own plane / 1 write halo,
        field 0 pressure, 1..3 auxiliary x/y/z, 4 psi."""
        self._check(library().afd_halo(self._h, side, direction, field, C.c_void_p(dev_ptr), cap))

    def kernel_stats(self):
        L = library()
        out = {}
        buf = C.create_string_buffer(64)
        k = 0
        while True:
            n, ms = C.c_int64(), C.c_double()
            if L.afd_kernel_stats(self._h, k, buf, 64, C.byref(n), C.byref(ms)) != OK:
                break
            out[buf.value.decode()] = (n.value, ms.value)
            k += 1
        return out

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.afd_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
