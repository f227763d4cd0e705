"""ctypes binding of include/afd_surrogate.h: the learned impulse-response
surrogate (Fourier-feature MLP on tcgen05 BF16 GEMMs) and its raw GEMM.

The surrogate has no counterpart in the reference. The workflow around it
(training data from the batched FDTD engine, decimation to 8 kHz, error
prediction and FDTD fallback) is in surrogate_workflow.py.
"""
import ctypes as C

import numpy as np

from . import afd

WEIGHT, BIAS, GRAD_WEIGHT, GRAD_BIAS, FOURIER, FEATURES = 0, 1, 2, 3, 4, 5

EXPORTS = ["afd_mlp_default_params", "afd_mlp_create", "afd_mlp_destroy", "afd_mlp_last_error",
           "afd_mlp_set_stream", "afd_mlp_train_step", "afd_mlp_gradients", "afd_mlp_predict", "afd_mlp_sync",
           "afd_mlp_get", "afd_mlp_set_weights", "afd_gemm_bf16", "afd_gemm_bf16_async"]


class MlpParams(C.Structure):
    _fields_ = [("n_in", C.c_int32), ("n_freq", C.c_int32), ("hidden", C.c_int32), ("n_layers", C.c_int32),
                ("n_out", C.c_int32), ("batch", C.c_int32), ("device", C.c_int32), ("fourier_sigma", C.c_float),
                ("seed", C.c_uint64), ("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float),
                ("eps", C.c_float), ("reserved", C.c_int32 * 8)]


_bound = False


def _lib():
    global _bound
    L = afd.library()
    if not _bound:
        P, vp, i32, i64, f32 = C.POINTER, C.c_void_p, C.c_int32, C.c_int64, C.c_float
        sig = {
            "afd_mlp_default_params": (None, [P(MlpParams)]),
            "afd_mlp_create": (C.c_int, [P(vp), P(MlpParams)]),
            "afd_mlp_destroy": (None, [vp]),
            "afd_mlp_last_error": (C.c_char_p, [vp]),
            "afd_mlp_set_stream": (C.c_int, [vp, vp]),
            "afd_mlp_train_step": (C.c_int, [vp, vp, vp, i32, P(f32)]),
            "afd_mlp_gradients": (C.c_int, [vp, vp, vp, i32, P(f32)]),
            "afd_mlp_predict": (C.c_int, [vp, vp, i32, vp]),
            "afd_mlp_sync": (C.c_int, [vp]),
            "afd_mlp_get": (C.c_int, [vp, i32, i32, P(f32), i64]),
            "afd_mlp_set_weights": (C.c_int, [vp, i32, P(f32), P(f32)]),
            "afd_gemm_bf16": (C.c_int, [vp, vp, vp, i32, i32, i32, vp]),
            "afd_gemm_bf16_async": (C.c_int, [vp, vp, vp, i32, i32, i32, vp, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _bound = True
    return L


def default_params(**kw):
    p = MlpParams()
    _lib().afd_mlp_default_params(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def _addr(a):
    """Address of a numpy array (host) or of a torch tensor (device)."""
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return C.c_void_p(a.ctypes.data)


class Mlp:
    """The surrogate network on one GPU. Inputs may be numpy float32 arrays
    or contiguous float32 torch tensors on the device."""

    def __init__(self, params=None, **kw):
        L = _lib()
        self.params = params if params is not None else default_params(**kw)
        h = C.c_void_p()
        st = L.afd_mlp_create(C.byref(h), C.byref(self.params))
        if st != afd.OK:
            raise afd.AfdError(st, L.afd_mlp_last_error(None).decode())
        self._h = h

    def _check(self, st):
        if st != afd.OK:
            raise afd.AfdError(st, _lib().afd_mlp_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            _lib().afd_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        self._check(_lib().afd_mlp_set_stream(self._h, C.c_void_p(stream)))

    @staticmethod
    def _f32(a):
        if hasattr(a, "data_ptr"):
            return a
        return np.ascontiguousarray(a, dtype=np.float32)

    def train_step(self, x, y, want_loss=True):
        x, y = self._f32(x), self._f32(y)
        loss = C.c_float()
        self._check(_lib().afd_mlp_train_step(self._h, _addr(x), _addr(y), int(x.shape[0]),
                                              C.byref(loss) if want_loss else None))
        return loss.value if want_loss else None

    def gradients(self, x, y):
        x, y = self._f32(x), self._f32(y)
        loss = C.c_float()
        self._check(_lib().afd_mlp_gradients(self._h, _addr(x), _addr(y), int(x.shape[0]), C.byref(loss)))
        return loss.value

    def predict(self, x, out=None):
        x = self._f32(x)
        n = int(x.shape[0])
        if out is None:
            out = np.empty((n, self.params.n_out), np.float32)
        self._check(_lib().afd_mlp_predict(self._h, _addr(x), n, _addr(out)))
        return out

    def sync(self):
        self._check(_lib().afd_mlp_sync(self._h))

    def get(self, what, layer=0):
        p = self.params
        F = 2 * p.n_freq
        dims = [F] + [p.hidden] * (p.n_layers - 1) + [p.n_out]
        if what == FOURIER:
            shape = (p.n_in, p.n_freq)
        elif what == FEATURES:
            shape = (p.batch, F)
        elif what in (WEIGHT, GRAD_WEIGHT):
            shape = (dims[layer + 1], dims[layer])
        else:
            shape = (dims[layer + 1],)
        out = np.empty(shape, np.float32)
        self._check(_lib().afd_mlp_get(self._h, what, layer, out.ctypes.data_as(C.POINTER(C.c_float)), out.size))
        return out

    def set_weights(self, layer, w, b):
        w = np.ascontiguousarray(w, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        self._check(_lib().afd_mlp_set_weights(self._h, layer, w.ctypes.data_as(C.POINTER(C.c_float)),
                                               b.ctypes.data_as(C.POINTER(C.c_float))))

    def weights(self):
        return [(self.get(WEIGHT, l), self.get(BIAS, l)) for l in range(self.params.n_layers)]


def gemm_bf16(a, b, c, stream=0):
    """c[M][N] (float32 device tensor) = a[M][K] @ b[N][K]^T, a and b bf16
    device tensors (torch), through the tcgen05 kernel."""
    M, K = a.shape
    N = b.shape[0]
    L = _lib()
    st = L.afd_gemm_bf16(C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), C.c_void_p(c.data_ptr()), M, N, K,
                         C.c_void_p(stream))
    if st != afd.OK:
        raise afd.AfdError(st, L.afd_mlp_last_error(None).decode())
    return c


def gemm_bf16_async(a, b, c, status, stream=0):
    """The same GEMM queued on `stream` without synchronising; a pipeline
    wait that expired ORs 1 into status (an int32 device tensor of one
    element, zeroed by the caller)."""
    M, K = a.shape
    N = b.shape[0]
    L = _lib()
    st = L.afd_gemm_bf16_async(C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), C.c_void_p(c.data_ptr()), M, N,
                               K, C.c_void_p(stream), C.c_void_p(status.data_ptr()))
    if st != afd.OK:
        raise afd.AfdError(st, L.afd_mlp_last_error(None).decode())
    return c
