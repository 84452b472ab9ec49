"""Troubled-cell indicator network (fin_mlp_* of the C ABI).

A 20 -> 32 -> 32 -> 1 GELU network with BF16 weights and activations and FP32
accumulation, trained and run on tcgen05 tensor cores.  Its inputs are the
5-point undivided differences of the four characteristic fields at a face,
each normalised by its local maximum; its label is whether FINESS's own
WENO5-JS weights at that face depart from the linear weights
(max_k |w_k - d_k| / d_k > 0.1, lib/WenoReconstruct.cpp:104,131-134).
"""
import ctypes as C
import os

import numpy as np

from .solver import FinError, load_library

NIN = 20
_HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(_HERE, "data", "indicator_weights.npz")
# the same network trained on ideal-MHD faces (finess_b200/mhd.py's hybrid form)
DEFAULT_MHD_WEIGHTS = os.path.join(_HERE, "data", "indicator_mhd_weights.npz")


def _lib():
    lib = load_library()
    if not getattr(lib, "_mlp_bound", False):
        vp = C.c_void_p
        fp = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        u8 = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
        lib.fin_mlp_nparam.restype = C.c_int
        lib.fin_mlp_last_error.restype = C.c_char_p
        lib.fin_mlp_create.argtypes = [C.c_void_p, C.c_ulonglong, C.POINTER(vp)]
        lib.fin_mlp_destroy.argtypes = [vp]
        lib.fin_mlp_get_params.argtypes = [vp, fp]
        lib.fin_mlp_set_params.argtypes = [vp, fp]
        lib.fin_mlp_forward.argtypes = [vp, fp, C.c_longlong, fp]
        lib.fin_mlp_gradients.argtypes = [vp, fp, u8, C.c_longlong, C.c_float, fp, C.POINTER(C.c_float)]
        lib.fin_mlp_train.argtypes = [vp, fp, u8, C.c_longlong, C.c_int, C.c_int, C.c_float, C.c_float,
                                      C.c_ulonglong, fp]
        for n in ("fin_mlp_create", "fin_mlp_destroy", "fin_mlp_get_params", "fin_mlp_set_params",
                  "fin_mlp_forward", "fin_mlp_gradients", "fin_mlp_train"):
            getattr(lib, n).restype = C.c_int
        lib._mlp_bound = True
    return lib


def _check(lib, rc):
    if rc != 0:
        raise FinError(rc, lib.fin_mlp_last_error().decode())


class MLP:
    def __init__(self, params=None, seed=0):
        self.lib = _lib()
        self.nparam = self.lib.fin_mlp_nparam()
        h = C.c_void_p()
        if params is None:
            _check(self.lib, self.lib.fin_mlp_create(None, seed, C.byref(h)))
        else:
            p = np.ascontiguousarray(params, dtype=np.float32)
            assert p.size == self.nparam
            _check(self.lib, self.lib.fin_mlp_create(p.ctypes.data_as(C.c_void_p), seed, C.byref(h)))
        self.h = h

    @classmethod
    def load(cls, path=DEFAULT_WEIGHTS):
        return cls(params=np.load(path)["params"])

    def close(self):
        if getattr(self, "h", None):
            self.lib.fin_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self):
        out = np.zeros(self.nparam, dtype=np.float32)
        _check(self.lib, self.lib.fin_mlp_get_params(self.h, out))
        return out

    @params.setter
    def params(self, p):
        _check(self.lib, self.lib.fin_mlp_set_params(self.h, np.ascontiguousarray(p, dtype=np.float32)))

    def forward(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        z = np.zeros(X.shape[0], dtype=np.float32)
        _check(self.lib, self.lib.fin_mlp_forward(self.h, X, X.shape[0], z))
        return z

    def gradients(self, X, y, pos_weight=1.0):
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.uint8)
        g = np.zeros(self.nparam, dtype=np.float32)
        loss = C.c_float()
        _check(self.lib, self.lib.fin_mlp_gradients(self.h, X, y, X.shape[0], pos_weight, g, C.byref(loss)))
        return g, loss.value

    def train(self, X, y, epochs=5, batch=4096, lr=3e-3, pos_weight=1.0, seed=0):
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.uint8)
        losses = np.zeros(epochs, dtype=np.float32)
        _check(self.lib, self.lib.fin_mlp_train(self.h, X, y, X.shape[0], epochs, batch, lr, pos_weight, seed,
                                                losses))
        return losses
