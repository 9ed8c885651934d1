"""The learned surrogate: generator parameters -> output statistics, and the inverse fit.

The network (a multilayer perceptron on the tensor cores, libfwt's fwt_mlp_*) maps the five
generator parameters of an ensemble realisation -- Hurst exponent H, core-size ratio
sigma_max / sigma_min, density multiplier, number of levels and circulation exponent -- to
45 statistics of the woven field: log E(k) on 32 log-spaced wavenumbers, the flatness
S_4 / S_2^2 at 8 separations and the scaling exponents zeta_2 .. zeta_6.  It is trained on
realisations the generator itself produces (fastweavturb_b200.configs.surrogate_member) and
drives an inverse fit of the parameters to a target set of statistics, with the generator as
the judge of the result and as the fallback.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from .api import Context, FwtError, Params, _check, _ptr, library, sp_exponents, sp_separations

N_IN, N_OUT = 5, 45
PARAM_LO = np.array([0.3, 2.0, 0.5, 2.0, 1.2])    # H, sigma ratio, density, levels, Gamma exponent
PARAM_HI = np.array([0.8, 8.0, 4.0, 4.0, 1.5])


def _lib():
    L = library()
    if not getattr(L, "_mlp_bound", False):
        vp, ip, fp, dp = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)
        L.fwt_mlp_create.argtypes = [ip, ip, ip, ip, ip, ip, ctypes.c_uint64, ctypes.POINTER(vp)]
        L.fwt_mlp_destroy.argtypes = [vp]
        L.fwt_mlp_nparams.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.fwt_mlp_get_params.argtypes = [vp, fp]
        L.fwt_mlp_set_params.argtypes = [vp, fp]
        L.fwt_mlp_forward.argtypes = [vp, fp, ip, fp]
        L.fwt_mlp_loss_grad.argtypes = [vp, fp, fp, fp, ip, dp, fp, fp]
        L.fwt_mlp_train_step.argtypes = [vp, fp, fp, fp, ip, ctypes.c_float, dp]
        L.fwt_gemm_bf16.argtypes = [vp, vp, vp, ip, ip, ip, ip, vp]
        for n in ("fwt_mlp_create", "fwt_mlp_destroy", "fwt_mlp_nparams", "fwt_mlp_get_params", "fwt_mlp_set_params",
                  "fwt_mlp_forward", "fwt_mlp_loss_grad", "fwt_mlp_train_step", "fwt_gemm_bf16"):
            getattr(L, n).restype = ctypes.c_int
        L._mlp_bound = True
    return L


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class MLP:
    """The tensor-core perceptron (include/fwt.h, fwt_mlp_*)."""

    def __init__(self, n_in=N_IN, width=256, depth=4, n_out=N_OUT, batch_max=4096, seed=0, device=0):
        self.widths = [n_in] + [width] * depth + [n_out]
        self.batch_max = batch_max
        self._h = ctypes.c_void_p()
        _check(_lib().fwt_mlp_create(device, n_in, width, depth, n_out, batch_max, seed, ctypes.byref(self._h)))
        n = ctypes.c_int64()
        _check(_lib().fwt_mlp_nparams(self._h, ctypes.byref(n)))
        self.nparams = n.value

    def close(self):
        if self._h:
            _lib().fwt_mlp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        out = np.zeros(self.nparams, dtype=np.float32)
        _check(_lib().fwt_mlp_get_params(self._h, _ptr(out, ctypes.c_float)))
        return out

    def set_params(self, p):
        p = _f32(p)
        _check(_lib().fwt_mlp_set_params(self._h, _ptr(p, ctypes.c_float)))

    def forward(self, x):
        x = _f32(x)
        y = np.zeros((x.shape[0], self.widths[-1]), dtype=np.float32)
        _check(_lib().fwt_mlp_forward(self._h, _ptr(x, ctypes.c_float), x.shape[0], _ptr(y, ctypes.c_float)))
        return y

    def loss_grad(self, x, t, w_out=None, params=True, inputs=True):
        x, t = _f32(x), _f32(t)
        w = None if w_out is None else _f32(w_out)
        loss = ctypes.c_double()
        gp = np.zeros(self.nparams, dtype=np.float32) if params else None
        gx = np.zeros_like(x) if inputs else None
        _check(_lib().fwt_mlp_loss_grad(self._h, _ptr(x, ctypes.c_float), _ptr(t, ctypes.c_float),
                                        None if w is None else _ptr(w, ctypes.c_float), x.shape[0],
                                        ctypes.byref(loss), None if gp is None else _ptr(gp, ctypes.c_float),
                                        None if gx is None else _ptr(gx, ctypes.c_float)))
        return loss.value, gp, gx

    def train_step(self, x, t, lr, w_out=None):
        x, t = _f32(x), _f32(t)
        w = None if w_out is None else _f32(w_out)
        loss = ctypes.c_double()
        _check(_lib().fwt_mlp_train_step(self._h, _ptr(x, ctypes.c_float), _ptr(t, ctypes.c_float),
                                         None if w is None else _ptr(w, ctypes.c_float), x.shape[0],
                                         ctypes.c_float(lr), ctypes.byref(loss)))
        return loss.value


def gemm_bf16(A_dev, B_dev, C_dev, M, N, K, ldc=None, stream=None):
    """C = A . B^T on the tensor cores for device pointers (BF16 A, B; FP32 C)."""
    _check(_lib().fwt_gemm_bf16(A_dev, B_dev, C_dev, M, N, K, ldc or N, stream))
