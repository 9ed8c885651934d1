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

from .api import _check, _ptr, library

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


# ------------------------------------------------------------------------------ statistics
N_SHELLS, N_FLAT = 32, 8


def features(st, N):
    """The 45 statistics of one realisation: log E(k) at 32 log-spaced wavenumbers in
    [1, N/2] (linear in log-log between shells), the flatness at the first 8 distinct
    separations of the reference's S_p grid and zeta_2 .. zeta_6."""
    Ek = np.maximum(np.asarray(st["Ek"], dtype=np.float64), 1e-300)
    k = np.arange(1, len(Ek) + 1, dtype=np.float64)
    kq = np.exp(np.linspace(0.0, np.log(N / 2), N_SHELLS))
    logE = np.interp(np.log(kq), np.log(k), np.log(Ek))
    r = np.asarray(st["r"])
    rows = [0] + [i for i in range(1, len(r)) if r[i] != r[i - 1]]
    flat = np.asarray(st["flat"])[rows[:N_FLAT]]
    zeta = np.asarray(st["zeta"])[1:6]
    return np.concatenate([logE, flat, zeta])


def fit_error(y, y_target):
    """(mean |d log E|, mean relative flatness error): the fit is within 2 % when both <= 0.02."""
    y, t = np.asarray(y), np.asarray(y_target)
    eE = float(np.mean(np.abs(y[:N_SHELLS] - t[:N_SHELLS])))
    eF = float(np.mean(np.abs(y[N_SHELLS:N_SHELLS + N_FLAT] - t[N_SHELLS:N_SHELLS + N_FLAT]) /
                       np.abs(t[N_SHELLS:N_SHELLS + N_FLAT])))
    return eE, eF


def draw_params(rng, n):
    """n parameter draws of the ensemble family: H ~ U[0.3, 0.8], levels in {2, 3, 4},
    sigma ratio 2^(levels-1), density ~ U[0.5, 4], circulation exponent ~ U[1.2, 1.5]."""
    lev = rng.integers(2, 5, n).astype(np.float64)
    return np.stack([rng.uniform(0.3, 0.8, n), 2.0 ** (lev - 1), rng.uniform(0.5, 4.0, n), lev,
                     rng.uniform(1.2, 1.5, n)], axis=1)


def generate(P, seeds, N=64, ens=None):
    """Statistics of one realisation per parameter row, by the batched generator."""
    from .configs import surrogate_member
    from .ensemble import Ensemble
    own = ens is None
    ens = ens or Ensemble()
    members = [surrogate_member(p, int(s), N=N) for p, s in zip(P, seeds)]
    stats, secs, rate = ens.run(members)
    Y = np.stack([features(s, N) for s in stats])
    if own:
        ens.close()
    return Y, secs


class Surrogate:
    """The network with its input scaling (to [-1, 1] over the parameter box) and output
    standardisation (training-set mean and deviation)."""

    def __init__(self, width=256, depth=4, seed=0, batch_max=4096):
        self.net = MLP(N_IN, width, depth, N_OUT, batch_max=batch_max, seed=seed)
        self.ymu = np.zeros(N_OUT)
        self.ysd = np.ones(N_OUT)

    @staticmethod
    def xin(P):
        return 2.0 * (np.asarray(P) - PARAM_LO) / (PARAM_HI - PARAM_LO) - 1.0

    def fit(self, P, Y, steps=3000, batch=256, lr=1e-3, seed=0):
        rng = np.random.default_rng(seed)
        self.ymu = Y.mean(axis=0)
        self.ysd = Y.std(axis=0) + 1e-9
        X = self.xin(P)
        T = (Y - self.ymu) / self.ysd
        losses = []
        for s in range(steps):
            idx = rng.choice(len(X), size=min(batch, len(X)), replace=False)
            lr_s = lr * (0.1 ** (s / steps))          # exponential decay to lr/10
            losses.append(self.net.train_step(X[idx], T[idx], lr_s))
        return np.array(losses)

    def predict(self, P):
        return self.net.forward(self.xin(P)) * self.ysd + self.ymu

    def close(self):
        self.net.close()


def inverse_fit(sur, y_target, starts=64, iters=200, lr=0.05, seed=0):
    """Parameters whose predicted statistics best match y_target (spectrum and flatness):
    Adam on the network's input gradient from `starts` random starts for each level count,
    all level counts in one batch (levels and the sigma ratio held at their discrete values);
    returns the best predicted parameters of each level count, best first."""
    rng = np.random.default_rng(seed)
    w = np.zeros(N_OUT)
    w[:N_SHELLS + N_FLAT] = 1.0                    # fit the spectrum and the flatness
    t = (np.asarray(y_target) - sur.ymu) / sur.ysd
    levels = (2.0, 3.0, 4.0)
    P = draw_params(rng, starts * len(levels))
    P[:, 3] = np.repeat(levels, starts)
    P[:, 1] = 2.0 ** (P[:, 3] - 1)
    X = Surrogate.xin(P).astype(np.float32)
    m1 = np.zeros_like(X)
    m2 = np.zeros_like(X)
    free = np.array([1, 0, 1, 0, 1], dtype=np.float32)   # H, density, Gamma exponent
    T = np.repeat(t[None, :], len(X), axis=0).astype(np.float32)
    for it in range(1, iters + 1):
        _, _, gx = sur.net.loss_grad(X, T, w_out=w, params=False, inputs=True)
        g = gx * free
        m1 = 0.9 * m1 + 0.1 * g
        m2 = 0.999 * m2 + 0.001 * g * g
        X -= lr * (m1 / (1 - 0.9 ** it)) / (np.sqrt(m2 / (1 - 0.999 ** it)) + 1e-8)
        X = np.clip(X, -1.0, 1.0)
    Y = sur.net.forward(X) * sur.ysd + sur.ymu
    err = np.array([sum(fit_error(y, y_target)) for y in Y])
    best = []
    for j, lev in enumerate(levels):
        i = j * starts + int(np.argmin(err[j * starts:(j + 1) * starts]))
        Pfit = (X[i] + 1.0) / 2.0 * (PARAM_HI - PARAM_LO) + PARAM_LO
        Pfit[3], Pfit[1] = lev, 2.0 ** (lev - 1)
        best.append((err[i], Pfit))
    best.sort(key=lambda b: b[0])
    return [b[1] for b in best]


def within(e, tol=0.02):
    """A fit is within tol when both its spectrum and its flatness error are."""
    return max(e) <= tol


def refine_with_generator(cands, y_target, seed_eval, runs, N=64, ens=None, seed=5, rounds_per_shrink=2,
                          tol=None, t0=None):
    """Generator-judged search from starting candidates: the candidates are run, then the
    remaining runs perturb the best one's continuous parameters (H, density, circulation
    exponent; the level count stays) in batches of 4 with a radius that shrinks by 0.7 every
    `rounds_per_shrink` batches, keeping improvements.  With `tol`, the search stops as soon
    as the best fit is within tol.  Returns (params, (errE, errF), runs, trace) where trace
    lists (runs, seconds since t0, best errE + errF, within tol) after every batch."""
    t0 = time.perf_counter() if t0 is None else t0
    rng = np.random.default_rng(seed)
    P = np.array(cands, dtype=np.float64)
    Y, _ = generate(P, [seed_eval] * len(P), N=N, ens=ens)
    fe = [fit_error(y, y_target) for y in Y]
    i = int(np.argmin([sum(e) for e in fe]))
    best, best_fe, best_y = P[i].copy(), fe[i], Y[i]
    used = len(P)
    trace = [(used, time.perf_counter() - t0, sum(best_fe), within(best_fe, tol or 0.02))]
    span = PARAM_HI - PARAM_LO
    radius, rnd = 0.15, 0
    while used < runs and not (tol is not None and within(best_fe, tol)):
        k = min(4, runs - used)
        Q = np.repeat(best[None, :], k, axis=0)
        for j in (0, 2, 4):
            Q[:, j] = np.clip(Q[:, j] + rng.normal(0, radius * span[j], k), PARAM_LO[j], PARAM_HI[j])
        Yq, _ = generate(Q, [seed_eval] * k, N=N, ens=ens)
        used += k
        for q, y in zip(Q, Yq):
            e = fit_error(y, y_target)
            if sum(e) < sum(best_fe):
                best, best_fe, best_y = q.copy(), e, y
        trace.append((used, time.perf_counter() - t0, sum(best_fe), within(best_fe, tol or 0.02)))
        rnd += 1
        if rnd % rounds_per_shrink == 0:
            radius *= 0.7
    return best, best_fe, used, trace


def fit_surrogate_driven(sur, y_target, seed_eval, runs, N=64, ens=None, tol=None):
    """The network's best parameters for each level count start the generator-judged search.
    Returns (params, (errE, errF), seconds, runs, trace); the network's time is in both."""
    t0 = time.perf_counter()
    p, e, used, trace = refine_with_generator(inverse_fit(sur, y_target), y_target, seed_eval, runs, N=N,
                                              ens=ens, tol=tol, t0=t0)
    return p, e, time.perf_counter() - t0, used, trace


def fit_generator_only(y_target, seed_eval, runs, N=64, ens=None, seed=1, tol=None):
    """The method without the network: one random draw per level count starts the same
    generator-judged search."""
    t0 = time.perf_counter()
    P = draw_params(np.random.default_rng(seed), 3)
    P[:, 3] = [2.0, 3.0, 4.0]
    P[:, 1] = 2.0 ** (P[:, 3] - 1)
    p, e, used, trace = refine_with_generator(list(P), y_target, seed_eval, runs, N=N, ens=ens, tol=tol, t0=t0)
    return p, e, time.perf_counter() - t0, used, trace
