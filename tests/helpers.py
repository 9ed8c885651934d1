"""Shared test helpers: build the same workload for the CUDA library and for the oracle."""
from __future__ import annotations

import numpy as np


def oracle_inputs(O, w, line_e=None):
    """(Params, Centerlines) of workload `w` drawn with the oracle's own generator."""
    xyz = []
    t = 0
    for L in w.levels:
        for _ in range(L.tubes):
            xyz.append(O.fbb_tube(w.seed, t, L.nodes, L.H, L.dB))
            t += 1
    xyz = np.concatenate(xyz)
    signs = np.array([O.fbb_sign(w.seed, i) for i in range(w.ntubes)])
    npoint, sig, gam, nT = w.line_arrays(signs)
    p = O.Params(N=w.N, N_downsample=w.N, line_s=1, line_e=line_e or w.ntubes, sigma_ratio=w.sigma_ratio,
                 eta_t=w.eta_t, ntf_times=w.ntf_times, ntf_pre=w.ntf_pre, Rtube_ratio=w.Rtube_ratio,
                 dzeta_sup=w.dzeta_sup, sigma=sig, Gamma=gam, n_T=nT, if_filter=np.zeros(len(npoint), dtype=np.int32))
    return p, O.Centerlines(npoint=npoint, xyz=xyz)


def gpu_params(F, w, precision=32, deposit_mode=0, **kw):
    return F.Params(N=w.N, N_downsample=w.N, line_s=1, line_e=w.ntubes, sigma_ratio=w.sigma_ratio, eta_t=w.eta_t,
                    ntf_times=w.ntf_times, ntf_pre=w.ntf_pre, Rtube_ratio=w.Rtube_ratio, dzeta_sup=w.dzeta_sup,
                    precision=precision, deposit_mode=deposit_mode, **kw)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
