"""Shared test helpers: build the same workload for the CUDA library and for the oracle."""
from __future__ import annotations

import numpy as np


def oracle_inputs(O, w, line_e=None):
    """(Params, Centerlines) of workload `w` drawn with the oracle's own generator: one stream
    numbered across the levels, or (w.level_streams) one stream per level."""
    from fastweavturb_b200.configs import level_seed

    xyz, signs = [], []
    t = 0
    for lv, L in enumerate(w.levels):
        for k in range(L.tubes):
            if w.level_streams:
                s = level_seed(w.seed, lv)
                xyz.append(O.fbb_tube(s, k, L.nodes, L.H, L.dB))
                signs.append(O.fbb_sign(s, k))
            else:
                xyz.append(O.fbb_tube(w.seed, t, L.nodes, L.H, L.dB))
                signs.append(O.fbb_sign(w.seed, t))
            t += 1
    xyz = np.concatenate(xyz)
    signs = np.array(signs)
    npoint, sig, gam, nT = w.line_arrays(signs)
    p = O.Params(N=w.N, N_downsample=w.N, line_s=1, line_e=line_e or w.ntubes, sigma_ratio=w.sigma_ratio,
                 eta_t=w.eta_t, ntf_times=w.ntf_times, ntf_pre=w.ntf_pre, Rtube_ratio=w.Rtube_ratio,
                 dzeta_sup=w.dzeta_sup, sigma=sig, Gamma=gam, n_T=nT, if_filter=np.zeros(len(npoint), dtype=np.int32))
    return p, O.Centerlines(npoint=npoint, xyz=xyz)


def gpu_params(F, w, precision=32, deposit_mode=0, **kw):
    a = dict(N=w.N, N_downsample=w.N, line_s=1, line_e=w.ntubes, sigma_ratio=w.sigma_ratio, eta_t=w.eta_t,
             ntf_times=w.ntf_times, ntf_pre=w.ntf_pre, Rtube_ratio=w.Rtube_ratio, dzeta_sup=w.dzeta_sup,
             precision=precision, deposit_mode=deposit_mode)
    a.update(kw)
    return F.Params(**a)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def two_tubes(O, N=24, seed=4):
    """Two closed fBb tubes of different core size and sign on an N^3 grid (oracle inputs)."""
    xyz = np.concatenate([O.fbb_tube(seed, 0, 96, 0.7, 0.5), O.fbb_tube(seed, 1, 128, 0.6, 0.3)])
    p = O.Params(N=N, N_downsample=N, line_s=1, line_e=2, sigma_ratio=1.0, sigma=np.array([0.3, 0.17]),
                 Gamma=np.array([1.0, -0.6]), n_T=np.array([1, 1], dtype=np.int32),
                 if_filter=np.zeros(2, dtype=np.int32))
    return p, O.Centerlines(npoint=np.array([96, 128], dtype=np.int64), xyz=xyz)


def sp_close(sp, sp_ref, q, rtol):
    """S_{q+1}(r) against a reference: |a - b| <= rtol max(|b|, s), s = (max_r S_2)^((q+1)/2) the
    natural size of |du|^(q+1).  Odd orders change sign and pass through zero, where a purely
    relative bound would demand agreement far below the rounding of the sum."""
    sp = np.asarray(sp, dtype=np.float64)
    sp_ref = np.asarray(sp_ref, dtype=np.float64)
    s = float(np.max(np.abs(sp_ref[1]))) ** ((q + 1) / 2.0)
    a, b = sp[q], sp_ref[q]
    bound = rtol * np.maximum(np.abs(b), s)
    bad = np.abs(a - b) > bound
    assert not bad.any(), f"S_{q + 1}: {a[bad]} vs {b[bad]} (bound {bound[bad]})"


def fp64_floor(O, p, cl, **kw):
    """The reference algorithm's own FP64 rounding floor on a workload: the relative L2 distance
    between the oracle's plain build and its FMA-contracted build (oracle.lib_fma), or None on a
    host without FMA.  Returns (floor, plain deposit)."""
    a, _ = O.deposit(p, cl, **kw)
    if not O.has_fma():
        return None, a
    b, _ = O.deposit(p, cl, contracted=True, **kw)
    return rel_l2(b, a), a


def tol64(floor):
    """FP64 tolerance against the oracle: four times the reference's own rounding floor
    (fp64_floor), and never below 1e-12; 5e-11 where the floor cannot be measured."""
    return 5e-11 if floor is None else max(1e-12, 4.0 * floor)
