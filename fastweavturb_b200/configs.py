"""Synthetic woven-field workloads (the shapes the benchmark and tests run on).

A workload is a set of scale levels; level l holds ``tubes`` closed fractional-Brownian-bridge
centerlines of ``nodes`` nodes with core size ``sigma``, circulation magnitude ``Gamma`` and
rms node step ``dB``.  No public dataset exists for this path; every workload is drawn from
its seed (Philox streams, see csrc/k_fbb.cu).

Named workloads (grid N, levels, sigma_l, tubes n_l, nodes per tube, H):

* ``cfg0``  64^3,   l = 0..2, sigma_l = 0.3*2^-l, n_l = 4*4^l, 256*2^l nodes, H = 0.7
* ``cfg1``  256^3,  l = 0..5, sigma_l = 0.4*2^-l, n_l = 4*4^l, 256*2^l nodes, H = 0.7
* ``cfg2``  1024^3, l = 0..7, sigma_l = 0.5*2^-l, n_l = 2*4^l, 256*2^l nodes, H = 0.7
* ``ensemble``: realisations with N in {64, 96, 128, 192, 256}, H ~ U[0.3, 0.8], 3..6 levels,
  density multiplier ~ U[0.5, 4] on n_l = 4*4^l, circulation exponent ~ U[1.2, 1.5]

Circulation: Gamma_l = +-(sigma_l/sigma_0)^e with a random sign per tube (e = 4/3 unless
drawn).  The core is constant along each tube (sigma_ratio = 1), eta = 0, Rtube_ratio = 3,
ntf_times = 50, ntf_pre = 1000, dzeta_sup = 1e-4.

Node step: dB_l = 10 sigma_l.  The reference generator uses dB = c_B * sigma_min with
c_B = 40 and sigma_max = 4 sigma_min (FBB_with_parameters.m:14-15,35-36), so its node step is
10 sigma_max and its step-to-truncation-radius ratio dB / (3 sigma_max) is 10/3; with a
constant core (sigma_max = sigma) the same geometry is dB = 10 sigma.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

C_B_EFF = 10.0


@dataclass
class Level:
    tubes: int
    nodes: int
    sigma: float
    Gamma: float
    H: float
    dB: float


@dataclass
class Workload:
    name: str
    N: int
    levels: list
    seed: int = 0
    sigma_ratio: float = 1.0
    eta_t: float = 0.0
    ntf_times: int = 50
    ntf_pre: int = 1000
    Rtube_ratio: float = 3.0
    dzeta_sup: float = 1e-4
    # True: each level draws its tubes from its own stream (seed, level), so a level's tube
    # count changes only that level's last tubes; False: one stream numbered across levels
    level_streams: bool = False
    extra: dict = field(default_factory=dict)

    @property
    def ntubes(self):
        return sum(l.tubes for l in self.levels)

    @property
    def nnodes(self):
        return sum(l.tubes * l.nodes for l in self.levels)

    def line_arrays(self, signs):
        """Per-line npoint, sigma, Gamma (signed), n_T for tube order level by level."""
        npoint, sig, gam = [], [], []
        t = 0
        for L in self.levels:
            for _ in range(L.tubes):
                npoint.append(L.nodes)
                sig.append(L.sigma)
                gam.append(L.Gamma * signs[t])
                t += 1
        n = len(npoint)
        return (np.array(npoint, dtype=np.int64), np.array(sig), np.array(gam), np.ones(n, dtype=np.int32))

    def gen_arrays(self):
        return ([L.tubes for L in self.levels], [L.nodes for L in self.levels], [L.H for L in self.levels],
                [L.dB for L in self.levels])


def _levels(nlev, sigma0, tubes0, nodes0, H, gexp=4.0 / 3.0, density=1.0):
    out = []
    for l in range(nlev):
        s = sigma0 * 2.0 ** (-l)
        out.append(Level(tubes=max(1, int(round(density * tubes0 * 4 ** l))), nodes=nodes0 * 2 ** l, sigma=s,
                         Gamma=(s / sigma0) ** gexp, H=H, dB=C_B_EFF * s))
    return out


def cfg0(seed=0):
    return Workload("cfg0: 64^3, 3 levels, sigma_l=0.3*2^-l, n_l=4*4^l, 256*2^l nodes, H=0.7", 64,
                    _levels(3, 0.3, 4, 256, 0.7), seed=seed)


def cfg1(seed=0):
    return Workload("cfg1: 256^3, 6 levels, sigma_l=0.4*2^-l, n_l=4*4^l, 256*2^l nodes, H=0.7", 256,
                    _levels(6, 0.4, 4, 256, 0.7), seed=seed)


def cfg2(seed=0):
    return Workload("cfg2: 1024^3, 8 levels, sigma_l=0.5*2^-l, n_l=2*4^l, 256*2^l nodes, H=0.7", 1024,
                    _levels(8, 0.5, 2, 256, 0.7), seed=seed)


def ensemble_member(seed, N=None, rng=None):
    """One realisation of the batched ensemble: parameters drawn from `seed`."""
    rng = rng or np.random.default_rng(seed)
    if N is None:
        N = int(rng.choice([64, 96, 128, 192, 256]))
    H = float(rng.uniform(0.3, 0.8))
    nlev = int(rng.integers(3, 7))
    dens = float(rng.uniform(0.5, 4.0))
    gexp = float(rng.uniform(1.2, 1.5))
    w = Workload(f"ensemble member seed={seed}: N={N}, H={H:.3f}, levels={nlev}, density={dens:.2f}, "
                 f"Gamma exponent={gexp:.3f}", N, _levels(nlev, 0.4, 4, 256, H, gexp=gexp, density=dens), seed=seed)
    w.extra = {"H": H, "levels": nlev, "density": dens, "gexp": gexp, "sigma_ratio_levels": 2.0 ** (nlev - 1)}
    w.level_streams = True
    return w


def surrogate_member(params, seed, N=64):
    """A realisation for the learned surrogate from its five inputs (H, sigma_max/sigma_min,
    density multiplier, levels, circulation exponent): the ensemble family of
    ensemble_member with 64 * 2^l nodes per tube (a quarter of the benchmark's, so thousands
    of realisations fit the training budget) and sigma_max/sigma_min = 2^(levels - 1).  Its
    levels draw from separate streams, so with the seed fixed the statistics change gradually
    with the density (tubes are added or removed at the end of a level) and continuously with
    H and the circulation exponent."""
    H, _, dens, nlev, gexp = params
    nlev = int(round(nlev))
    w = Workload(f"surrogate member seed={seed}: N={N}, H={H:.3f}, levels={nlev}, density={dens:.2f}, "
                 f"Gamma exponent={gexp:.3f}", N, _levels(nlev, 0.4, 4, 64, float(H), gexp=float(gexp),
                                                           density=float(dens)), seed=seed)
    w.extra = {"H": H, "levels": nlev, "density": dens, "gexp": gexp, "sigma_ratio_levels": 2.0 ** (nlev - 1)}
    w.level_streams = True
    return w


def small(N=32, seed=1, nlev=2, tubes0=2, nodes0=64, sigma0=0.4, H=0.7):
    """A small workload for parity tests (the FP64 oracle finishes it in seconds)."""
    return Workload(f"small: {N}^3, {nlev} levels", N, _levels(nlev, sigma0, tubes0, nodes0, H), seed=seed)


CONFIGS = {"cfg0": cfg0, "cfg1": cfg1, "cfg2": cfg2}


def level_seed(seed, level):
    """Seed of one level's stream (level_streams workloads): a 64-bit mix of both."""
    return (seed * 0x9E3779B97F4A7C15 + (level + 1) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF


def build_workload(ctx, w: Workload):
    """Generate the workload's centerlines on the context's GPU and set them as its input.

    Returns the torch tensors holding the node coordinates (they must outlive the context's
    use of them) and the per-line arrays."""
    import torch

    from .api import fbb_signs

    dev = torch.device("cuda", ctx.params.device)
    n = w.nnodes
    xyz = torch.empty((3, n), dtype=torch.float64, device=dev)
    tubes, nodes, H, dB = w.gen_arrays()
    if w.level_streams:
        off, signs = 0, []
        for l in range(len(tubes)):
            s = level_seed(w.seed, l)
            if tubes[l] > 0:
                ctx.fbb_generate(s, tubes[l:l + 1], nodes[l:l + 1], H[l:l + 1], dB[l:l + 1],
                                 xyz[0, off:].data_ptr(), xyz[1, off:].data_ptr(), xyz[2, off:].data_ptr())
                signs.append(fbb_signs(s, int(tubes[l])))
            off += int(tubes[l]) * int(nodes[l])
        signs = np.concatenate(signs) if signs else np.zeros(0, dtype=np.int32)
    else:
        ctx.fbb_generate(w.seed, tubes, nodes, H, dB, xyz[0].data_ptr(), xyz[1].data_ptr(), xyz[2].data_ptr())
        signs = fbb_signs(w.seed, w.ntubes)
    npoint, sig, gam, nT = w.line_arrays(signs)
    ctx.set_centerlines_device(npoint, xyz[0].data_ptr(), xyz[1].data_ptr(), xyz[2].data_ptr(), sig, gam, nT)
    return xyz, (npoint, sig, gam, nT)
