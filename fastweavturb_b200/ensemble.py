"""Batched ensembles of woven fields on one GPU, and the autotuner of the deposition kernels.

An ensemble is a list of workloads of uneven grid sizes and parameters (configs.
ensemble_member, configs.surrogate_member).  Ensemble keeps one libfwt context per grid size,
so the FFT plans and device buffers of a size are made once and reused by every realisation
of that size; each realisation's centerlines are generated on the device, the field is built
and its statistics stay on the device until read.

Autotuner: before the first realisation of a grid size, the deposition of a probe
realisation is timed with the chord-piece kernel limit at each candidate value (the tube
radius in grid spacings up to which the piece kernel is used instead of the sub-segment
kernel) and the fastest is kept for the rest of that size.  Both kernels give the same
field within FP32 rounding; only the speed differs.
"""
from __future__ import annotations

import time

import numpy as np

from .api import Context, Params, sp_exponents, sp_separations
from .configs import build_workload

TUNE_CANDIDATES = (0.0, 2.5, 5.0, 8.0)


class Ensemble:
    def __init__(self, device=0, tune=True, Sp_order=6):
        self.device = device
        self.tune = tune
        self.Sp_order = Sp_order
        self.ctx = {}
        self.tuned = {}
        self.tune_log = {}

    def context(self, N):
        if N not in self.ctx:
            self.ctx[N] = Context(Params(N=N, N_downsample=N, line_s=1, line_e=0, sigma_ratio=1.0, device=self.device,
                                         pdf_bins=201, Sp_order=self.Sp_order, vorticity_output=0))
        return self.ctx[N]

    def _load(self, ctx, w):
        return build_workload(ctx, w)

    def autotune(self, w):
        """Time the deposition of workload w for every candidate limit; keep the fastest."""
        import torch
        ctx = self.context(w.N)
        keep = self._load(ctx, w)
        times = {}
        for cells in TUNE_CANDIDATES:
            ctx.set_piece_radius_limit(cells)
            ctx.deposit(1, w.ntubes)        # warm (allocations for this kernel choice)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.deposit(1, w.ntubes)
            torch.cuda.synchronize()
            times[cells] = time.perf_counter() - t0
        best = min(times, key=times.get)
        ctx.set_piece_radius_limit(best)
        self.tuned[w.N] = best
        self.tune_log[w.N] = times
        del keep
        return best

    def run(self, members, stats=True):
        """Build every member; returns (per-member statistics, device seconds, Mpts/s)."""
        import torch
        out = []
        t_total = 0.0
        for w in members:
            ctx = self.context(w.N)
            if self.tune and w.N not in self.tuned:
                self.autotune(w)
            xyz = self._load(ctx, w)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.run()
            torch.cuda.synchronize()
            t_total += time.perf_counter() - t0
            out.append(member_statistics(ctx, w.N, self.Sp_order) if stats else None)
            del xyz
        pts = sum(w.N ** 3 for w in members)
        return out, t_total, pts / t_total / 1e6

    def close(self):
        for c in self.ctx.values():
            c.close()
        self.ctx = {}


def member_statistics(ctx, N, Sp_order=6):
    """E(k) of u (after normalisation), S_p at the reference separations, zeta_p and flatness."""
    s = ctx.cal_helicity()
    Ek = ctx.spectrum(1)
    r, Sp = ctx.Sp_calculate(pmax=max(Sp_order, 4))
    rdr = r * (2 * np.pi / N)
    zeta, flat = sp_exponents(rdr, Sp) if len(r) >= 10 else (np.full(Sp.shape[0], np.nan), Sp[3] / Sp[1] ** 2)
    return {"Ek": Ek, "r": r, "Sp": Sp, "zeta": zeta, "flat": flat, "up": s["up"], "Etot": s["Etot"]}
