"""Batched ensembles of woven fields on one GPU, and the autotuner of the deposition kernels.

An ensemble is a list of workloads of uneven grid sizes and parameters (configs.
ensemble_member, configs.surrogate_member).  Ensemble keeps `workers` libfwt contexts per grid
size, each with its own CUDA stream, so the FFT plans and device buffers of a size are made
once and reused by every realisation of that size, and up to `workers` realisations are in
flight at once (one host thread each; the library releases the interpreter during its calls):
small fields, whose kernels fill a fraction of the GPU and whose phases end in short host
synchronisations, overlap on the device.  The contexts share the device memory: each is capped
at its share (plan), which sizes its batches of lines.  Each realisation's centerlines are
generated on the device, the field is built and its statistics stay on the device until read.

Autotuner: before the first realisation of a grid size, the deposition of a probe
realisation is timed over the deposition kernels' selection limits, one after the other: the
tube radius (grid spacings) up to which lines take the chord-piece kernel instead of the
sub-segment kernel, then the radius up to which pieces are deposited without tiles (the
scatter kernel), then the radius up to which the remaining pieces are rasterised once instead
of searched per tile.  Each setting is timed twice (the faster kept); one replaces the library's
default only if it is at least 5 % faster, and is then kept for the rest of that size.  Every
choice gives the same field within FP32 rounding; only the speed differs.  (The tile shape itself,
16 x 8 x 8 points, is fixed at compile time.)

    python -m fastweavturb_b200.ensemble [--members 64] [--workers 4]

runs the benchmark ensemble (configs.ensemble_member with seeds 1..members) and prints its
Mpts/s next to the same members built one at a time.
"""
from __future__ import annotations

import queue
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from .api import Context, Params, sp_exponents
from .configs import build_workload

TUNE_CANDIDATES = (0.0, 2.5, 5.0, 8.0)          # chord-piece kernel radius limit
SCATTER_CANDIDATES = (0.0, 2.5, 5.0, 8.0)       # scatter kernel (no tiles) radius limit
RASTER_CANDIDATES = (0.0, 1.5, 2.5, 4.0)        # rasterised pieces radius limit
DEFAULTS = (8.0, 5.0, 0.0)                      # the library's defaults of the three limits


class Ensemble:
    def __init__(self, device=0, tune=True, Sp_order=6, workers=4, mem_cap=None):
        self.device = device
        self.tune = tune
        self.Sp_order = Sp_order
        self.workers = max(1, int(workers))
        self.mem_cap = mem_cap     # device bytes per context, or per grid size (plan() sets them)
        self.ctx = {}
        self.tuned = {}
        self.tune_log = {}
        self._lock = threading.Lock()

    def context(self, N, slot=0):
        """Context `slot` of grid size N (created on first use, with its own stream)."""
        with self._lock:
            key = (N, slot)
            if key not in self.ctx:
                self.ctx[key] = Context(Params(N=N, N_downsample=N, line_s=1, line_e=0, sigma_ratio=1.0,
                                               device=self.device, pdf_bins=201, Sp_order=self.Sp_order,
                                               vorticity_output=0, mem_cap=self._cap(N)))
                if N in self.tuned:
                    self._apply(self.ctx[key], self.tuned[N])
            return self.ctx[key]

    @staticmethod
    def _apply(ctx, tuned):
        piece, scatter, raster = tuned
        ctx.set_piece_radius_limit(piece)
        ctx.set_scatter_radius_limit(scatter)
        ctx.set_raster_radius_limit(raster)

    def _load(self, ctx, w):
        return build_workload(ctx, w)

    def autotune(self, w):
        """Time the deposition of workload w over the piece limit, then the scatter limit, then
        the raster limit (each at the best of the earlier ones); keep the fastest of each."""
        import torch
        ctx = self.context(w.N)
        keep = self._load(ctx, w)

        def timed():
            ctx.deposit(1, w.ntubes)        # warm (allocations for this kernel choice)
            best = float("inf")
            for _ in range(2):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                ctx.deposit(1, w.ntubes)
                torch.cuda.synchronize()
                best = min(best, time.perf_counter() - t0)
            return best

        def pick(kind, candidates, default):
            return self.pick(times, kind, candidates, default)

        times = {}
        ctx.set_raster_radius_limit(-1.0)
        ctx.set_scatter_radius_limit(-1.0)
        for cells in TUNE_CANDIDATES:
            ctx.set_piece_radius_limit(cells)
            times[("piece", cells)] = timed()
        best_piece = pick("piece", TUNE_CANDIDATES, DEFAULTS[0])
        ctx.set_piece_radius_limit(best_piece)
        for cells in SCATTER_CANDIDATES:
            ctx.set_scatter_radius_limit(cells)
            times[("scatter", cells)] = timed()
        best_scatter = pick("scatter", SCATTER_CANDIDATES, DEFAULTS[1])
        ctx.set_scatter_radius_limit(best_scatter)
        for cells in RASTER_CANDIDATES:
            ctx.set_raster_radius_limit(cells)
            times[("raster", cells)] = timed()
        best_raster = pick("raster", RASTER_CANDIDATES, DEFAULTS[2])
        tuned = (best_piece, best_scatter, best_raster)
        with self._lock:
            for (n, _), c in self.ctx.items():
                if n == w.N:
                    self._apply(c, tuned)
        self.tuned[w.N] = tuned
        self.tune_log[w.N] = times
        del keep
        return self.tuned[w.N]

    @staticmethod
    def pick(times, kind, candidates, default, margin=0.05):
        """The setting of `kind` to keep from times[(kind, value)] (seconds): the fastest
        candidate if it beats the default by at least `margin`, else the default (one probe
        realisation and millisecond timings do not separate closer settings)."""
        best = min(candidates, key=lambda v: times[(kind, v)])
        return best if times[(kind, best)] < (1.0 - margin) * times[(kind, default)] else default

    def slots_for(self, N):
        """Contexts kept for grid size N: every worker for small fields, fewer for large ones,
        which fill the GPU by themselves and whose buffers (tile lists, records, three N^3
        fields) run to gigabytes."""
        cap = self.workers if N <= 96 else (2 if N <= 128 else 1)
        return max(1, min(self.workers, cap))

    def plan(self, members, total=None):
        """Share the GPU's memory between the contexts the members will use: 80 % of the device
        memory, 2 GB per context and the rest in proportion to N^3 (a context's fields, and
        the tile lists of its thick tubes, grow with N^3).  Each context's share is its cap
        (Params.mem_cap), which also bounds its batches of lines and its list of pairs handed to
        FP64.  Without it every context would size its batch buffers for 4 Mi nodes (gigabytes
        each) and sixteen contexts of five grid sizes would not fit.  Runs once, before the
        first context is made; returns the caps by grid size."""
        if self.mem_cap is not None:
            return self.mem_cap
        import torch
        sizes = sorted({w.N for w in members} | {n for (n, _) in self.ctx})
        slots = {N: self.slots_for(N) for N in sizes}
        if total is None:
            total = torch.cuda.mem_get_info(self.device)[1]
        base = 2.0e9
        spare = max(0.0, 0.8 * total - base * sum(slots.values()))
        vol = sum(slots[N] * N ** 3 for N in sizes)
        self.mem_cap = {N: int(base + spare * N ** 3 / vol) for N in sizes}
        return self.mem_cap

    def _cap(self, N):
        if isinstance(self.mem_cap, dict):
            return self.mem_cap.get(N, 0)
        return int(self.mem_cap or 0)

    def run(self, members, stats=True):
        """Build every member, up to `workers` at once; returns (per-member statistics in
        member order, wall seconds of the build, Mpts/s = sum N^3 / wall)."""
        import torch
        self.plan(members)
        for w in members:
            if self.tune and w.N not in self.tuned:
                self.autotune(w)
        torch.cuda.synchronize(self.device)
        slots = {}
        for N in sorted({w.N for w in members}):
            slots[N] = queue.Queue()
            for k in range(self.slots_for(N)):
                slots[N].put(k)

        def build(w):
            torch.cuda.set_device(self.device)
            slot = slots[w.N].get()
            try:
                ctx = self.context(w.N, slot)
                xyz = self._load(ctx, w)
                ctx.run()
                # the statistics are read back on the context's stream: after them no kernel
                # of this realisation still uses xyz
                res = member_statistics(ctx, w.N, self.Sp_order) if stats else ctx.cal_helicity()
                del xyz
                return res
            finally:
                slots[w.N].put(slot)

        t0 = time.perf_counter()
        if self.workers == 1:
            out = [build(w) for w in members]
        else:
            with ThreadPoolExecutor(max_workers=self.workers) as ex:
                out = list(ex.map(build, members))
        t_total = time.perf_counter() - t0
        if not stats:
            out = [None] * len(out)
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


def cfg3_members(n=64, seed0=1):
    """The benchmark ensemble: n realisations, seeds seed0.., grid sizes, levels, H, density and
    circulation exponent drawn per realisation (configs.ensemble_member)."""
    from .configs import ensemble_member
    return [ensemble_member(seed0 + k) for k in range(n)]


def main(argv=None):
    import argparse
    import json

    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--workers", type=int, default=4)
    args = ap.parse_args(argv)
    members = cfg3_members(args.members)
    ens = Ensemble(workers=args.workers, tune=True)
    ens.plan(members)
    ens.run(members[:min(4, len(members))], stats=False)     # warm: plans, buffers, autotuning
    _, t_conc, rate = ens.run(members, stats=False)
    # the same members one at a time (the sum of the single-field times)
    ens.workers = 1
    _, t_seq, rate_seq = ens.run(members, stats=False)
    ens.close()
    torch.cuda.synchronize()
    print(json.dumps({"members": len(members), "points": sum(w.N ** 3 for w in members),
                      "sizes": {str(N): sum(1 for w in members if w.N == N) for N in sorted({w.N for w in members})},
                      "concurrent_s": t_conc, "concurrent_mpts_s": rate, "sequential_s": t_seq,
                      "sequential_mpts_s": rate_seq, "tuned": {str(k): v for k, v in ens.tuned.items()}}))


if __name__ == "__main__":
    main()
