#!/usr/bin/env python
"""bench.py -- woven Mpts/s of the field-construction path on B200.

One step = one woven field built from centerlines already on the device: centerline set-up
(periodic arc length, quintic splines, adaptive sub-segmentation), Burgers-tube deposition,
spectral Biot-Savart omega -> u with E(k), normalisation, PDFs, S_p(r) and the downsampled
field output, i.e. the reference program's tube.f90:392-1188 (its file writing excluded).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config cfg1] [--precision 32]
    python bench.py --impl reference ...      # the CPU implementation of the path (see below)

metric  "woven Mpts/s": N^3 grid points per step / step time, summed over ranks.
value   device time (CUDA events on the library's stream), centerline nodes resident in HBM.
e2e     the same metric through the public C-ABI from pinned host memory: the host->device
        copy of the nodes, the whole path, and the device->host copy of the statistics and of
        the downsampled field each step.
Multi-GPU: the path does not shard (one field per GPU); each rank builds its own
realisation (seed = rank) -- replicas, weak scaling.  No data-path collective.

The reference arm (--impl reference) times the FP64 CPU restatement of the reference
(oracle/, the Fortran reference cannot be compiled in this image) on the host cores: each
step deposits a bounded sample of the workload's lines (the first tube of every level),
scales each level by its tube count, and adds the full-size spectral path and statistics
(S_p on two separations scaled to all), giving an estimated whole-field time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


# --------------------------------------------------------------------------- clocks sampler
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# --------------------------------------------------------------------------- replicas
def max_over_ranks(ms, dist=None, device="cpu"):
    """The job's time is its slowest rank's: all-reduce MAX of a per-rank device time."""
    if dist is None:
        return float(ms)
    import torch

    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, steps, N, ms):
    """Mpts/s of the whole job: every rank builds `steps` fields of N^3 points in `ms`."""
    return world * steps * N ** 3 / (ms / 1e3) / 1e6


# --------------------------------------------------------------------------- CPU sample
def cpu_sample_estimate(w, nthreads=None):
    """Estimated FP64 CPU time (s) of one whole woven field of workload `w` with the oracle:
    deposition of the first tube of each level scaled by the level's tube count, plus the
    full-size spectral path, PDFs and S_p (two separations scaled to all)."""
    from oracle import oracle as O

    O.build()
    nthreads = nthreads or os.cpu_count() or 1
    O.set_fft_workers(nthreads)
    N = w.N
    t_dep = 0.0
    vor = np.zeros((3, N, N, N))
    t0 = 0
    for L in w.levels:
        xyz = O.fbb_tube(w.seed, t0, L.nodes, L.H, L.dB)
        p = O.Params(N=N, N_downsample=N, line_s=1, line_e=1, sigma_ratio=w.sigma_ratio, eta_t=w.eta_t,
                     ntf_times=w.ntf_times, ntf_pre=w.ntf_pre, Rtube_ratio=w.Rtube_ratio, dzeta_sup=w.dzeta_sup,
                     sigma=np.array([L.sigma]), Gamma=np.array([L.Gamma]), n_T=np.array([1], dtype=np.int32),
                     if_filter=np.zeros(1, dtype=np.int32))
        cl = O.Centerlines(npoint=np.array([L.nodes]), xyz=xyz)
        t = time.perf_counter()
        O.deposit(p, cl, nthreads=nthreads, vor=vor)
        t_dep += (time.perf_counter() - t) * L.tubes
        t0 += L.tubes
    t = time.perf_counter()
    O.spectrum(vor)
    vel = O.biot_savart(vor)
    O.normalise(vor, vel)
    O.spectrum(vel)
    t_spec = time.perf_counter() - t
    t = time.perf_counter()
    O.pdf(vel.astype(np.float32).reshape(3 * N, N, N))
    O.pdf(vor.astype(np.float32).reshape(3 * N, N, N))
    t_pdf = time.perf_counter() - t
    rr = O.sp_separations(N)
    t = time.perf_counter()
    O.structure_functions(vel, pmax=10, r=rr[:2], nthreads=nthreads)
    t_sp = (time.perf_counter() - t) * len(rr) / 2.0   # cost is linear in the number of separations
    est = t_dep + t_spec + t_pdf + t_sp
    return est, {"deposit_s": t_dep, "spectral_s": t_spec, "stats_s": t_pdf + t_sp, "threads": nthreads}


def run_reference(args):
    """The reference arm: the oracle's FP64 CPU path on the host cores (rank 0 only)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from fastweavturb_b200.configs import CONFIGS

    w = CONFIGS[args.config](seed=0)
    nthreads = os.cpu_count() or 1
    # one untimed sample warms the caches and builds the oracle; more would only cost minutes
    for _ in range(min(args.warmup, 1)):
        cpu_sample_estimate(w, nthreads)
    ests = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e, _ = cpu_sample_estimate(w, nthreads)
        ests.append(e)
    wall = time.perf_counter() - t0
    est = float(np.mean(ests))
    val = w.N ** 3 / est / 1e6
    line = {
        "impl": "reference", "metric": "woven Mpts/s", "value": val, "unit": "Mpts/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": est * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded fBb centerlines)",
        "config": {"workload": w.name, "N": w.N, "lines": w.ntubes, "nodes": w.nnodes},
        "cpu_baseline": {"value": val, "unit": "Mpts/s", "cores": nthreads, "kind": "port",
                         "sample": "first tube of every level deposited and scaled by tube count; full-size FFT "
                                   "path, PDFs, S_p at 2 separations scaled; estimated whole-field seconds "
                                   f"{est:.2f}, sample wall {wall / max(args.steps, 1):.1f} s/step"},
        "e2e": {"value": val, "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------------------- GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fwt", choices=["fwt", "reference"])
    ap.add_argument("--config", default="cfg1")
    ap.add_argument("--precision", type=int, default=32)
    ap.add_argument("--deposit-mode", type=int, default=0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--level", type=int, default=None,
                    help="deposit only this scale level of the workload (a bounded case for profiler captures)")
    ap.add_argument("--lines", type=int, default=None,
                    help="with --level: keep only the first LINES tubes of that level")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch

    import fastweavturb_b200 as F
    from fastweavturb_b200.configs import CONFIGS, build_workload

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    w = CONFIGS[args.config](seed=rank)
    if args.level is not None:
        w.levels = [w.levels[args.level]]
        w.name += f" -- level {args.level} only (profiling case)"
        if args.lines:
            w.levels[0].tubes = min(w.levels[0].tubes, args.lines)
            w.name += f", first {w.levels[0].tubes} lines"
    stream = torch.cuda.current_stream()
    params = F.Params(N=w.N, N_downsample=w.N, line_s=1, line_e=w.ntubes, sigma_ratio=w.sigma_ratio,
                      eta_t=w.eta_t, ntf_times=w.ntf_times, ntf_pre=w.ntf_pre, Rtube_ratio=w.Rtube_ratio,
                      dzeta_sup=w.dzeta_sup, precision=args.precision, deposit_mode=args.deposit_mode,
                      device=local, stream=stream.cuda_stream)
    ctx = F.Context(params)
    xyz, (npoint, sig, gam, nT) = build_workload(ctx, w)
    torch.cuda.synchronize()

    for _ in range(args.warmup):
        ctx.run()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ktimes = {}
    launches = 0
    e0.record(stream)
    for _ in range(args.steps):
        ctx.run()
        for k, (ms, n) in ctx.kernel_times().items():
            a = ktimes.setdefault(k, [0.0, 0])
            a[0] += ms
            a[1] += n
        launches += ctx.counters()["launches"]
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks.stop()
    ms = e0.elapsed_time(e1)
    t_max = max_over_ranks(ms, dist, "cuda")
    ms_step = t_max / args.steps
    value = whole_job_rate(world, args.steps, w.N, t_max)
    counters = ctx.counters()

    # dominant kernel and its roofline
    peaks, pk_kind = measured_peaks()
    dom = max(ktimes.items(), key=lambda kv: kv[1][0])
    dom_name, (dom_ms, dom_n) = dom
    dep_launches = ktimes.get("deposit", [0.0, 0])[1] // args.steps
    kb = _kernel_bytes(ctx, w, counters, args.precision, dep_launches)
    dom_bytes = kb.get(dom_name)
    roofline = None
    if dom_n:
        avg_ms = dom_ms / dom_n
        per_launch_bytes = (dom_bytes / max(1, ktimes[dom_name][1] // args.steps)) if dom_bytes else None
        achieved = per_launch_bytes / (avg_ms / 1e3) / 1e9 if per_launch_bytes else None
        roofline = {"kernel": dom_name, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                    "unit": "GB/s", "frac": (achieved / peaks["hbm_gbs"]) if achieved else None,
                    "traffic": None, "peak_kind": pk_kind, "avg_launch_ms": avg_ms,
                    "share_of_step": dom_ms / max(ms, 1e-9)}

    # end to end through the public API from pinned host memory
    e2e = None
    if not args.no_e2e:
        host = xyz.T.contiguous().cpu().pin_memory()
        hx = host.numpy()
        nd = params.N_downsample
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            ctx.set_centerlines(npoint, hx, sig, gam, nT)
            ctx.run()
            ctx.output_v()
        f1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(f0.elapsed_time(f1), dist, "cuda")
        h2d = int(hx.nbytes)
        d2h = int(2 * nd ** 3 * 4 + 2 * (w.N // 2) * 8 + 2 * params.pdf_bins * 8 * 2
                  + 10 * len(F.sp_separations(w.N)) * 8)
        e2e = {"value": whole_job_rate(world, args.steps, w.N, ems), "unit": "Mpts/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": ems / args.steps}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        est, parts = cpu_sample_estimate(w)
        cpu = {"value": w.N ** 3 / est / 1e6, "unit": "Mpts/s", "cores": parts["threads"], "kind": "port",
               "sample": "FP64 oracle: first tube of every level deposited and scaled by the level's tube count, "
                         "full-size spectral path and statistics (S_p on 2 separations scaled to all); "
                         f"estimated whole-field {est:.1f} s"}

    if rank == 0:
        line = {
            "metric": "woven Mpts/s", "value": value, "unit": "Mpts/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == 32 else "f64",
            "data": "synthetic (seeded fBb centerlines generated on the GPU)",
            "config": {"workload": w.name, "N": w.N, "lines": w.ntubes, "nodes": w.nnodes,
                       "sections": counters["sections"], "subsegments": counters["subsegments"],
                       "cell_pairs": counters["pairs"], "precision": args.precision,
                       "deposit": "tile-owned cell lists" if args.deposit_mode == 0 else "reference box walk",
                       "l2": "inputs larger than L2 (omega, u, spectra, sub-segment records >> 126 MB)",
                       "parallelism": f"replicas x{world}"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clocks.summary(),
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in ktimes.items()},
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()
    return 0


def _kernel_bytes(ctx, w, counters, precision, dep_launches):
    """Algorithmic bytes per step of each kernel category: section presampling reads the node
    data and writes coefficients; the deposition writes omega in its first launch, reads and
    writes it in each later launch (one launch per batch of lines), and reads one 224-byte
    sub-segment record plus a 4-byte cell-list entry per (tile, sub-segment) pair; the fused
    Biot-Savart reads and writes the half spectrum once."""
    N = w.N
    rb = 4 if precision == 32 else 8
    n3 = N ** 3
    nh = N * N * (N // 2 + 1)
    secs = counters["sections"] + counters["lines"]
    subseg_record = 224
    field = 3 * n3 * rb * (1 + 2 * max(0, dep_launches - 1))
    return {
        "section_presample": secs * (3 * 8 + 6 * 8 + 8) + secs * (18 * 8 + 4 + 8),
        "deposit": field + counters["pairs"] * (4 + subseg_record) if counters["pairs"]
        else counters["subsegments"] * subseg_record + field,
        "biot_savart": 2 * 3 * nh * 2 * rb,
        "cufft": 6 * 3 * n3 * rb * 2,
        "statistics": 3 * n3 * rb * 4,
        "centerline_setup": counters["subsegments"] * (subseg_record + 8 * 8),
        "binning": counters["pairs"] * 8 * 3 + counters["subsegments"] * subseg_record,
        "generator": 0,
    }


if __name__ == "__main__":
    sys.exit(main())
