#!/usr/bin/env python
"""bench.py -- woven Mpts/s of the field-construction path on B200.

One step = one woven field built from centerlines already on the device: centerline set-up
(periodic arc length, quintic splines, adaptive sub-segmentation), Burgers-tube deposition,
spectral Biot-Savart omega -> u with E(k), normalisation, PDFs, S_p(r) and the downsampled
field output, i.e. the reference program's tube.f90:392-1188 (its file writing excluded).
The default workload is the 1024^3, 8-level field (cfg2).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config cfg2] [--precision 32]
    python bench.py --impl reference ...      # the CPU implementation of the path (see below)

metric  "woven Mpts/s": N^3 grid points per step / step time, summed over ranks.
value   FP32 device time (CUDA events on the library's stream), centerline nodes resident in HBM.
e2e     the same metric through the public C-ABI between pinned host buffers: the host->device
        copy of the nodes, the whole path, and the device->host copy of the statistics and of
        the downsampled field each step (min(K, 3) steps unless --e2e-steps).
fp64    the same workload through the FP64 tile path (--fp64-steps fields): its Mpts/s, the
        FP32 / FP64 ratio and the FP32 errors against it (relative L2 of omega, u and E(k),
        relative errors of S_2..S_6).
Multi-GPU: the path does not shard (one field per GPU); each rank builds its own
realisation (seed = rank) -- replicas, weak scaling.  No data-path collective.

The reference arm (--impl reference) times the FP64 CPU restatement of the reference
(oracle/; the Fortran reference cannot be compiled in this image) on the host cores: each
step is a bounded sample (the first tube of every level on a reduced grid, the spectral path
and statistics at <= 256^3), scaled to an estimated whole-field time.
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
# Algorithmic bytes of the path (per grid point, FP32): omega written 12; R2C reads 12, writes the
# half spectrum 12; the fused Biot-Savart / spectra / energy pass reads and writes it (24); C2R
# reads 12, writes 12; statistics and the field output read u and omega (24) and write <= 8:
# 116 B per point (232 in FP64).  Deposition adds the centerline data: about 200 B per node
# (coordinates, arc length, derivatives, the section's spline and sub-segment set-up).
PATH_BYTES_PER_POINT = {32: 116, 64: 232}
# FP32 operations of one accepted (point, chord) pair of the constant-core path (FMA = 2): the
# three plane/cylinder tests (about 20), the quintic and its derivative by Horner (54), the
# divided-difference offset of the piece kernels (34), x - c(zeta), rho^2, |c'|^2, the tangent,
# the Burgers profile and the fixed-point scaling (about 37), with two hardware rsqrt/exp
FLOPS_PER_PAIR = 145
# nominal FP32 FMA peak of a B200: 148 SMs x 128 lanes x 2 flops x 1.965 GHz
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12
DEPOSIT_BYTES_PER_POINT = {32: 12, 64: 24}
BYTES_PER_NODE = 200


def level_sample_grid(w, L):
    """Grid of the CPU sample of level L: the box walk of the reference costs (box points per
    sub-segment) x (sub-segments), and its boxes span 2 Rtube + a chord, so on a grid N' with
    Rtube >= 4 grid spacings the cost of a tube scales as (N / N')^3.  The smallest such grid
    (at least 64) bounds the sample; levels thinner than that keep the workload's grid."""
    Rt = w.Rtube_ratio * L.sigma * w.sigma_ratio
    n = 64
    while n < w.N and Rt * n / (2 * np.pi) < 4.0:
        n *= 2
    return min(n, w.N)


_SAMPLE_GRIDS = {}


def _sample_field(n):
    """One (3, n, n, n) FP64 array per sample grid, kept across samples: the deposition only adds
    into it, so its contents do not matter to the timing, and allocating 26 GB per 1024^3 sample
    would cost more than the deposition."""
    if n not in _SAMPLE_GRIDS:
        _SAMPLE_GRIDS[n] = np.zeros((3, n, n, n))
    return _SAMPLE_GRIDS[n]


def cpu_sample_estimate(w, nthreads=None):
    """Estimated FP64 CPU time (s) of one whole woven field of workload `w` with the oracle,
    from a bounded sample: the first tube of every level deposited on the level's sample grid
    (level_sample_grid) and scaled by (N / N')^3 and the level's tube count; the spectral path,
    the PDFs and S_p (two separations, scaled to all) on a grid of at most 256^3, scaled by the
    FFT's N^3 log N or the statistics' N^3."""
    from oracle import oracle as O

    O.build()
    nthreads = nthreads or os.cpu_count() or 1
    O.set_fft_workers(nthreads)
    N = w.N
    t_dep = 0.0
    t0 = 0
    for L in w.levels:
        n = level_sample_grid(w, L)
        xyz = O.fbb_tube(w.seed, t0, L.nodes, L.H, L.dB)
        p = O.Params(N=n, N_downsample=n, line_s=1, line_e=1, sigma_ratio=w.sigma_ratio, eta_t=w.eta_t,
                     ntf_times=w.ntf_times, ntf_pre=w.ntf_pre, Rtube_ratio=w.Rtube_ratio, dzeta_sup=w.dzeta_sup,
                     sigma=np.array([L.sigma]), Gamma=np.array([L.Gamma]), n_T=np.array([1], dtype=np.int32),
                     if_filter=np.zeros(1, dtype=np.int32))
        cl = O.Centerlines(npoint=np.array([L.nodes]), xyz=xyz)
        t = time.perf_counter()
        O.deposit(p, cl, nthreads=nthreads, vor=_sample_field(n))
        t_dep += (time.perf_counter() - t) * L.tubes * (N / n) ** 3
        t0 += L.tubes
    ns = min(N, 256)
    rng = np.random.default_rng(0)
    vor = rng.standard_normal((3, ns, ns, ns))
    t = time.perf_counter()
    O.spectrum(vor)
    vel = O.biot_savart(vor)
    O.normalise(vor, vel)
    O.spectrum(vel)
    t_spec = (time.perf_counter() - t) * (N / ns) ** 3 * np.log(N ** 3) / np.log(ns ** 3)
    t = time.perf_counter()
    O.pdf(vel.astype(np.float32).reshape(3 * ns, ns, ns))
    O.pdf(vor.astype(np.float32).reshape(3 * ns, ns, ns))
    t_pdf = (time.perf_counter() - t) * (N / ns) ** 3
    rr = O.sp_separations(ns)
    t = time.perf_counter()
    O.structure_functions(vel, pmax=10, r=rr[:2], nthreads=nthreads)
    t_sp = (time.perf_counter() - t) / 2.0 * len(O.sp_separations(N)) * (N / ns) ** 3
    est = t_dep + t_spec + t_pdf + t_sp
    grids = [level_sample_grid(w, L) for L in w.levels]
    return est, {"deposit_s": t_dep, "spectral_s": t_spec, "stats_s": t_pdf + t_sp, "threads": nthreads,
                 "sample": f"FP64 oracle: the first tube of every level deposited on grids {grids} and scaled by "
                           f"(N/N')^3 x tubes; spectral path, PDFs and S_p (2 separations) at {ns}^3 scaled to "
                           f"{N}^3 (N^3 log N, N^3, separations); estimated whole field {est:.1f} s"}


def run_reference(args):
    """The reference arm: the oracle's FP64 CPU path on the host cores (rank 0 only).  Each
    step is one bounded sample (cpu_sample_estimate); ms_per_step is its measured wall time and
    value the whole-field throughput estimated from it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from fastweavturb_b200.configs import CONFIGS

    w = CONFIGS[args.config](seed=0)
    nthreads = os.cpu_count() or 1
    for _ in range(min(args.warmup, 1)):   # builds the oracle and warms the caches
        cpu_sample_estimate(w, nthreads)
    ests, walls = [], []
    for _ in range(args.steps):
        t = time.perf_counter()
        e, parts = cpu_sample_estimate(w, nthreads)
        walls.append(time.perf_counter() - t)
        ests.append(e)
    est = float(np.mean(ests))
    val = w.N ** 3 / est / 1e6
    line = {
        "impl": "reference", "metric": "woven Mpts/s", "value": val, "unit": "Mpts/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(walls)) * 1e3,
        "estimated_field_ms": est * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded fBb centerlines)",
        "config": {"workload": w.name, "N": w.N, "lines": w.ntubes, "nodes": w.nnodes},
        "cpu_baseline": {"value": val, "unit": "Mpts/s", "cores": nthreads, "kind": "port",
                         "sample": parts["sample"] + "; ms_per_step is the sample's wall time"},
        "e2e": {"value": val, "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------------------- GPU arm
def timed_runs(ctx, stream, steps, torch):
    """Device ms of `steps` whole runs (CUDA events on the library's stream), the summed
    per-category kernel times, and the launches of this library's kernels."""
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ktimes, launches = {}, 0
    e0.record(stream)
    for _ in range(steps):
        ctx.run()
        for k, (ms, n) in ctx.kernel_times().items():
            a = ktimes.setdefault(k, [0.0, 0])
            a[0] += ms
            a[1] += n
        launches += ctx.counters()["launches"]
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), ktimes, launches


def rel_l2_device(a, b, torch):
    """||a - b|| / ||b|| of two fields (3, N, N, N) of any precision, in FP64 on b's device, by
    z-slabs (a may be held in host memory)."""
    num = den = 0.0
    for c in range(3):
        for z in range(0, a.shape[1], 64):
            x = a[c, z:z + 64].to(b.device).double()
            y = b[c, z:z + 64].double()
            num += float(torch.sum((x - y) ** 2))
            den += float(torch.sum(y * y))
    return (num / den) ** 0.5 if den > 0 else float("nan")


def rel_l2(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fwt", choices=["fwt", "reference"])
    ap.add_argument("--config", default="cfg2")
    ap.add_argument("--precision", type=int, default=32)
    ap.add_argument("--deposit-mode", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=None,
                    help="steps of the end-to-end leg (default: min(steps, 3))")
    ap.add_argument("--fp64-steps", type=int, default=1,
                    help="fields of the FP64 leg (FP64 tile path, same workload): its Mpts/s and the FP32 "
                         "errors against it; 0 skips the leg")
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

    def workload():
        w = CONFIGS[args.config](seed=rank)
        if args.level is not None:
            w.levels = [w.levels[args.level]]
            w.name += f" -- level {args.level} only (profiling case)"
            if args.lines:
                w.levels[0].tubes = min(w.levels[0].tubes, args.lines)
                w.name += f", first {w.levels[0].tubes} lines"
        return w

    w = workload()
    stream = torch.cuda.current_stream()

    def make_ctx(precision, mode):
        prm = F.Params(N=w.N, N_downsample=w.N, line_s=1, line_e=w.ntubes, sigma_ratio=w.sigma_ratio,
                       eta_t=w.eta_t, ntf_times=w.ntf_times, ntf_pre=w.ntf_pre, Rtube_ratio=w.Rtube_ratio,
                       dzeta_sup=w.dzeta_sup, precision=precision, deposit_mode=mode, device=local,
                       stream=stream.cuda_stream)
        ctx = F.Context(prm)
        xyz, arrs = build_workload(ctx, w)
        torch.cuda.synchronize()
        return prm, ctx, xyz, arrs

    params, ctx, xyz, (npoint, sig, gam, nT) = make_ctx(args.precision, args.deposit_mode)
    for _ in range(args.warmup):
        ctx.run()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms, ktimes, launches = timed_runs(ctx, stream, args.steps, torch)
    if dist:
        dist.barrier()
    clocks.stop()
    t_max = max_over_ranks(ms, dist, "cuda")
    ms_step = t_max / args.steps
    value = whole_job_rate(world, args.steps, w.N, t_max)
    counters = ctx.counters()

    # dominant kernel and its roofline (algorithmic bytes: deposition writes omega, 12 B per
    # point, and reads the centerline data, about 200 B per node)
    peaks, pk_kind = measured_peaks()
    dom_name, (dom_ms, dom_n) = max(ktimes.items(), key=lambda kv: kv[1][0])
    rb = 4 if args.precision == 32 else 8
    step_bytes = {"deposit": DEPOSIT_BYTES_PER_POINT[args.precision] * w.N ** 3 + BYTES_PER_NODE * w.nnodes}
    roofline = None
    if dom_n:
        launches_per_step = dom_n / args.steps
        avg_ms = dom_ms / dom_n
        per_launch = step_bytes.get(dom_name, 0) / launches_per_step if dom_name in step_bytes else None
        achieved = per_launch / (avg_ms / 1e3) / 1e9 if per_launch else None
        roofline = {"kernel": dom_name, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                    "unit": "GB/s", "frac": (achieved / peaks["hbm_gbs"]) if achieved else None,
                    "traffic": deposit_traffic(w, counters, launches_per_step) if dom_name == "deposit" else None,
                    "peak_kind": pk_kind, "avg_launch_ms": avg_ms, "launches_per_step": launches_per_step,
                    "algorithmic_bytes_per_launch": per_launch, "share_of_step": dom_ms / max(ms, 1e-9),
                    "bytes_model": "12 B per grid point (omega) + 200 B per centerline node, per step"}
        acc = counters.get("accepted", 0)
        if dom_name == "deposit" and acc:
            roofline["accepted_pairs_per_step"] = acc
            roofline["accepted_pairs_per_s"] = acc / (dom_ms / args.steps / 1e3)
            # the deposition is instruction-bound, not HBM-bound: its FP32 arithmetic ceiling
            tf = roofline["accepted_pairs_per_s"] * FLOPS_PER_PAIR / 1e12
            roofline["fp32_ceiling"] = {"flops_per_pair": FLOPS_PER_PAIR, "achieved_tflops": tf,
                                        "peak_tflops": FP32_PEAK_TFLOPS, "peak_kind": "nominal",
                                        "frac": tf / FP32_PEAK_TFLOPS}
    whole_path = {"bytes_per_step": PATH_BYTES_PER_POINT[args.precision] * w.N ** 3 + BYTES_PER_NODE * w.nnodes}
    whole_path["achieved_gbs"] = whole_path["bytes_per_step"] / (ms_step / 1e3) / 1e9
    whole_path["frac"] = whole_path["achieved_gbs"] / peaks["hbm_gbs"]

    # end to end through the public API from pinned host memory
    e2e = None
    if not args.no_e2e:
        # the nodes to pinned host memory, one coordinate at a time; the generator's device copy
        # is released first, since the library now holds its own (at 1024^3 both do not fit)
        host = torch.empty((w.nnodes, 3), dtype=torch.float64, pin_memory=True)
        for d in range(3):
            host[:, d].copy_(xyz[d])
        xyz = None
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        hx = host.numpy()
        nd = params.N_downsample
        # the result goes to pinned host memory as the inputs come from it (into a fresh
        # pageable array the driver's staging takes 2.1 s for the 8.6 GB of cfg2, 0.17 s pinned)
        hout = torch.empty(2 * nd ** 3, dtype=torch.float32, pin_memory=True)
        ho = hout.numpy()
        ne = args.e2e_steps or min(args.steps, 3)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(ne):
            # the upload runs behind the deposition, batch by batch (fwt_set_centerlines_async)
            ctx.set_centerlines(npoint, hx, sig, gam, nT, async_upload=True)
            ctx.run()
            ctx.output_v(out=ho)
        f1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(f0.elapsed_time(f1), dist, "cuda")
        h2d = int(hx.nbytes)
        d2h = int(2 * nd ** 3 * 4 + 2 * (w.N // 2) * 8 + 2 * params.pdf_bins * 8 * 2
                  + 10 * len(F.sp_separations(w.N)) * 8)
        e2e = {"value": whole_job_rate(world, ne, w.N, ems), "unit": "Mpts/s", "steps": ne,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": ems / ne}
        del host, hout

    # the FP64 leg: the same workload through the FP64 tile path; FP32 errors against it
    fp64 = None
    if args.fp64_steps > 0 and args.precision == 32 and world == 1:
        ctx.run()
        ew32, eu32 = ctx.spectrum(0), ctx.spectrum(1)
        ctx.cal_helicity()
        _, sp32 = ctx.Sp_calculate(pmax=10)
        # the FP32 fields wait in host memory while the FP64 context holds the device
        w32 = ctx.field_tensor(0).cpu()
        u32 = ctx.field_tensor(1).cpu()
        ctx.close()
        xyz = None
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        _, ctx64, xyz64, _ = make_ctx(64, 0)
        ms64, kt64, _ = timed_runs(ctx64, stream, args.fp64_steps, torch)
        ew64, eu64 = ctx64.spectrum(0), ctx64.spectrum(1)
        ctx64.cal_helicity()
        _, sp64 = ctx64.Sp_calculate(pmax=10)
        err = {"omega_rel_l2": rel_l2_device(w32, ctx64.field_tensor(0), torch),
               "u_rel_l2": rel_l2_device(u32, ctx64.field_tensor(1), torch),
               "Ek_omega_rel_l2": rel_l2(ew32, ew64), "Ek_u_rel_l2": rel_l2(eu32, eu64)}
        # S_p per entry, relative to the larger of the entry and the natural size (max S_2)^(p/2):
        # odd orders pass through zero
        s2max = float(np.max(np.abs(sp64[1])))
        for q in range(1, 6):
            den = np.maximum(np.abs(sp64[q]), s2max ** ((q + 1) / 2.0))
            err[f"S{q + 1}_rel"] = float(np.max(np.abs(sp32[q] - sp64[q]) / den))
        v64 = whole_job_rate(1, args.fp64_steps, w.N, ms64)
        fp64 = {"value": v64, "unit": "Mpts/s", "steps": args.fp64_steps, "ms_per_step": ms64 / args.fp64_steps,
                "path": "FP64 tile path (FP32 candidate tests, the reference's FP64 tests and arithmetic)",
                "fp32_over_fp64": value / v64, "errors_fp32_vs_fp64": err,
                "kernel_ms_per_step": {k: v[0] / args.fp64_steps for k, v in kt64.items()}}
        ctx64.close()
        del w32, u32, xyz64
        ctx = None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        est, parts = cpu_sample_estimate(w)
        cpu = {"value": w.N ** 3 / est / 1e6, "unit": "Mpts/s", "cores": parts["threads"], "kind": "port",
               "sample": parts["sample"]}

    if rank == 0:
        line = {
            "metric": "woven Mpts/s", "value": value, "unit": "Mpts/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == 32 else "f64",
            "data": "synthetic (seeded fBb centerlines generated on the GPU)",
            "config": {"workload": w.name, "N": w.N, "lines": w.ntubes, "nodes": w.nnodes,
                       "sections": counters["sections"], "subsegments": counters["subsegments"],
                       "cell_pairs": counters["pairs"], "accepted_pairs": counters["accepted"],
                       "pairs_fp64": counters["redone_fp64"],
                       "precision": args.precision,
                       "deposit": "tile-owned cell lists" if args.deposit_mode == 0 else "reference box walk",
                       "l2": "inputs larger than L2 (omega, u, spectra, sub-segment records >> 126 MB)",
                       "parallelism": f"replicas x{world}"},
            "roofline": roofline, "whole_path_roofline": whole_path, "cpu_baseline": cpu, "e2e": e2e,
            "fp64": fp64, "gpu_launches": launches, "clocks": clocks.summary(),
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in ktimes.items()},
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if ctx is not None:
        ctx.close()
    return 0


def deposit_traffic(w, counters, launches_per_step):
    """DRAM bytes per deposition launch from the ncu capture summarised in
    profiles/deposit_traffic.txt (bytes per accepted pair and per grid point of a bounded case,
    scaled to this workload's per-launch counts), or None without that summary."""
    path = os.path.join(ROOT, "profiles", "deposit_traffic.txt")
    if not os.path.exists(path):
        return None
    vals = {}
    with open(path) as f:
        for ln in f:
            if ":" in ln and not ln.startswith("#"):
                k, v = ln.split(":", 1)
                try:
                    vals[k.strip()] = float(v.split()[0])
                except (ValueError, IndexError):
                    pass
    if "bytes_per_accepted_pair" not in vals or "bytes_per_grid_point" not in vals:
        return None
    per_step = vals["bytes_per_accepted_pair"] * counters.get("accepted", 0) + \
        vals["bytes_per_grid_point"] * w.N ** 3
    return per_step / max(launches_per_step, 1)


if __name__ == "__main__":
    sys.exit(main())
