"""The surrogate experiment: train on generator realisations, then fit parameters to a
held-out target with and without the network, both judged by the generator.

The reference has no surrogate; this is the learned-surrogate workload that sits on top of the
batched generator (64^3 realisations here, parameters H, density multiplier, Gamma exponent and
level count drawn as in the ensemble configuration).

    python -m fastweavturb_b200.surrogate_experiment [--train 4096] [--N 64] [--steps 3000]
                                                    [--runs 96] [--tol 0.02] [--targets 4]

Prints one JSON line: data-generation and training times, the held-out prediction error
(against predicting the training mean), and for inverse fits to held-out draws the surrogate-
driven fit against the same generator-judged search started from random draws instead of the
network's proposals.  Both stop once spectrum and flatness are within `tol` or after `runs`
generator runs; per fit the line gives each one's errors, runs, wall time (the network's
inverse fit included), whether it reached `tol`, and the wall time each needed to reach the
error the worse of the two ended with; beside them the error of the training set's mean
statistics (the fit that uses no information about the target).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--valid", type=int, default=64)
    ap.add_argument("--N", type=int, default=64)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--runs", type=int, default=96, help="generator run budget of each fit")
    ap.add_argument("--tol", type=float, default=0.02, help="a fit stops once spectrum and flatness are within tol")
    ap.add_argument("--targets", type=int, default=4, help="held-out target draws")
    args = ap.parse_args(argv)

    from .ensemble import Ensemble
    from .surrogate import (Surrogate, draw_params, fit_error, fit_generator_only, fit_surrogate_driven, generate,
                            within)

    rng = np.random.default_rng(args.seed)
    ens = Ensemble()
    P = draw_params(rng, args.train + args.valid)
    seeds = 1000 + np.arange(len(P))
    t0 = time.perf_counter()
    Y, dev_s = generate(P, seeds, N=args.N, ens=ens)
    t_gen = time.perf_counter() - t0
    Ptr, Ytr, Pva, Yva = P[:args.train], Y[:args.train], P[args.train:], Y[args.train:]
    sur = Surrogate(seed=args.seed)
    t0 = time.perf_counter()
    losses = sur.fit(Ptr, Ytr, steps=args.steps)
    t_train = time.perf_counter() - t0
    pred = sur.predict(Pva)
    err_net = float(np.sqrt(np.mean(((pred - Yva) / sur.ysd) ** 2)))
    err_mean = float(np.sqrt(np.mean(((Ytr.mean(axis=0) - Yva) / sur.ysd) ** 2)))
    # inverse fits to held-out draws: both searches stop at the tolerance or at the run budget
    fits = []
    for k in range(args.targets):
        p_true = draw_params(np.random.default_rng(args.seed + 99 + k), 1)[0]
        seed_t = 424242 + k
        y_t, _ = generate(p_true[None, :], [seed_t], N=args.N, ens=ens)
        p_s, e_s, t_s, r_s, tr_s = fit_surrogate_driven(sur, y_t[0], seed_t, args.runs, N=args.N, ens=ens,
                                                        tol=args.tol)
        p_g, e_g, t_g, r_g, tr_g = fit_generator_only(y_t[0], seed_t, args.runs, N=args.N, ens=ens, seed=k + 1,
                                                      tol=args.tol)
        e_m = fit_error(Ytr.mean(axis=0), y_t[0])
        # the wall time each search needs to reach the error the worse of the two ends with
        common = max(tr_s[-1][2], tr_g[-1][2])
        reach = lambda tr: next(t for (_, t, e, _) in tr if e <= common)
        fits.append({"target": p_true.tolist(), "training_mean": {"err_logE": e_m[0], "err_flat": e_m[1]},
                     "common_err": common,
                     "surrogate": {"params": p_s.tolist(), "err_logE": e_s[0], "err_flat": e_s[1], "wall_s": t_s,
                                   "runs": r_s, "within_tol": within(e_s, args.tol),
                                   "wall_s_to_common": reach(tr_s)},
                     "generator_only": {"params": p_g.tolist(), "err_logE": e_g[0], "err_flat": e_g[1],
                                        "wall_s": t_g, "runs": r_g, "within_tol": within(e_g, args.tol),
                                        "wall_s_to_common": reach(tr_g)}})
    summary = {}
    for m in ("surrogate", "generator_only"):
        summary[m] = {"mean_err": float(np.mean([f[m]["err_logE"] + f[m]["err_flat"] for f in fits])),
                      "within_tol": int(sum(f[m]["within_tol"] for f in fits)),
                      "mean_wall_s": float(np.mean([f[m]["wall_s"] for f in fits])),
                      "mean_wall_s_to_common": float(np.mean([f[m]["wall_s_to_common"] for f in fits])),
                      "mean_runs": float(np.mean([f[m]["runs"] for f in fits]))}
    line = {
        "experiment": "surrogate", "N": args.N, "train": args.train, "valid": args.valid,
        "generation_s": t_gen, "generation_Mpts_per_s": len(P) * args.N ** 3 / dev_s / 1e6,
        "autotune": {str(k): v for k, v in ens.tuned.items()}, "train_s": t_train, "steps": args.steps,
        "loss_first": float(losses[0]), "loss_last": float(np.mean(losses[-50:])),
        "valid_rms_std_units": {"network": err_net, "training_mean": err_mean},
        "run_budget": args.runs, "tol": args.tol, "fits": fits, "summary": summary,
        "mean_err": {"training_mean": float(np.mean([f["training_mean"]["err_logE"] + f["training_mean"]["err_flat"]
                                                      for f in fits])),
                     "surrogate": summary["surrogate"]["mean_err"],
                     "generator_only": summary["generator_only"]["mean_err"]},
    }
    print(json.dumps(line))
    sur.close()
    ens.close()
    return line


if __name__ == "__main__":
    main()
