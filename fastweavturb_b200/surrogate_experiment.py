"""The surrogate experiment: train on generator realisations, then fit parameters to a
held-out target with and without the network, both judged by the generator.

The reference has no surrogate; this is the learned-surrogate workload that sits on top of the
batched generator (64^3 realisations here, parameters H, density multiplier, Gamma exponent and
level count drawn as in the ensemble configuration).

    python -m fastweavturb_b200.surrogate_experiment [--train 1024] [--N 64] [--steps 3000]

Prints one JSON line: data-generation and training times, the held-out prediction error
(against predicting the training mean), and for inverse fits to held-out draws the spectrum
and flatness errors and wall times of the surrogate-driven fit and of the same
generator-judged search started from random draws instead of the network's proposals, each
with the same number of generator runs, beside the error of the training set's mean
statistics (the fit that uses no information about the target).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=1024)
    ap.add_argument("--valid", type=int, default=64)
    ap.add_argument("--N", type=int, default=64)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--runs", type=int, default=24, help="generator runs of each fit")
    ap.add_argument("--targets", type=int, default=4, help="held-out target draws")
    args = ap.parse_args(argv)

    from .ensemble import Ensemble
    from .surrogate import Surrogate, draw_params, fit_error, fit_generator_only, fit_surrogate_driven, generate

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
    # inverse fits to held-out draws, the same generator budget with and without the network
    fits = []
    for k in range(args.targets):
        p_true = draw_params(np.random.default_rng(args.seed + 99 + k), 1)[0]
        seed_t = 424242 + k
        y_t, _ = generate(p_true[None, :], [seed_t], N=args.N, ens=ens)
        p_s, e_s, t_s, r_s = fit_surrogate_driven(sur, y_t[0], seed_t, args.runs, N=args.N, ens=ens)
        p_g, e_g, t_g, r_g = fit_generator_only(y_t[0], seed_t, args.runs, N=args.N, ens=ens, seed=k + 1)
        e_m = fit_error(Ytr.mean(axis=0), y_t[0])
        fits.append({"target": p_true.tolist(), "training_mean": {"err_logE": e_m[0], "err_flat": e_m[1]},
                     "surrogate": {"params": p_s.tolist(), "err_logE": e_s[0], "err_flat": e_s[1], "wall_s": t_s,
                                   "runs": r_s, "within_2pct": bool(max(e_s) <= 0.02)},
                     "generator_only": {"params": p_g.tolist(), "err_logE": e_g[0], "err_flat": e_g[1],
                                        "wall_s": t_g, "runs": r_g, "within_2pct": bool(max(e_g) <= 0.02)}})
    line = {
        "experiment": "surrogate", "N": args.N, "train": args.train, "valid": args.valid,
        "generation_s": t_gen, "generation_Mpts_per_s": len(P) * args.N ** 3 / dev_s / 1e6,
        "autotune": {str(k): v for k, v in ens.tuned.items()}, "train_s": t_train, "steps": args.steps,
        "loss_first": float(losses[0]), "loss_last": float(np.mean(losses[-50:])),
        "valid_rms_std_units": {"network": err_net, "training_mean": err_mean},
        "runs_per_fit": args.runs, "fits": fits,
        "mean_err": {"training_mean": float(np.mean([f["training_mean"]["err_logE"] + f["training_mean"]["err_flat"]
                                                      for f in fits])),
                     "surrogate": float(np.mean([f["surrogate"]["err_logE"] + f["surrogate"]["err_flat"] for f in fits])),
                     "generator_only": float(np.mean([f["generator_only"]["err_logE"] + f["generator_only"]["err_flat"]
                                                       for f in fits]))},
    }
    print(json.dumps(line))
    sur.close()
    ens.close()
    return line


if __name__ == "__main__":
    main()
