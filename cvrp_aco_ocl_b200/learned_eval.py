"""Train the edge prior on colony-labelled instances and measure what it buys.

    python -m cvrp_aco_ocl_b200.learned_eval train --count 20000 --out prior.npz
    python -m cvrp_aco_ocl_b200.learned_eval eval --weights prior.npz --sizes 500,1000,1200 --out eval.json

Training set: generated instances with 100-500 nodes (mixed and large
generators alternately), each labelled with the best tour plain batched GPU
ACO finds in a fixed number of iterations.

Evaluation, per held-out instance (seeds disjoint from training): the plain
colony runs a fixed number of iterations; its final best length is the
target.  The learned colony (graph + network forward + prior upload counted in
its wall time) runs until it is within 1% of that target or has used the plain
colony's whole wall time.  Every best tour is rechecked for feasibility and
its length recomputed in FP64.
"""
from __future__ import annotations

import argparse
import json
import time
from typing import Dict, List

import numpy as np

from . import prior as PR
from ._lib import MODE_THROUGHPUT
from .aco import Problem, Solver, check_solution, default_params, tour_length
from . import instances as I

# Held-out instances use fixed seeds from here up; the training instances' seeds
# are drawn by gen_batch from its own random stream over [0, 2**31), so a
# coincidence has negligible probability.
EVAL_SEED = 900001


def colony_params(n: int, ants: int, nn_ants: int, seed: int):
    p = default_params(n)
    p.mode, p.n_ants, p.nn_ants, p.nn_ls = MODE_THROUGHPUT, ants, min(nn_ants, n - 2), min(25, n - 2)
    p.seed_time, p.rnd_seed = 1796300000, seed
    return p


def run_arm(prob: Problem, params, *, prior_fn=None, max_iters: int, step: int, target: float = 0.0,
            time_cap: float = float("inf")) -> Dict:
    """Iterate in blocks of `step`, recording (seconds, best length) after each;
    stop at max_iters, at best <= target, or past time_cap seconds."""
    t0 = time.perf_counter()
    pr = prior_fn() if prior_fn else None
    with Solver(prob, params) as S:
        if pr is not None:
            S.set_prior(pr)
        S.init()
        trace = [(time.perf_counter() - t0, S.best()[1], 0)]
        it = 0
        while it < max_iters:
            S.iterate(step)
            it += step
            t = time.perf_counter() - t0
            best = S.best()[1]
            trace.append((t, best, it))
            if (target > 0 and best <= target) or t >= time_cap:
                break
        tour, length = S.best()
    ok = check_solution(prob, tour)
    _, l64 = tour_length(prob.distance, tour)
    return {"trace": trace, "best": float(length), "best_fp64": float(l64), "feasible": bool(ok), "iters": it,
            "seconds": trace[-1][0]}


def time_to(trace, target: float):
    for t, b, _ in trace:
        if b <= target:
            return t
    return None


def held_out_instance(n: int, r: int):
    """Held-out instance r of n nodes (n - 1 customers): mixed generator for
    even r, large for odd r, seeds disjoint from the training set."""
    seed = EVAL_SEED + 1000 * n + r
    inst = I.gen_mixed(seed, n - 1) if r % 2 == 0 else I.gen_large(seed, n - 1)
    return seed, inst


def time_to_equal_cost(scorer: PR.EdgeScorer, n: int, count: int, plain_iters: int, ants: int, nn_ants: int,
                       gamma: float = PR.DEFAULT_GAMMA, step: int = 10, first: int = 0) -> Dict:
    """The metric's second half on `count` held-out instances of n nodes: the
    plain colony's best after `plain_iters` iterations, rechecked in FP64, is
    the target; the learned colony's wall time to come within 1% of it (graph
    build, network forward and prior upload inside that time), over the plain
    colony's wall time.  Both arms run `ants` ants on `nn_ants`-long candidate
    lists (2-opt on 25-NN lists).  Instances the learned colony does not reach
    within the plain colony's time count as ratio 1 in the median."""
    recs = []
    for r in range(first, first + count):
        seed, inst = held_out_instance(n, r)
        prob = Problem.from_instance(inst)
        from .aco import compute_distances
        prob.distance = compute_distances(prob.x, prob.y, prob.dis_type)
        plain = run_arm(prob, colony_params(n, ants, nn_ants, seed), max_iters=plain_iters, step=step)
        target = plain["best_fp64"] * 1.01
        learned = run_arm(prob, colony_params(n, ants, nn_ants, seed),
                          prior_fn=lambda: scorer.prior(prob, gamma=gamma),
                          max_iters=10 * plain_iters, step=step, target=target, time_cap=plain["seconds"])
        hit = time_to(learned["trace"], target)
        recs.append({"n": n, "seed": seed, "plain_best_fp64": plain["best_fp64"], "plain_seconds": plain["seconds"],
                     "plain_iters": plain["iters"], "target_fp64": target, "learned_seconds_to_target": hit,
                     "learned_best_fp64": learned["best_fp64"], "learned_iters": learned["iters"],
                     "feasible": plain["feasible"] and learned["feasible"],
                     "ratio": (hit / plain["seconds"]) if hit is not None else None})
    ratios = [x["ratio"] if x["ratio"] is not None else 1.0 for x in recs]
    return {"instances": recs, "median_ratio": float(np.median(ratios)) if ratios else None,
            "within_half_time": sum(1 for x in recs if x["ratio"] is not None and x["ratio"] <= 0.5),
            "count": len(recs), "all_feasible": all(x["feasible"] for x in recs)}


def evaluate(scorer: PR.EdgeScorer, sizes: List[int], per_size: int, plain_iters: int, ants: int, gamma: float,
             step: int = 10, log=print) -> Dict:
    out = {"config": {"sizes": sizes, "per_size": per_size, "plain_iters": plain_iters, "ants": ants,
                      "gamma": gamma, "plain_nn_ants": 25, "learned_nn_ants": PR.K_GRAPH}, "instances": []}
    for n in sizes:
        for r in range(per_size):
            seed = EVAL_SEED + 1000 * n + r
            inst = I.gen_mixed(seed, n - 1) if r % 2 == 0 else I.gen_large(seed, n - 1)
            prob = Problem.from_instance(inst)
            from .aco import compute_distances
            prob.distance = compute_distances(prob.x, prob.y, prob.dis_type)
            plain = run_arm(prob, colony_params(n, ants, 25, seed), max_iters=plain_iters, step=step)
            target = plain["best"] * 1.01
            learned = run_arm(prob, colony_params(n, ants, PR.K_GRAPH, seed),
                              prior_fn=lambda: scorer.prior(prob, gamma=gamma),
                              max_iters=10 * plain_iters, step=step, target=target, time_cap=plain["seconds"])
            t_plain_hit = time_to(plain["trace"], target)
            t_learn_hit = time_to(learned["trace"], target)
            half = plain["seconds"] / 2
            learned_at_half = min([b for t, b, _ in learned["trace"] if t <= half] or [float("inf")])
            rec = {"n": n, "seed": seed, "plain_best": plain["best"], "plain_seconds": plain["seconds"],
                   "plain_best_fp64": plain["best_fp64"], "target": target, "plain_time_to_target": t_plain_hit,
                   "learned_time_to_target": t_learn_hit, "learned_best": learned["best"],
                   "learned_best_fp64": learned["best_fp64"], "learned_best_at_half_time": learned_at_half,
                   "feasible": plain["feasible"] and learned["feasible"],
                   "ratio": (t_learn_hit / plain["seconds"]) if t_learn_hit is not None else None}
            out["instances"].append(rec)
            log(f"n={n} seed={seed}: plain {plain['best']:.1f} in {plain['seconds']:.2f}s; learned reaches "
                f"{target:.1f} at {t_learn_hit if t_learn_hit is None else round(t_learn_hit, 3)}s "
                f"(ratio {rec['ratio']}); learned best {learned['best']:.1f}")
    ratios = [x["ratio"] for x in out["instances"]]
    out["summary"] = {
        "met_1pct_within_half_time": sum(1 for x in ratios if x is not None and x <= 0.5),
        "instances": len(ratios),
        "median_ratio": float(np.median([x if x is not None else 1.0 for x in ratios])),
    }
    return out


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--count", type=int, default=20000)
    t.add_argument("--n-min", type=int, default=100)
    t.add_argument("--n-max", type=int, default=500)
    t.add_argument("--label-iters", type=int, default=100)
    t.add_argument("--epochs", type=int, default=10)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--graphs-per-step", type=int, default=32)
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--out", required=True)
    e = sub.add_parser("eval")
    e.add_argument("--weights", required=True)
    e.add_argument("--sizes", default="500,1000,1200")
    e.add_argument("--per-size", type=int, default=2)
    e.add_argument("--plain-iters", type=int, default=300)
    e.add_argument("--ants", type=int, default=256)
    e.add_argument("--gamma", type=float, default=PR.DEFAULT_GAMMA)
    e.add_argument("--out", required=True)
    a = ap.parse_args()
    if a.cmd == "train":
        t0 = time.perf_counter()
        graphs, labels, costs = PR.make_training_set(a.count, a.n_min, a.n_max, a.seed, a.label_iters, log=print)
        t1 = time.perf_counter()
        S = PR.EdgeScorer(seed=a.seed)
        hist = PR.train(S, graphs, labels, epochs=a.epochs, graphs_per_step=a.graphs_per_step, lr=a.lr, log=print)
        t2 = time.perf_counter()
        S.save(a.out, {"count": a.count, "n_min": a.n_min, "n_max": a.n_max, "label_iters": a.label_iters,
                       "epochs": a.epochs, "lr": a.lr, "loss": hist, "label_seconds": t1 - t0,
                       "train_seconds": t2 - t1})
        print(json.dumps({"label_seconds": t1 - t0, "train_seconds": t2 - t1, "loss": hist}))
    else:
        S = PR.EdgeScorer.load(a.weights)
        res = evaluate(S, [int(v) for v in a.sizes.split(",")], a.per_size, a.plain_iters, a.ants, a.gamma)
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
        print(json.dumps(res["summary"]))


if __name__ == "__main__":
    main()
