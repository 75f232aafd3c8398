"""What the trained edge prior buys: on held-out instances (seeds outside the
training set) the colony with the shipped network's prior reaches shorter
FP64-checked tours than the plain colony after the same number of
iterations, and comes within 1% of the plain colony's final best in at most
half of its wall time (the metric's second half, here on a small case).  The
plain colony is the yardstick and the fallback."""
import numpy as np
import pytest

from cvrp_aco_ocl_b200 import MODE_THROUGHPUT, Problem, Solver, default_params
from cvrp_aco_ocl_b200 import instances as I
from cvrp_aco_ocl_b200 import prior as PR
from cvrp_aco_ocl_b200.aco import check_solution, compute_distances, tour_length

pytestmark = pytest.mark.gpu


def colony(n, nn_ants, seed):
    p = default_params(n)
    p.mode, p.n_ants, p.nn_ants, p.nn_ls = MODE_THROUGHPUT, 128, nn_ants, 25
    p.seed_time, p.rnd_seed = 1796300000, seed
    return p


def best_after(prob, params, iters, prior=None):
    with Solver(prob, params) as S:
        if prior is not None:
            S.set_prior(prior)
        S.init()
        S.iterate(iters)
        tour, length = S.best()
    assert check_solution(prob, tour)
    return tour_length(prob.distance, tour)[1]


def test_prior_beats_plain_at_equal_iterations(gpu):
    scorer = PR.EdgeScorer.load()
    plain, learned = [], []
    for r, seed in enumerate((770001, 770002, 770003)):
        inst = I.gen_mixed(seed, 399) if r % 2 == 0 else I.gen_large(seed, 399)
        prob = Problem.from_instance(inst)
        prob.distance = compute_distances(prob.x, prob.y)
        plain.append(best_after(prob, colony(400, 25, seed), 40))
        learned.append(best_after(prob, colony(400, PR.K_GRAPH, seed), 40, scorer.prior(prob)))
    gains = [(p - l) / p for p, l in zip(plain, learned)]
    assert sum(g > 0 for g in gains) >= 2, gains
    assert np.mean(gains) > 0.005, gains


def test_time_to_equal_cost_gate_small_case(gpu):
    """Held-out n = 500 instances, 128 ants, 25-NN lists in both arms; the plain
    colony runs 300 iterations and its FP64-rechecked best (+1%) is the target;
    the learned colony's clock includes graph build, network forward and prior
    upload.  Gate: median time ratio <= 0.5, every tour feasible."""
    from cvrp_aco_ocl_b200.learned_eval import time_to_equal_cost
    res = time_to_equal_cost(PR.EdgeScorer.load(), 500, 3, 300, 128, 25)
    assert res["all_feasible"], res
    assert res["median_ratio"] is not None and res["median_ratio"] <= 0.5, res

