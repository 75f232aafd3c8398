"""Edge-scoring network on the device (tcgen05 BF16 kernels) against the FP64
oracle with the same BF16 operand rounding; the Adam step; training on
colony-labelled routes; the prior's effect on the colony."""
import math

import numpy as np
import pytest

from oracle import mpnn_oracle as M
from cvrp_aco_ocl_b200 import MODE_THROUGHPUT, Problem, Solver, default_params
from cvrp_aco_ocl_b200 import instances as I
from cvrp_aco_ocl_b200 import prior as PR

pytestmark = pytest.mark.gpu

SCORE_RTOL = 2e-3   # logits vs the bf16-emulating oracle (fp32 vs fp64 accumulation)
GRAD_RTOL = 2e-2    # per parameter block, relative L2 error of the gradient


def random_graphs(seed, sizes, k):
    rng = np.random.default_rng(seed)
    gs = []
    for n in sizes:
        nf = rng.uniform(0, 1, size=(n, M.F_NODE)).astype(np.float32)
        nbr = np.array([rng.choice([j for j in range(n) if j != i], size=k, replace=False) for i in range(n)],
                       np.int32).ravel()
        ef = rng.uniform(0, 1.5, size=n * k).astype(np.float32)
        gs.append(PR.Graph(n, k, nf, ef, nbr, None))
    return gs


def concat(gs):
    offs = np.cumsum([0] + [g.n for g in gs])
    nf = np.concatenate([g.node_feat for g in gs]).astype(np.float64)
    ef = np.concatenate([g.edge_feat for g in gs]).astype(np.float64)
    nbr = np.concatenate([g.nbr + o for g, o in zip(gs, offs[:-1])])
    return nf, ef, nbr


def block_errors(got, want):
    out = {}
    o = 0
    for name, sh in M.param_shapes():
        m = int(np.prod(sh))
        a, b = got[o:o + m], want[o:o + m]
        out[name] = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        o += m
    return out


@pytest.mark.parametrize("k,sizes", [(20, [37, 51]), (16, [64, 40]), (7, [30, 23, 90])])
def test_forward_matches_oracle(gpu, k, sizes):
    gs = random_graphs(k, sizes, k)
    flat = M.init_params(11)
    rng = np.random.default_rng(2)
    flat = (flat + rng.normal(0, 0.02, flat.shape)).astype(np.float32)
    S = PR.EdgeScorer(params=flat)
    got = S.scores(PR.GraphBatch(gs)).cpu().numpy()
    nf, ef, nbr = concat(gs)
    want, _ = M.forward(flat.astype(np.float64), nf, ef, nbr, k, bf16=True)
    assert np.max(np.abs(got - want)) <= SCORE_RTOL * (1.0 + np.max(np.abs(want)))


@pytest.mark.parametrize("k,sizes", [(20, [45, 33]), (16, [70]), (5, [40, 25])])
def test_gradient_matches_oracle(gpu, k, sizes):
    gs = random_graphs(100 + k, sizes, k)
    rng = np.random.default_rng(5)
    labels = [(rng.uniform(size=g.n * k) < 0.15).astype(np.float32) for g in gs]
    flat = M.init_params(3)
    flat = (flat + rng.normal(0, 0.02, flat.shape)).astype(np.float32)
    S = PR.EdgeScorer(params=flat)
    b = PR.GraphBatch(gs, labels)
    S.compute_grad(b, pos_weight=3.0)
    g_dev = S.grad.cpu().numpy().astype(np.float64)
    loss_dev = float(S.loss.item())
    nf, ef, nbr = concat(gs)
    s, saved = M.forward(flat.astype(np.float64), nf, ef, nbr, k, bf16=True)
    loss, ds = M.loss_and_dlogit(s, np.concatenate(labels), 3.0)
    g_orc = M.backward(flat.astype(np.float64), nf, ef, nbr, k, saved, ds, bf16=True)
    assert abs(loss_dev - loss) <= 1e-4 * (1 + abs(loss))
    errs = block_errors(g_dev, g_orc)
    bad = {kk: v for kk, v in errs.items() if not v <= GRAD_RTOL}
    assert not bad, bad


def test_adam_step_matches_numpy(gpu):
    import torch
    rng = np.random.default_rng(0)
    S = PR.EdgeScorer(seed=1)
    p0 = S.state().astype(np.float64)
    g = rng.normal(0, 1, S.count).astype(np.float32)
    S.grad.copy_(torch.from_numpy(g))
    m = np.zeros_like(p0); v = np.zeros_like(p0); p = p0.copy()
    for t in (1, 2):
        S.adam(1e-2)
        m = 0.9 * m + 0.1 * g
        v = 0.999 * v + 0.001 * g.astype(np.float64) ** 2
        p -= 1e-2 * (m / (1 - 0.9 ** t)) / (np.sqrt(v / (1 - 0.999 ** t)) + 1e-8)
    assert np.allclose(S.state(), p, rtol=1e-5, atol=1e-6)


def test_graph_features_and_labels():
    prob = Problem.from_instance(I.gen_mixed(3, 60))
    g = PR.build_graph(prob, 20)
    assert g.node_feat.shape == (61, 5) and g.nbr.shape == (61 * 20,)
    assert g.node_feat[0, 3] == 1 and g.node_feat[1:, 3].sum() == 0
    assert np.all(g.nbr != 0) and np.all(g.nbr != np.repeat(np.arange(61), 20))
    assert 0 <= g.node_feat[:, :2].min() and g.node_feat[:, :2].max() <= 1
    tour = np.concatenate([[0], np.arange(1, 61), [0]])
    y = PR.route_labels(g, tour)
    rows = np.repeat(np.arange(61), 20)
    for r, j, v in zip(rows, g.nbr, y):
        assert v == (1.0 if abs(int(r) - int(j)) == 1 else 0.0)


def test_uniform_prior_is_exact_and_removable(gpu):
    prob = Problem.from_instance(I.gen_mixed(9, 150))
    n = prob.num_node

    def params():
        p = default_params(n)
        p.mode, p.n_ants, p.nn_ants, p.nn_ls = MODE_THROUGHPUT, 64, 20, 20
        p.seed_time, p.rnd_seed = 1796300000, 5
        return p

    def run(prior=None, reset=False):
        with Solver(prob, params()) as S:
            if prior is not None:
                S.set_prior(prior)
            if reset:
                S.set_prior(None)
            S.init()
            S.iterate(3)
            return S.solutions()

    plain = run()
    ones = run(np.ones((n, n), np.float32))
    assert np.array_equal(plain[0], ones[0]) and np.array_equal(plain[1], ones[1])
    reset = run(np.full((n, n), 0.5, np.float32) + np.eye(n, dtype=np.float32), reset=True)
    assert np.array_equal(plain[0], reset[0])
    bad = np.ones((n, n), np.float32)
    bad[3, 4] = -1.0
    from cvrp_aco_ocl_b200 import AcoError
    with Solver(prob, params()) as S, pytest.raises(AcoError):
        S.set_prior(bad)


def test_training_lowers_loss_and_prior_gives_valid_tours(gpu):
    graphs, labels, costs = PR.make_training_set(48, 60, 120, seed=7, iters=20, ants=32, chunk=48)
    S = PR.EdgeScorer(seed=0)
    hist = PR.train(S, graphs, labels, epochs=6, graphs_per_step=8, lr=3e-3)
    assert hist[-1] < hist[0]
    prob = Problem.from_instance(I.gen_mixed(1234, 100))
    pr = S.prior(prob)
    assert pr.shape == (101, 101) and np.all(pr > 0)
    p = default_params(101)
    p.mode, p.n_ants, p.nn_ants, p.nn_ls = MODE_THROUGHPUT, 64, 20, 20
    from oracle import check_solution, compute_distances, tour_length_f64
    with Solver(prob, p) as SV:
        SV.set_prior(pr)
        SV.init()
        SV.iterate(5)
        tour, length = SV.best()
        d = compute_distances(prob.x, prob.y)
        assert check_solution(d, prob.demand, prob.vehicle_capacity, tour)
        assert abs(tour_length_f64(d, tour) - length) <= 1e-5 * length
