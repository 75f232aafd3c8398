"""Launch shapes and the autotuner on the device: every shape computes the
same tours and pheromone bit for bit, and the tuned configuration is one of
them."""
import numpy as np
import pytest

from cvrp_aco_ocl_b200 import MODE_PARITY, MODE_THROUGHPUT, Batch, Problem, Solver, default_params
from cvrp_aco_ocl_b200 import instances as I
from cvrp_aco_ocl_b200.tune import TuneTable, autotune, autotune_batch, build_table

pytestmark = pytest.mark.gpu


def params(n, A, mode, **kw):
    p = default_params(n)
    p.mode, p.n_ants, p.nn_ants, p.nn_ls = mode, A, min(25, n - 2), min(25, n - 2)
    p.seed_time, p.rnd_seed = 1796300000, 17
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def run(prob, p, iters=3):
    with Solver(prob, p) as S:
        S.init()
        S.iterate(iters)
        sol, lens = S.solutions()
        tau, tot = S.pheromone()
        return sol, lens, tau, tot


def same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("n_cust", [120, 400, 1100])
def test_throughput_shapes_identical(gpu, n_cust):
    prob = Problem.from_instance(I.gen_mixed(90 + n_cust, n_cust))
    n = prob.num_node
    ref = run(prob, params(n, 96, MODE_THROUGHPUT))
    # (ants per CTA, matrix staging, 2-opt warps, helper draws, route list, construct CTAs per SM)
    shapes = [(1, 0, 4, 1, -1, 0), (4, -1, 32, -1, 1, 1), (16, 0, 8, -1, -1, 2), (2, -1, 1, 1, 1, 0),
              (8, 0, 16, 1, -1, 0), (16, 0, 8, -1, 1, 2), (4, 0, 8, -1, -1, 2)]
    for apc, stage, lsw, draw, route, ctas in shapes[:4] if n > 1024 else shapes:
        with Solver(prob, params(n, 96, MODE_THROUGHPUT, ants_per_block=apc, stage_matrix=stage, ls_warps=lsw,
                                 draw_warps=draw, route_ls=route, construct_ctas=ctas)) as S:
            assert bool(S.config()[2] & 8) == (ctas == 2)
        got = run(prob, params(n, 96, MODE_THROUGHPUT, ants_per_block=apc, stage_matrix=stage, ls_warps=lsw,
                               draw_warps=draw, route_ls=route, construct_ctas=ctas))
        assert same(ref, got), (apc, stage, lsw, draw, route, ctas)


def test_parity_shapes_identical(gpu):
    prob = Problem.from_instance(I.gen_mixed(5, 150))
    n = prob.num_node
    ref = run(prob, params(n, 48, MODE_PARITY), iters=2)
    for apc, wpa, lsw in [(1, 8, 4), (4, 4, 16), (8, 2, 2)]:
        got = run(prob, params(n, 48, MODE_PARITY, ants_per_block=apc, warps_per_ant=wpa, ls_warps=lsw), iters=2)
        assert same(ref, got), (apc, wpa, lsw)


def test_invalid_shapes_rejected(gpu):
    from cvrp_aco_ocl_b200 import AcoError
    prob = Problem.from_instance(I.gen_mixed(6, 60))
    n = prob.num_node
    for kw in (dict(ls_warps=33), dict(stage_matrix=1), dict(mode=MODE_PARITY, ants_per_block=8, warps_per_ant=4),
               dict(construct_ctas=3), dict(construct_ctas=-1)):
        with pytest.raises(AcoError):
            Solver(prob, params(n, 32, kw.pop("mode", MODE_THROUGHPUT), **kw))


def test_autotune_single_and_result_unchanged(gpu):
    prob = Problem.from_instance(I.gen_mixed(7, 200))
    n = prob.num_node
    p = params(n, 200, MODE_THROUGHPUT)
    tuned, ms = autotune(prob, p, iters=2)
    assert ms > 0
    # 0 = the create-time model's choice, kept unless a candidate is reliably faster
    assert 0 <= tuned.ants_per_block <= 16 and tuned.stage_matrix in (0, -1) and 0 <= tuned.ls_warps <= 32
    assert same(run(prob, p), run(prob, tuned))


def test_autotune_parity(gpu):
    prob = Problem.from_instance(I.gen_mixed(8, 100))
    n = prob.num_node
    tuned, ms = autotune(prob, params(n, 64, MODE_PARITY), iters=1)
    assert tuned.warps_per_ant in (1, 2, 4, 8) and tuned.ants_per_block * tuned.warps_per_ant <= 16 and ms > 0


def test_autotune_batch_and_table(gpu, tmp_path):
    probs = [Problem.from_instance(I.gen_mixed(30 + k, m)) for k, m in enumerate([80, 150, 300, 120])]
    p = params(301, 32, MODE_THROUGHPUT)
    tuned, ms = autotune_batch(probs, p, iters=1)
    assert ms > 0 and tuned.ants_per_block >= 0  # 0: the create-time model kept
    t = build_table([61, 201], ants=32, iters=1)
    path = tmp_path / "tune.json"
    t.save(str(path))
    t2 = TuneTable.load(str(path))
    with Batch(probs, params(301, 32, MODE_THROUGHPUT), tune_table=t2) as B:
        B.init()
        B.iterate(1)
        assert B.status() == 0
