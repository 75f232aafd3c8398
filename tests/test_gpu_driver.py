"""The driver loop (main.cpp:80-88 with termination_condition, main.cpp:29-34)
through aco_run and the Python GACO.run, and the bounded device waits.

The termination tests stop a run at max_iteration, at max_runtime and at an
optimum equal to a best-so-far length the same seeds reach mid-run.  The
reference compares a best_so_far_ant that is only refreshed at exit, so its
optimum stop cannot fire mid-run; both drivers here compare the live
best-so-far instead.

The timeout tests make the construct's staging wait give up on its first poll
(aco_params.wait_limit = 1), check that the call reports ACO_ERR_TIMEOUT, and
that the same solver then runs on, bit-identical to a fresh one, once the limit
is restored and the status cleared.  No wait here can hang: the copies a timed
out wait leaves in flight are drained under the default bound.
"""
import ctypes
import time

import numpy as np
import pytest

from cvrp_aco_ocl_b200 import GACO, MODE_PARITY, MODE_THROUGHPUT, Batch, Problem, Solver, default_params
from cvrp_aco_ocl_b200 import instances as I
from cvrp_aco_ocl_b200._lib import lib

pytestmark = pytest.mark.gpu
ACO_ERR_TIMEOUT = -12


def params(inst, mode=MODE_THROUGHPUT, **kw):
    p = default_params(inst.n)
    p.n_ants, p.nloc, p.seed_time, p.rnd_seed, p.mode = 32, 64, 1796300000, 77, mode
    p.nn_ls, p.nn_ants = 20, 20
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def test_aco_run_stops_at_max_iteration(gpu):
    inst = I.gen_mixed(5, 80)
    with Solver(Problem.from_instance(inst), params(inst, max_iteration=9)) as S:
        S.init()
        it0 = S.iteration()
        done = S.run(0.0)
        assert S.iteration() == 9
        assert done == 9 - it0


def test_aco_run_stops_at_max_runtime(gpu):
    inst = I.gen_mixed(6, 300)
    p = params(inst, max_iteration=10**8, max_runtime=0.25, n_ants=128)
    with Solver(Problem.from_instance(inst), p) as S:
        S.init()
        t0 = time.perf_counter()
        done = S.run(0.0)
        dt = time.perf_counter() - t0
        assert done >= 1
        assert dt < 5.0  # the elapsed time since init reached 0.25 s, and the run stopped soon after
        assert S.iteration() < 10**8


@pytest.mark.parametrize("mode", [MODE_PARITY, MODE_THROUGHPUT])
def test_aco_run_stops_at_live_optimum(gpu, mode):
    """A second solver with the same seeds stops at the first iteration whose
    best-so-far is within 10*EPSILON of the optimum: the iteration at which the
    first solver recorded that length."""
    inst = I.gen_mixed(7, 60)
    prob = Problem.from_instance(inst)
    with Solver(prob, params(inst, mode, max_iteration=40)) as S:
        S.init()
        S.iterate(30)
        recs = S.records()  # (iteration, length, seconds) whenever the best-so-far improved
    assert len(recs) >= 2
    _, len_k, _ = recs[-1]  # the last improvement: reached mid-run
    # the first record within 10*EPSILON of it is where the second run must stop
    it_first = min(it for it, ln, _ in recs if abs(ln - len_k) < 0.01)
    assert it_first < 30
    with Solver(prob, params(inst, mode, max_iteration=40)) as S2:
        S2.init()
        S2.run(float(len_k))
        assert S2.iteration() in (it_first, it_first + 1)
        _, best = S2.best()
        assert abs(best - len_k) < 0.01
    # an optimum no run reaches: the run ends at max_iteration
    with Solver(prob, params(inst, mode, max_iteration=12)) as S3:
        S3.init()
        S3.run(1.0)
        assert S3.iteration() == 12


def test_gaco_run_terminates_like_the_driver_loop(gpu):
    inst = I.gen_mixed(8, 60)
    prob = Problem.from_instance(inst)
    prob.max_iteration, prob.n_ants, prob.nn_ls = 11, 24, 20
    g = GACO(prob, nloc=64, seed_time=1796300000, mode=MODE_THROUGHPUT, nn_ants=20)
    assert g.run() == 11
    assert prob.best_length < float("inf")
    # runtime bound
    prob2 = Problem.from_instance(inst)
    prob2.max_iteration, prob2.max_runtime, prob2.n_ants, prob2.nn_ls = 10**8, 0.2, 24, 20
    t0 = time.perf_counter()
    g2 = GACO(prob2, nloc=64, seed_time=1796300000, mode=MODE_THROUGHPUT, nn_ants=20)
    g2.run()
    assert time.perf_counter() - t0 < 10.0 and prob2.iteration > 1
    # optimum: the best a first run reached; the second run stops when it reaches it again
    prob3 = Problem.from_instance(inst)
    prob3.max_iteration, prob3.n_ants, prob3.nn_ls = 25, 24, 20
    g3 = GACO(prob3, nloc=64, seed_time=1796300000, mode=MODE_THROUGHPUT, nn_ants=20)
    g3.run()
    recs = g3.solver.records()
    target_it, target_len, _ = recs[-1]
    prob4 = Problem.from_instance(inst)
    prob4.max_iteration, prob4.n_ants, prob4.nn_ls, prob4.optimum = 25, 24, 20, float(target_len)
    g4 = GACO(prob4, nloc=64, seed_time=1796300000, mode=MODE_THROUGHPUT, nn_ants=20)
    g4.run()
    assert prob4.iteration <= target_it + 1
    assert abs(prob4.best_length - target_len) < 0.01


def test_construct_wait_timeout_is_reported_and_recoverable(gpu):
    inst = I.gen_mixed(9, 150)
    prob = Problem.from_instance(inst)
    with Solver(prob, params(inst, wait_limit=1)) as S, Solver(prob, params(inst)) as R:
        assert lib().aco_init(S.h) == ACO_ERR_TIMEOUT  # the bootstrap construct gave up on its staging wait
        S.set_wait_limit(0)
        S.init()  # init starts from a cleared status
        R.init()
        S.iterate(3)
        R.iterate(3)
        assert np.array_equal(S.solutions()[0], R.solutions()[0])
        assert np.array_equal(S.pheromone()[0], R.pheromone()[0])
        # a timed-out iteration (graph replay): reported, cleared, and the solver goes on
        S.set_wait_limit(1)
        assert lib().aco_iterate(S.h, 1) == ACO_ERR_TIMEOUT
        assert S.clear_status() == ACO_ERR_TIMEOUT
        assert S.status() == 0
        S.set_wait_limit(0)
        S.iterate(2)
        flags, bad = S.validate()
        assert bad == 0 and flags.all()


def test_batch_wait_timeout_is_reported(gpu):
    insts = [I.gen_mixed(20 + b, 100 + 40 * b) for b in range(4)]
    probs = [Problem.from_instance(x) for x in insts]
    p = params(insts[-1], wait_limit=1)
    B = Batch(probs, p)
    try:
        assert lib().aco_batch_init(B.h) == ACO_ERR_TIMEOUT
    finally:
        B.close()
    with Batch(probs, params(insts[-1])) as B2:  # the device stays usable
        B2.init()
        B2.iterate(2)
        inv, bad = B2.validate()
        assert bad == 0
