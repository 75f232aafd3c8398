"""Batched solving: many instances of uneven size served by the same launches.

Instance b of a batch must run exactly the iteration a single throughput-mode
solver with rnd_seed + b runs on it: tours, lengths, pheromone, total_info and
best-so-far are compared bit for bit, and one member is checked against the
oracle directly."""
import math

import numpy as np
import pytest

import oracle
from cvrp_aco_ocl_b200 import MODE_THROUGHPUT, AcoError, Batch, Problem, Solver, default_params
from cvrp_aco_ocl_b200 import instances as I

pytestmark = pytest.mark.gpu


def problem_of(inst, max_distance=math.inf, service_time=0.0):
    return Problem(name="b", x=np.asarray(inst.x, np.float32), y=np.asarray(inst.y, np.float32),
                   demand=np.asarray(inst.demand, np.int32), vehicle_capacity=int(inst.capacity),
                   max_distance=max_distance, service_time=service_time)


def batch_params(n, A, rs0, nn_ants=20, nn_ls=20, ls=True, **kw):
    p = default_params(n)
    p.mode = MODE_THROUGHPUT
    p.n_ants, p.nloc, p.seed_time, p.rnd_seed = A, 256, 1796300000, rs0
    p.nn_ants, p.nn_ls, p.ls_flag = nn_ants, nn_ls, int(ls)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def mixed_problems(seed, sizes):
    out = []
    for k, m in enumerate(sizes):
        inst = I.gen_mixed(seed + k, m) if m < 600 else I.gen_large(seed + k, m)
        out.append(problem_of(inst))
    return out


def assert_same(B, b, S):
    sb, lb = B.solutions(b)
    ss, ls_ = S.solutions()
    assert np.array_equal(sb, ss), f"solutions of instance {b}"
    assert np.array_equal(lb, ls_), f"lens of instance {b}"
    tb, xb = B.pheromone(b)
    ts, xs = S.pheromone()
    assert np.array_equal(tb, ts), f"tau of instance {b}"
    assert np.array_equal(xb, xs), f"total of instance {b}"
    bb, lbb = B.best(b)
    bs, lbs = S.best()
    assert np.array_equal(bb, bs) and lbb == lbs


@pytest.mark.parametrize("sizes,A,kw", [
    ([40, 120, 200, 75, 333, 64], 48, {}),   # uneven sizes, work items sorted by size
    ([100, 100, 100, 100], 128, {}),         # equal sizes
    ([700, 30, 999], 40, {}),                # one instance past the smem matrix limit
    # two construct CTAs per SM (tables of up to ~350 nodes staged, the rest read
    # through L2) against single solvers at one CTA per SM
    ([40, 120, 200, 75, 333, 64, 700, 999], 48, {"construct_ctas": 2}),
    ([150, 420, 1000], 96, {"construct_ctas": 2, "route_ls": 1}),
    # instances beyond 1024 nodes (register visited set off, candidate tables through L2) beside small ones
    ([1100, 300, 1500, 64], 40, {}),
])
def test_batch_members_match_single_solvers(gpu, sizes, A, kw):
    probs = mixed_problems(300 + len(sizes), sizes)
    rs0 = 9000 + A
    p = batch_params(max(pr.num_node for pr in probs), A, rs0, **kw)
    with Batch(probs, p) as B:
        assert B.size() == (len(probs), A * len(probs))
        if kw.get("construct_ctas") == 2:
            assert B.config()[2] & 8  # the two-CTA kernel runs
        B.init()
        B.iterate(3)
        for b, pr in enumerate(probs):
            with Solver(pr, batch_params(pr.num_node, A, rs0 + b)) as S:
                assert not S.config()[2] & 8
                S.init()
                S.iterate(3)
                assert_same(B, b, S)


def test_batch_route_level_2opt_matches_single_solvers(gpu):
    # the route list spans all instances of the batch; members still run exactly
    # the single solver's iteration (per-ant 2-opt kernel)
    probs = mixed_problems(420, [40, 120, 200, 75, 333])
    A, rs0 = 40, 777
    p = batch_params(max(pr.num_node for pr in probs), A, rs0, route_ls=1)
    with Batch(probs, p) as B:
        B.init()
        B.iterate(3)
        for b, pr in enumerate(probs):
            with Solver(pr, batch_params(pr.num_node, A, rs0 + b, route_ls=-1)) as S:
                S.init()
                S.iterate(3)
                assert_same(B, b, S)


def test_batch_member_matches_oracle(gpu):
    probs = mixed_problems(77, [150, 60, 90])
    A = 32
    with Batch(probs, batch_params(151, A, 555)) as B:
        B.init()
        B.iterate(2)
        for b in (0, 2):
            pr = probs[b]
            n = pr.num_node
            dist = oracle.compute_distances(pr.x, pr.y)
            nn = oracle.compute_nn_lists(dist, 20, 20)
            seeds, _ = oracle.make_seeds(1796300000, 555 + b, A, 256)
            O = oracle.Oracle(dist, pr.demand, pr.vehicle_capacity, A, 256, nn, seeds, ls_flag=True,
                              nn_ants_list=nn, n_threads=8)
            O.init_aco(throughput=True)
            O.run_iteration(throughput=True)
            O.run_iteration(throughput=True)
            sol, lens = B.solutions(b)
            assert np.array_equal(sol, O.solutions)
            assert np.array_equal(lens, O.lens)
            tau, tot = B.pheromone(b)
            assert np.array_equal(tau, O.tau) and np.array_equal(tot, O.total)


def test_batch_lists_clamped_per_instance(gpu):
    # nn_ls 30 is deeper than the 12-node instance allows; it is clamped to n-2 there
    probs = mixed_problems(5, [11, 150])
    A = 16
    with Batch(probs, batch_params(151, A, 71, nn_ants=20, nn_ls=30)) as B:
        B.init()
        B.iterate(2)
        with Solver(probs[0], batch_params(12, A, 71, nn_ants=10, nn_ls=10)) as S:
            S.init()
            S.iterate(2)
            assert_same(B, 0, S)
        with Solver(probs[1], batch_params(151, A, 72, nn_ants=20, nn_ls=30)) as S:
            S.init()
            S.iterate(2)
            assert_same(B, 1, S)


def test_batch_tours_valid(gpu):
    probs = mixed_problems(41, [50 + 37 * k for k in range(12)])
    A = 64
    with Batch(probs, batch_params(500, A, 1)) as B:
        B.init()
        B.iterate(4)
        for b, pr in enumerate(probs):
            sol, lens = B.solutions(b)
            T = 2 * pr.num_node
            dist = oracle.compute_distances(pr.x, pr.y)
            for a in range(0, A + 1, 7):
                t = sol[a * T:(a + 1) * T]
                t = t[: t[T - 1]]
                assert oracle.check_solution(dist, pr.demand, pr.vehicle_capacity, t)
                assert abs(oracle.tour_length_f64(dist, t) - float(lens[a])) <= 1e-5 * float(lens[a])


def test_batch_rejects_parity_mode_and_bad_instances(gpu):
    probs = mixed_problems(1, [50, 60])
    p = batch_params(61, 8, 1)
    p.mode = 0
    with pytest.raises(AcoError):
        Batch(probs, p)
    bad = mixed_problems(2, [40, 50])
    bad[1].demand[3] = bad[1].vehicle_capacity + 1  # a customer no vehicle can serve
    with pytest.raises(AcoError):
        Batch(bad, batch_params(51, 8, 1))


def test_pipelined_length_readback(gpu):
    # iteration k+1 is queued before the lengths of iteration k are read; every
    # read returns exactly the lengths a synchronous read gives after that iteration
    pr = mixed_problems(61, [150])[0]
    A = 64
    p = batch_params(pr.num_node, A, 5)
    with Solver(pr, p) as S, Solver(pr, batch_params(pr.num_node, A, 5)) as R:
        S.init(); R.init()
        tickets = []
        for k in range(6):
            S.enqueue(1)
            tickets.append(S.enqueue_lengths())
        want = []
        for k in range(6):
            R.iterate(1)
            want.append(R.solutions()[1])
        for k, t in enumerate(tickets[-4:]):  # four slots: the newest four tickets are readable
            assert np.array_equal(S.read_lengths(t), want[2 + k])
        with pytest.raises(AcoError):
            S.read_lengths(tickets[0])  # overwritten
