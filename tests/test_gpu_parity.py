"""CUDA path vs the reference (golden vectors from its own kernels) and vs the
oracle, through the C ABI.  Routes, lengths, seeds, elites, best-so-far records
and 2-opt results are compared bit for bit; the fp32 pheromone and total_info
matrices too (the deposit order is fixed, so they agree exactly; the reference's
own bar is 1e-6 relative)."""
import math

import numpy as np
import pytest

import oracle
from conftest import golden_cases, load_golden
from cvrp_aco_ocl_b200 import MODE_PARITY, MODE_THROUGHPUT, AcoError, Problem, Solver, default_params
from cvrp_aco_ocl_b200 import instances as I

pytestmark = pytest.mark.gpu
TAU_RTOL = 1e-6  # north-star tolerance for the fp32 pheromone matrix


def problem_of(x, y, demand, capacity, max_distance=math.inf, service_time=0.0):
    return Problem(name="t", x=np.asarray(x, np.float32), y=np.asarray(y, np.float32),
                   demand=np.asarray(demand, np.int32), vehicle_capacity=int(capacity),
                   max_distance=max_distance, service_time=service_time)


def params_for(n, A, nloc, T0, rs0, ls, nn_ls, mode=MODE_PARITY, **kw):
    p = default_params(n)
    p.n_ants, p.nloc, p.seed_time, p.rnd_seed = A, nloc, T0, rs0
    p.ls_flag, p.nn_ls, p.mode = int(ls), nn_ls, mode
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def assert_tau_close(got, want):
    assert np.array_equal(got, want) or np.allclose(got, want, rtol=TAU_RTOL, atol=0)


def compare_state(S, O_or_g, tag=None):
    sol, lens = S.solutions()
    tau, tot = S.pheromone()
    if tag is None:
        O = O_or_g
        want = dict(solutions=O.solutions, lens=O.lens, tau=O.tau, total=O.total, seeds=O.seeds)
    else:
        g = O_or_g
        want = dict(solutions=g[f"{tag}_solutions"], lens=g[f"{tag}_lens"], tau=g[f"{tag}_tau"],
                    total=g[f"{tag}_total"], seeds=g[f"{tag}_seeds"])
    assert np.array_equal(sol, want["solutions"]), "solutions"
    assert np.array_equal(lens, want["lens"]), "lens"
    assert np.array_equal(S.seeds(), want["seeds"]), "seeds"
    assert_tau_close(tau, want["tau"])
    assert_tau_close(tot, want["total"])


@pytest.mark.parametrize("case", golden_cases())
def test_iterations_match_reference_golden(gpu, case):
    g = load_golden(case)
    n, A, nloc, T0, rs0, ls, nn_ls, iters = (int(v) for v in g["meta"])
    prob = problem_of(g["x"], g["y"], g["demand"], int(g["capacity"]))
    with Solver(prob, params_for(n, A, nloc, T0, rs0, ls, nn_ls)) as S:
        S.init()
        for it in range(iters + 1):
            tag = "init" if it == 0 else f"it{it}"
            compare_state(S, g, tag)
            if it > 0:
                assert np.array_equal(S.elites(), g[f"{tag}_elites"])
            recs = S.records()
            assert [r[0] for r in recs] == list(g[f"{tag}_rec_iter"])
            assert np.array_equal(np.array([r[1] for r in recs], np.float32), g[f"{tag}_rec_len"])
            assert S.iteration() == it + 1
            if it < iters:
                S.iterate(1)


def build_pair(inst, A, nloc, T0, rs0, ls, nn_ls, mode=MODE_PARITY, nn_ants=0, **kw):
    prob = problem_of(inst.x, inst.y, inst.demand, inst.capacity)
    n = inst.n
    extra = dict(kw)
    if mode == MODE_THROUGHPUT:
        extra["nn_ants"] = nn_ants
    S = Solver(prob, params_for(n, A, nloc, T0, rs0, ls, nn_ls, mode=mode, **extra))
    dist = oracle.compute_distances(inst.x, inst.y)
    depth = max(nn_ls, nn_ants)
    nn = oracle.compute_nn_lists(dist, depth, depth) if depth > 0 else np.zeros((n, 0), np.int32)
    seeds, _ = oracle.make_seeds(T0, rs0, A, nloc)
    O = oracle.Oracle(dist, inst.demand, inst.capacity, A, nloc, nn[:, :nn_ls], seeds, ls_flag=ls,
                      nn_ants_list=nn[:, :nn_ants] if nn_ants else None, n_threads=8,
                      ls_pass_limit=kw.get("ls_pass_limit", 4096))
    return S, O


@pytest.mark.parametrize("wpa", [1, 2, 4, 8])
def test_construct_parity_warps_per_ant(gpu, wpa):
    inst = I.gen_mixed(101, 200)
    S, O = build_pair(inst, 40, 256, 1700001234, 77, False, 0, warps_per_ant=wpa, ants_per_block=2)
    with S:
        S.init(); O.init_aco()
        compare_state(S, O)
        S.iterate(2); O.run_iteration(); O.run_iteration()
        compare_state(S, O)


@pytest.mark.parametrize("n_cust,A,nloc,ls,nn_ls", [
    (200, 200, 256, True, 199),   # n=201 A=200 with the reference's full 2-opt lists
    (200, 64, 64, True, 25),
    (333, 48, 128, True, 30),
    (1000, 32, 256, True, 30),    # full-row parity at n=1001 (smem matrix does not fit)
])
def test_full_iterations_vs_oracle(gpu, n_cust, A, nloc, ls, nn_ls):
    inst = I.gen_mixed(7 + n_cust, n_cust) if n_cust < 1000 else I.gen_large(3, n_cust)
    S, O = build_pair(inst, A, nloc, 1796300000 + n_cust, 1234, ls, nn_ls)
    with S:
        S.init(); O.init_aco()
        compare_state(S, O)
        for _ in range(2):
            S.iterate(1); O.run_iteration()
            compare_state(S, O)
        assert np.array_equal(S.elites(), O.elites)


@pytest.mark.parametrize("draw", [-1, 1])  # the ant's warp draws / a helper warp draws ahead
def test_throughput_mode_vs_oracle(gpu, draw):
    inst = I.gen_mixed(5, 200)
    S, O = build_pair(inst, 100, 256, 1796300000, 4321, True, 25, mode=MODE_THROUGHPUT, nn_ants=25,
                      draw_warps=draw)
    with S:
        S.init(); O.init_aco(throughput=True)
        compare_state(S, O)
        for _ in range(3):
            S.iterate(1); O.run_iteration(throughput=True)
            compare_state(S, O)


@pytest.mark.parametrize("draw", [-1, 1])
def test_throughput_route_length_limit_vs_oracle(gpu, draw):
    """max_distance and service time: the candidate test adds the route-length
    check (finite-limit kernels) in both draw arrangements."""
    inst = I.gen_mixed(23, 150)
    dist = oracle.compute_distances(inst.x, inst.y)
    A, nloc, T0, rs = 64, 256, 1796300000, 515
    maxd, serv = float(np.max(dist[0]) * 2.6), 3.0
    prob = problem_of(inst.x, inst.y, inst.demand, inst.capacity, max_distance=maxd, service_time=serv)
    p = params_for(inst.n, A, nloc, T0, rs, True, 25, mode=MODE_THROUGHPUT, nn_ants=25, draw_warps=draw)
    nn = oracle.compute_nn_lists(dist, 25, 25)
    seeds, _ = oracle.make_seeds(T0, rs, A, nloc)
    O = oracle.Oracle(dist, inst.demand, inst.capacity, A, nloc, nn, seeds, ls_flag=True, nn_ants_list=nn,
                      max_dist=maxd, serv_time=serv, n_threads=8, ls_pass_limit=4096)
    with Solver(prob, p) as S:
        S.init(); O.init_aco(throughput=True)
        compare_state(S, O)
        for _ in range(2):
            S.iterate(1); O.run_iteration(throughput=True)
            compare_state(S, O)
        assert S.validate()[1] == 0


@pytest.mark.parametrize("per_route,n_cust,A,nn_ls", [(12.0, 200, 100, 25), (45.0, 200, 40, 25), (2.0, 150, 24, 25),
                                                     (300.0, 600, 12, 25), (45.0, 200, 40, 60)])
def test_route_level_2opt_vs_oracle(gpu, per_route, n_cust, A, nn_ls):
    """route_ls = 1: the construct lists every route of at most 255 nodes and one
    persistent kernel improves them, in registers up to 32 nodes (12 customers
    a route), through the route-local path beyond (45 customers a route; with
    2-opt lists of 25 entries both searches of an examination come from one load
    of the list, with 60 entries they run one after the other); many short
    routes (2 customers a route) fill the list; an ant with a route of more than
    255 nodes (300 customers a route) lists none and goes to the per-ant kernel.
    Same bits as the oracle and as the per-ant kernel alone."""
    inst = I.gen_mixed(900 + n_cust, n_cust, customers_per_route=per_route)
    S, O = build_pair(inst, A, 256, 1796300000, 93, True, nn_ls, mode=MODE_THROUGHPUT, nn_ants=25, route_ls=1)
    p2 = params_for(inst.n, A, 256, 1796300000, 93, True, nn_ls, mode=MODE_THROUGHPUT, nn_ants=25, route_ls=-1)
    prob = problem_of(inst.x, inst.y, inst.demand, inst.capacity)
    with S, Solver(prob, p2) as S2:
        S.init(); S2.init(); O.init_aco(throughput=True)
        compare_state(S, O)
        for _ in range(3):
            S.iterate(1); S2.iterate(1); O.run_iteration(throughput=True)
            compare_state(S, O)
            a, b = S.solutions(), S2.solutions()
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("A,ranks", [(1100, 8), (4, 6), (1, 3)])
def test_elites_many_and_few_ants(gpu, A, ranks):
    """get_elites with more ants than one pass of the statistics block (knock-out
    rounds) and with fewer ants than ranks (rounds past the last finite length
    take index 0)."""
    inst = I.gen_mixed(31, 40)
    n = inst.n
    dist = oracle.compute_distances(inst.x, inst.y)
    nn = oracle.compute_nn_lists(dist, 20, 20)
    seeds, _ = oracle.make_seeds(1796300000, 77, A, 256)
    prob = problem_of(inst.x, inst.y, inst.demand, inst.capacity)
    p = params_for(n, A, 256, 1796300000, 77, True, 20, mode=MODE_THROUGHPUT, nn_ants=20, ras_ranks=ranks)
    O = oracle.Oracle(dist, inst.demand, inst.capacity, A, 256, nn, seeds, ls_flag=True, nn_ants_list=nn,
                      ras_ranks=ranks, n_threads=8, ls_pass_limit=4096)
    with Solver(prob, p) as S:
        S.init(); O.init_aco(throughput=True)
        compare_state(S, O)
        for _ in range(2):
            S.iterate(1); O.run_iteration(throughput=True)
            compare_state(S, O)


@pytest.mark.parametrize("draw", [-1, 1])
def test_throughput_large_no_smem_matrix(gpu, draw):
    inst = I.gen_large(11, 1000)
    S, O = build_pair(inst, 48, 256, 1796300000, 99, True, 30, mode=MODE_THROUGHPUT, nn_ants=30, draw_warps=draw)
    with S:
        S.init(); O.init_aco(throughput=True)
        compare_state(S, O)
        S.iterate(1); O.run_iteration(throughput=True)
        compare_state(S, O)


def test_tours_valid_and_fp64_recheck(gpu):
    inst = I.gen_mixed(21, 200)
    S, O = build_pair(inst, 64, 256, 1796300000, 5, True, 25)
    with S:
        S.init()
        S.iterate(5)
        sol, lens = S.solutions()
        dist = oracle.compute_distances(inst.x, inst.y)
        for a in range(65):
            t = S.tour(sol, a)
            assert oracle.check_solution(dist, inst.demand, inst.capacity, t)
            assert abs(oracle.tour_length_f64(dist, t) - float(lens[a])) <= 1e-5 * float(lens[a])
        best, blen = S.best()
        assert blen == lens[64]
        assert blen <= lens[:64].min() + 1e-3


def test_phase_entry_points_match_oracle(gpu):
    """construct / local_search / update_statistics / pheromone_update one at a time."""
    inst = I.gen_mixed(31, 120)
    S, O = build_pair(inst, 30, 128, 1796300000, 17, True, 20)
    with S:
        S.init(); O.init_aco()
        S.construct(); O.construct()
        compare_state(S, O)
        S.local_search(); O.local_search()
        compare_state(S, O)
        S.update_statistics(); O.find_best(); O.update_best_so_far(0.0)
        O.get_elites()
        sol, lens = S.solutions()
        assert np.array_equal(sol, O.solutions) and np.array_equal(lens, O.lens)
        assert np.array_equal(S.elites(), O.elites)
        S.pheromone_update(); O.evaporation(); O.deposit(); O.compute_total_info()
        compare_state(S, O)


def test_random_pheromone_state_construct(gpu):
    """construct from an arbitrary (seeded random) pheromone matrix, including
    exact ties between candidates."""
    inst = I.gen_uniform_small(8, 80)
    S, O = build_pair(inst, 24, 64, 1796300000, 3, False, 0)
    rng = np.random.default_rng(0)
    n = inst.n
    tot = rng.choice(np.array([0.25, 0.5, 1.0], np.float32), size=n * n).astype(np.float32)
    with S:
        S.init(); O.init_aco()
        S.set_state(total=tot)
        O.total[:] = tot
        S.construct(); O.construct()
        compare_state(S, O)


def test_step_limit_is_reported_not_hung(gpu):
    """All-zero choice_info: every step returns to the depot; the reference
    would loop forever (kernel.cl:438,461).  The kernel stops after 2n-3
    steps with ACO_ERR_STEP_LIMIT, like the oracle."""
    inst = I.gen_uniform_small(4, 20)
    S, O = build_pair(inst, 8, 32, 1, 2, False, 0)
    with S:
        S.init(); O.init_aco()
        z = np.zeros(inst.n * inst.n, np.float32)
        S.set_state(total=z)
        O.total[:] = z
        with pytest.raises(AcoError) as ei:
            S.construct()
        assert ei.value.code == -7
        assert O.construct() == -7
        sol, lens = S.solutions()
        assert np.array_equal(lens[:8], O.lens[:8])


def test_infeasible_instance_rejected(gpu):
    inst = I.gen_uniform_small(4, 20)
    dem = inst.demand.copy()
    dem[5] = inst.capacity + 1
    prob = problem_of(inst.x, inst.y, dem, inst.capacity)
    with pytest.raises(AcoError) as ei:
        Solver(prob, params_for(inst.n, 8, 32, 1, 2, False, 0))
    assert ei.value.code == -2


def test_ls_pass_limit_reports_like_oracle(gpu):
    """A route that is still improving when its pass budget runs out reports
    ACO_ERR_LS_LIMIT (the oracle reports the same status).  Tours stay valid;
    they are not matched bit for bit on this error path (routes run in parallel
    and the depot's don't-look bit is only fixed for converged routes)."""
    inst = I.gen_mixed(41, 150)
    S, O = build_pair(inst, 20, 64, 1796300000, 8, True, 30, ls_pass_limit=1)
    with S:
        try:
            S.init()
            code = 0
        except AcoError as e:
            code = e.code
        ocode = O.init_aco()
        assert code == ocode == -8
        sol, lens = S.solutions()
        dist = oracle.compute_distances(inst.x, inst.y)
        for a in range(20):
            t = S.tour(sol, a)
            assert oracle.check_solution(dist, inst.demand, inst.capacity, t)
            assert lens[a] == oracle.tour_length(dist, t)


def test_two_solvers_independent(gpu):
    a = I.gen_uniform_small(1, 50)
    b = I.gen_mixed(2, 100)
    S1, O1 = build_pair(a, 16, 64, 10, 20, True, 49)
    S2, O2 = build_pair(b, 16, 64, 11, 21, True, 25)
    with S1, S2:
        S1.init(); S2.init(); O1.init_aco(); O2.init_aco()
        S1.iterate(1); S2.iterate(2); O1.run_iteration(); O2.run_iteration(); O2.run_iteration()
        compare_state(S1, O1)
        compare_state(S2, O2)


@pytest.mark.parametrize("mode", [MODE_PARITY, MODE_THROUGHPUT])
def test_integer_exponents_and_many_ranks(gpu, mode):
    """alpha=2, beta=3, rho=0.2 and 10 elite ranks: the general exponent path of
    the row pass and the deposit of ranks beyond the eighth."""
    inst = I.gen_mixed(61, 150)
    n, A, nloc, T0, rs0 = inst.n, 48, 256, 1796300000, 313
    prob = problem_of(inst.x, inst.y, inst.demand, inst.capacity)
    p = params_for(n, A, nloc, T0, rs0, True, 20, mode=mode, alpha=2.0, beta=3.0, rho=0.2, ras_ranks=10)
    if mode == MODE_THROUGHPUT:
        p.nn_ants = 20
    dist = oracle.compute_distances(inst.x, inst.y)
    nn = oracle.compute_nn_lists(dist, 20, 20)
    seeds, _ = oracle.make_seeds(T0, rs0, A, nloc)
    O = oracle.Oracle(dist, inst.demand, inst.capacity, A, nloc, nn, seeds, ls_flag=True, alpha=2.0, beta=3.0,
                      rho=0.2, ras_ranks=10, nn_ants_list=nn if mode == MODE_THROUGHPUT else None, n_threads=8)
    thr = mode == MODE_THROUGHPUT
    with Solver(prob, p) as S:
        S.init(); O.init_aco(throughput=thr)
        compare_state(S, O)
        for _ in range(3):
            S.iterate(1); O.run_iteration(throughput=thr)
            compare_state(S, O)
        assert np.array_equal(S.elites(), O.elites)


@pytest.mark.parametrize("draw", [-1, 1])
def test_throughput_candidate_table_in_global_memory(gpu, draw):
    """n=1201 with 25-candidate lists: the table does not fit in shared memory
    and is read through L2; results stay bit-exact."""
    inst = I.gen_large(17, 1200)
    S, O = build_pair(inst, 32, 256, 1796300000, 8, True, 25, mode=MODE_THROUGHPUT, nn_ants=25, draw_warps=draw)
    with S:
        S.init(); O.init_aco(throughput=True)
        compare_state(S, O)
        S.iterate(1); O.run_iteration(throughput=True)
        compare_state(S, O)


@pytest.mark.parametrize("mode,n_cust,A", [(MODE_PARITY, 100, 48), (MODE_THROUGHPUT, 200, 64),
                                           (MODE_THROUGHPUT, 600, 32)])
def test_swap_stage_vs_oracle(gpu, mode, n_cust, A):
    """ls_flag = 3: 2-opt then the inter-route swap of the CPU local search."""
    inst = I.gen_mixed(400 + n_cust, n_cust) if n_cust < 500 else I.gen_large(400 + n_cust, n_cust)
    S, O = build_pair(inst, A, 256, 1796300000, 55, 3, 25, mode=mode,
                      nn_ants=25 if mode == MODE_THROUGHPUT else 0)
    thr = mode == MODE_THROUGHPUT
    with S:
        S.init(); O.init_aco(throughput=thr)
        compare_state(S, O)
        for _ in range(2):
            S.iterate(1); O.run_iteration(throughput=thr)
            compare_state(S, O)
        flags, bad = S.validate()
        assert bad == 0


@pytest.mark.parametrize("mode,n_cust,A,ls", [(MODE_PARITY, 80, 32, 1), (MODE_THROUGHPUT, 200, 64, 3),
                                              (MODE_THROUGHPUT, 150, 48, 0)])
def test_random_descent_stage_vs_oracle(gpu, mode, n_cust, A, ls):
    """ns_rounds > 0: the reference's random neighbourhood moves after the local search."""
    inst = I.gen_mixed(600 + n_cust, n_cust)
    n, nloc, T0, rs0, rounds = inst.n, 256, 1796300000, 77, 40
    prob = problem_of(inst.x, inst.y, inst.demand, inst.capacity)
    p = params_for(n, A, nloc, T0, rs0, ls, 25, mode=mode, ns_rounds=rounds)
    if mode == MODE_THROUGHPUT:
        p.nn_ants = 25
    dist = oracle.compute_distances(inst.x, inst.y)
    nn = oracle.compute_nn_lists(dist, 25, 25)
    seeds, _ = oracle.make_seeds(T0, rs0, A, nloc)
    O = oracle.Oracle(dist, inst.demand, inst.capacity, A, nloc, nn, seeds, ls_flag=ls,
                      nn_ants_list=nn if mode == MODE_THROUGHPUT else None, n_threads=8,
                      ns_rounds=rounds, ns_seed=rs0)
    thr = mode == MODE_THROUGHPUT
    with Solver(prob, p) as S:
        S.init(); O.init_aco(throughput=thr)
        compare_state(S, O)
        for _ in range(3):
            S.iterate(1); O.run_iteration(throughput=thr)
            compare_state(S, O)
        assert S.validate()[1] == 0


@pytest.mark.parametrize("per_route,n_cust,A", [(12.0, 200, 64), (45.0, 200, 40), (8.0, 700, 48)])
def test_fused_2opt_matches_oracle_and_separate_kernel(gpu, per_route, n_cust, A):
    """The construct kernel improving routes as they complete (fuse_ls = 1) gives
    the bits of the separate 2-opt kernel (fuse_ls = 0) and of the oracle; with
    45 customers a route, routes longer than 32 nodes go to the 2-opt kernel."""
    inst = I.gen_mixed(700 + n_cust, n_cust, customers_per_route=per_route)
    S, O = build_pair(inst, A, 256, 1796300000, 91, True, 25, mode=MODE_THROUGHPUT, nn_ants=25, fuse_ls=1)
    p2 = params_for(inst.n, A, 256, 1796300000, 91, True, 25, mode=MODE_THROUGHPUT, nn_ants=25, fuse_ls=0)
    prob = problem_of(inst.x, inst.y, inst.demand, inst.capacity)
    with S, Solver(prob, p2) as S2:
        S.init(); S2.init(); O.init_aco(throughput=True)
        compare_state(S, O)
        for _ in range(3):
            S.iterate(1); S2.iterate(1); O.run_iteration(throughput=True)
            compare_state(S, O)
            a, b = S.solutions(), S2.solutions()
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
