"""The oracle pinned to the reference: golden vectors produced by the
reference's own kernels (tests/golden/make_golden.py), the reference compiled
for the CPU where its sources exist, and known answers of the RNG."""
import math
import os

import numpy as np
import pytest

import oracle
from conftest import golden_cases, load_golden
from cvrp_aco_ocl_b200 import instances as I


def oracle_from_golden(g, n_threads=1):
    n, A, nloc, T0, rs0, ls, nn_ls, iters = (int(v) for v in g["meta"])
    seeds, _ = oracle.make_seeds(T0, rs0, A, nloc)
    nn = g["nn"][:, :nn_ls]
    O = oracle.Oracle(g["dist"], g["demand"], int(g["capacity"]), A, nloc, nn, seeds, ls_flag=bool(ls),
                      n_threads=n_threads)
    return O, iters


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_matches_reference_golden(case):
    g = load_golden(case)
    O, iters = oracle_from_golden(g)
    dist = oracle.compute_distances(g["x"], g["y"])
    assert np.array_equal(dist, g["dist"])
    assert O.init_aco() == 0
    for it in range(iters + 1):
        tag = "init" if it == 0 else f"it{it}"
        assert np.array_equal(O.seeds, g[f"{tag}_seeds"]), tag
        assert np.array_equal(O.solutions, g[f"{tag}_solutions"]), tag
        assert np.array_equal(O.lens, g[f"{tag}_lens"]), tag
        assert np.array_equal(O.tau, g[f"{tag}_tau"]), tag
        assert np.array_equal(O.total, g[f"{tag}_total"]), tag
        if it > 0:
            assert np.array_equal(O.elites, g[f"{tag}_elites"]), tag
        assert O.num_bsf == int(g[f"{tag}_num_bsf"][0])
        recs = O.record_list()
        assert [r[0] for r in recs] == list(g[f"{tag}_rec_iter"])
        assert np.array_equal(np.array([r[1] for r in recs], np.float32), g[f"{tag}_rec_len"])
        if it < iters:
            assert O.run_iteration() == 0


def test_oracle_threads_identical():
    g = load_golden("c1_ls")
    O1, _ = oracle_from_golden(g, 1)
    O4, _ = oracle_from_golden(g, 4)
    O1.init_aco(); O4.init_aco()
    for _ in range(2):
        O1.run_iteration(); O4.run_iteration()
    assert np.array_equal(O1.solutions, O4.solutions)
    assert np.array_equal(O1.tau, O4.tau)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference sources not built here")
@pytest.mark.parametrize("seed,nc,A,nloc,ls,nn_ls", [(21, 30, 17, 32, True, 0), (22, 45, 64, 64, False, 0),
                                                      (23, 90, 20, 128, True, 12)])
def test_oracle_matches_reference_live(tmp_path, seed, nc, A, nloc, ls, nn_ls):
    inst = I.gen_uniform_small(seed, nc) if nc < 60 else I.gen_mixed(seed, nc)
    p = str(tmp_path / "x.vrp")
    I.write_vrplib(inst, p)
    info = oracle.ref_read_instance(p)
    T0, rs0 = 1796300000 + seed, 1000 + seed
    seeds, _ = oracle.make_seeds(T0, rs0, A, nloc)
    with oracle.RefSession(p, A, nloc, T0, rs0, nn_ls=nn_ls, ls_flag=ls) as R:
        nn = info["nn"][:, :R.nn_ls]
        O = oracle.Oracle(info["dist"], inst.demand, inst.capacity, A, nloc, nn, seeds, ls_flag=ls)
        R.init_aco(); O.init_aco()
        for _ in range(4):
            R.run_iteration(); O.run_iteration()
            assert np.array_equal(R.read("solutions"), O.solutions)
            assert np.array_equal(R.read("pheromone", np.float32), O.tau)
            assert np.array_equal(R.read("seeds"), O.seeds)


def test_ran01_known_answers():
    # Park-Miller minimal standard: 16807^10000 from seed 1 is 1043618065 (Park & Miller 1988)
    s = 1
    for _ in range(10000):
        _, s = oracle.ran01(s)
    assert s == 1043618065
    # Schrage equals 16807 * (x mod m) mod m for any int, INT_MIN and m included
    m = 2**31 - 1
    for x in [0, 1, -1, 12345, -987654321, 2**31 - 1, -(2**31), 2**31 - 2, 127773, -127773]:
        _, got = oracle.ran01(x)
        assert got == (16807 * (x % m)) % m, x


def test_race_exp1_accuracy():
    # the throughput sampler's exponential clock -ln(u): within a few ulp (3e-7 absolute +
    # relative) of the true value over every draw ran01 can return, exact 0 at u = 1
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.integers(1, 2**31 - 1, 20000), [1, 2, 3, 2**31 - 2, 2**30, 2**31 - 64]])
    for x in xs:
        u = np.float32(np.float32(int(x)) * np.float32(4.656612873077392578125e-10))
        got = oracle.race_exp1(float(u))
        want = -float(np.log(np.float64(u)))
        assert got >= 0.0 and math.copysign(1.0, got) > 0  # +0, never -0 (the key orders bits)
        assert abs(got - want) <= 3e-7 + 3e-7 * abs(want), (x, got, want)
    assert oracle.race_exp1(1.0) == 0.0 and math.copysign(1.0, oracle.race_exp1(1.0)) > 0


def test_seed_formula_overflow_to_int_min():
    # (A-1)*A*A + T0 beyond 2^31 converts to INT_MIN like x86 cvttss2si (g_aco.cpp:718)
    seeds, _ = oracle.make_seeds(1796300000, 5, 1001, 32)
    assert (seeds == -(2**31)).any()
    assert oracle.lib().orc_f2i_x86(3.0e9) == -(2**31)
    assert oracle.lib().orc_f2i_x86(float("nan")) == -(2**31)
    assert oracle.lib().orc_f2i_x86(-2.5) == -2


def literal_tournament(vals):
    """kernel.cl:343-366 executed literally: returns the surviving index."""
    prob = list(vals)
    idx = list(range(len(vals)))
    offset = len(vals)
    while offset > 0:
        if offset % 2 != 0:
            if prob[offset - 1] > prob[0]:
                prob[0], idx[0] = prob[offset - 1], idx[offset - 1]
        offset //= 2
        for i in range(offset):
            if prob[i + offset] > prob[i]:
                prob[i], idx[i] = prob[i + offset], idx[i + offset]
    return idx[0]


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 31, 51, 64, 100, 201, 1001])
def test_tournament_priority_matches_literal_tree(n):
    prio = oracle.tournament_priority(n)
    assert sorted(prio) == list(range(n))
    rng = np.random.default_rng(n)
    for _ in range(300):
        vals = rng.integers(0, 3, size=n).astype(np.float32)  # heavy ties
        want = literal_tournament(vals)
        m = vals.max()
        tied = np.nonzero(vals == m)[0]
        got = tied[np.argmin(prio[tied])]
        assert got == want


def test_nn_lists_sort_tie_order():
    # integer grid: many equal distances, so the quicksort tie order matters
    inst = I.gen_uniform_small(3, 60, coord_max=6)
    d = oracle.compute_distances(inst.x, inst.y)
    nn = oracle.compute_nn_lists(d, 59, 59)
    assert nn.shape == (61, 59)
    for i in range(61):
        row = nn[i]
        assert 0 not in row and i not in row
        assert np.all(np.diff(d[i, row]) >= 0)


def test_check_solution_and_lengths():
    g = load_golden("c1_ls")
    n = int(g["meta"][0])
    T = 2 * n
    sol = g["it3_solutions"]
    for a in range(int(g["meta"][1]) + 1):
        t = sol[a * T:(a + 1) * T]
        tour = t[: t[T - 1]]
        assert oracle.check_solution(g["dist"], g["demand"], int(g["capacity"]), tour)
        assert oracle.tour_length(g["dist"], tour) == g["it3_lens"][a]
        assert abs(oracle.tour_length_f64(g["dist"], tour) - g["it3_lens"][a]) < 1e-3
    bad = np.array([0, 1, 1, 0], np.int32)
    assert not oracle.check_solution(g["dist"], g["demand"], int(g["capacity"]), bad)


def random_tours(inst, count, seed, dist=None):
    """Valid tours: customers in random order, cut into routes greedily by
    capacity and (given the distances) by the route-length limit."""
    import math
    rng = np.random.default_rng(seed)
    md = inst.max_distance if math.isfinite(inst.max_distance) else math.inf
    out = []
    for _ in range(count):
        order = rng.permutation(np.arange(1, inst.n))
        tour, load, rlen = [0], 0, 0.0
        for c in order:
            d = int(inst.demand[c])
            if dist is not None:
                prev = tour[-1]
                longer = rlen + dist[prev, c] + inst.service_time + dist[c, 0]
            else:
                longer = 0.0
            if load + d > inst.capacity or (tour[-1] != 0 and longer > md * 0.999):
                tour.append(0)
                load, rlen = 0, 0.0
            rlen += (dist[tour[-1], c] + inst.service_time) if dist is not None else 0.0
            tour.append(int(c))
            load += d
        tour.append(0)
        out.append(np.array(tour, np.int32))
    return out


@pytest.mark.skipif(not oracle.ref_available(), reason="reference sources not built here")
@pytest.mark.parametrize("seed,nc,max_distance,service", [(31, 40, None, 0.0), (32, 120, None, 0.0),
                                                          (33, 50, 400.0, 2.0)])
def test_swap_matches_reference_swap(tmp_path, seed, nc, max_distance, service):
    """The oracle's swap stage against the reference's own LocalSearch::swap."""
    import dataclasses
    import math
    inst = I.gen_uniform_small(seed, nc) if nc < 60 else I.gen_mixed(seed, nc)
    if max_distance is not None:
        inst = dataclasses.replace(inst, max_distance=max_distance, service_time=service)
    p = str(tmp_path / "x.vrp")
    I.write_vrplib(inst, p)
    info = oracle.ref_read_instance(p)
    md = inst.max_distance if math.isfinite(inst.max_distance) else math.inf
    changed = checked = 0
    for t in random_tours(inst, 16, seed, info["dist"]):
        if not oracle.check_solution(info["dist"], inst.demand, inst.capacity, t, md, inst.service_time):
            continue
        want = oracle.ref_swap(p, t)
        got, k = oracle.swap(info["dist"], inst.demand, inst.capacity, t, md, inst.service_time)
        assert np.array_equal(got, want)
        assert oracle.check_solution(info["dist"], inst.demand, inst.capacity, got, md, inst.service_time)
        checked += 1
        changed += int(k > 0)
    assert checked >= 4 and changed > 0


def test_random_restatement_matches_libc():
    """glibc random() (the generator NeighbourSearch draws from) restated."""
    import ctypes
    libc = ctypes.CDLL("libc.so.6")
    libc.random.restype = ctypes.c_long
    for seed in (1, 2, 12345, 2**31 - 1, 777777):
        libc.srandom(ctypes.c_uint(seed))
        want = [libc.random() for _ in range(500)]
        assert oracle.random_stream(seed, 500) == want


@pytest.mark.skipif(not oracle.ref_available(), reason="reference sources not built here")
@pytest.mark.parametrize("seed,nc,apply", [(41, 40, False), (42, 40, True), (43, 120, True)])
def test_neighbourhood_moves_match_reference(tmp_path, seed, nc, apply):
    """Proposals (type, validity, gain, positions) and applied moves of the
    restated NeighbourSearch against the reference's own code."""
    inst = I.gen_uniform_small(seed, nc) if nc < 60 else I.gen_mixed(seed, nc)
    p = str(tmp_path / "x.vrp")
    I.write_vrplib(inst, p)
    info = oracle.ref_read_instance(p)
    for k, t in enumerate(random_tours(inst, 3, seed, info["dist"])):
        want, wt = oracle.ref_ns_proposals(p, t, 1000 + k, 300, apply)
        got, gt = oracle.ns_proposals(info["dist"], inst.demand, inst.capacity, t, 1000 + k, 300, apply)
        assert got == want
        assert np.array_equal(gt, wt)
        if apply:
            assert oracle.check_solution(info["dist"], inst.demand, inst.capacity, gt)
