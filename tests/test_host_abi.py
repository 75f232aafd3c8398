"""Host side of the boundary (no GPU needed): the C ABI loads and exports every
symbol include/cvrp_aco.h declares, and the host routines behind it (VRPLIB
reader, distances, NN lists, seeds, validation) match the oracle and the
reference's own host code."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

import oracle
from conftest import ROOT, has_gpu, load_golden
from cvrp_aco_ocl_b200 import (AcoError, Problem, check_solution, compute_distances, compute_nn_lists,
                               default_params, init_problem, make_seeds, read_instance_file, tour_length)
from cvrp_aco_ocl_b200 import _lib
from cvrp_aco_ocl_b200 import instances as I

REF_DATASET = os.path.join(os.environ.get("CVRP_REFERENCE_DIR", "/root/reference"), "dataset")


def header_symbols():
    src = open(os.path.join(ROOT, "include", "cvrp_aco.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(aco_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(_lib.EXPORTED) == syms


def test_strerror_and_defaults():
    L = _lib.lib()
    assert L.aco_strerror(0) == b"ok"
    assert b"step" in L.aco_strerror(-7)
    p = default_params(51)
    assert (p.n_ants, p.nn_ls, p.ras_ranks, p.nloc, p.max_iteration, p.ls_flag) == (51, 49, 6, 256, 250, 1)
    assert abs(p.rho - 0.1) < 1e-7 and p.alpha == 1.0 and p.beta == 2.0


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_create_without_device_reports_no_device():
    inst = I.gen_uniform_small(1, 10)
    prob = Problem.from_instance(inst)
    from cvrp_aco_ocl_b200 import Solver
    with pytest.raises(AcoError) as ei:
        Solver(prob)
    assert ei.value.code == -4


def test_invalid_params_rejected_before_device():
    inst = I.gen_uniform_small(1, 10)
    prob = Problem.from_instance(inst)
    from cvrp_aco_ocl_b200 import Solver
    for field, val in [("nloc", 48), ("nloc", 2048), ("ras_ranks", 0), ("ras_ranks", 33), ("nn_ls", 10),
                       ("warps_per_ant", 3), ("rho", 0.0), ("ls_ants", 9), ("ls_ants", -1), ("draw_warps", 2),
                       ("draw_warps", -2), ("route_ls", 2), ("fuse_ls", 2), ("ls_flag", 2), ("ns_rounds", -1)]:
        p = default_params(inst.n)
        setattr(p, field, val)
        with pytest.raises(AcoError) as ei:
            Solver(prob, p)
        assert ei.value.code == -1, field
    dem = inst.demand.copy()
    dem[3] = inst.capacity + 5
    bad = Problem.from_instance(inst)
    bad.demand = dem
    with pytest.raises(AcoError) as ei:
        Solver(bad)
    assert ei.value.code == -2


@pytest.mark.parametrize("seed,nc", [(1, 50), (2, 200), (3, 500)])
def test_distances_and_nn_lists_match_oracle(seed, nc):
    inst = I.gen_mixed(seed, nc)
    d = compute_distances(inst.x, inst.y)
    assert np.array_equal(d, oracle.compute_distances(inst.x, inst.y))
    for depth in (25, nc - 1):
        assert np.array_equal(compute_nn_lists(d, depth, depth), oracle.compute_nn_lists(d, depth, depth))


def test_nn_lists_ties_match_oracle():
    inst = I.gen_uniform_small(5, 120, coord_max=8)  # many equal distances
    d = compute_distances(inst.x, inst.y)
    assert np.array_equal(compute_nn_lists(d, 119, 119), oracle.compute_nn_lists(d, 119, 119))


@pytest.mark.parametrize("dt", [1, 2, 3])
def test_other_distance_types_match_oracle(dt):
    inst = I.gen_uniform_small(9, 40, coord_max=90)
    x = inst.x + np.float32(0.37)
    assert np.array_equal(compute_distances(x, inst.y, dt), oracle.compute_distances(x, inst.y, dt))


@pytest.mark.parametrize("T0,rs,A,nloc", [(1796300000, 12345, 50, 256), (0, 1, 7, 32), (1796300000, 5, 1001, 32),
                                          (-5, -77, 13, 64)])
def test_seeds_match_oracle(T0, rs, A, nloc):
    got, rs_got = make_seeds(T0, rs, A, nloc)
    want, rs_want = oracle.make_seeds(T0, rs, A, nloc)
    assert np.array_equal(got, want) and rs_got == rs_want


def test_reader_roundtrip_and_checks(tmp_path):
    inst = I.gen_mixed(4, 60)
    inst.max_distance = 5000.0
    inst.service_time = 2.5
    p = str(tmp_path / "a.vrp")
    I.write_vrplib(inst, p)
    prob = read_instance_file(p)
    assert prob.num_node == inst.n and prob.vehicle_capacity == inst.capacity
    assert np.array_equal(prob.x, inst.x) and np.array_equal(prob.y, inst.y)
    assert np.array_equal(prob.demand, inst.demand)
    assert prob.max_distance == np.float32(5000.0) and prob.service_time == np.float32(2.5)
    init_problem(prob)
    assert prob.n_ants == inst.n and prob.nn_ls == inst.n - 2
    g = load_golden("c1_ls")
    gp = Problem(name="g", x=g["x"], y=g["y"], demand=g["demand"], vehicle_capacity=int(g["capacity"]))
    n = int(g["meta"][0])
    sol = g["it3_solutions"]
    t = sol[:2 * n][: sol[2 * n - 1]]
    assert check_solution(gp, t)
    l32, l64 = tour_length(g["dist"], t)
    assert l32 == g["it3_lens"][0] and abs(l64 - l32) < 1e-3
    assert not check_solution(gp, np.array([0, 1, 2, 0], np.int32))


def test_reader_errors(tmp_path):
    p = tmp_path / "bad.vrp"
    p.write_text("NAME : x\nTYPE : TSP\nDIMENSION : 3\n")
    with pytest.raises(AcoError) as ei:
        read_instance_file(str(p))
    assert ei.value.code == -11
    with pytest.raises(AcoError):
        read_instance_file(str(tmp_path / "missing.vrp"))
    p.write_text("NAME : x\nTYPE : CVRP\nDIMENSION : 3\nCAPACITY : 5\nNODE_COORD_SECTION\n1 0 0\n2 1 1\n3 2 2\nEOF\n")
    with pytest.raises(AcoError):
        read_instance_file(str(p))  # no DEMAND_SECTION: the reference loops forever here


@pytest.mark.skipif(not (oracle.ref_available() and os.path.isdir(REF_DATASET)), reason="reference not present")
@pytest.mark.parametrize("rel", ["CMT/CMT1.vrp", "CMT/CMT6.vrp", "Golden/Golden_1.vrp", "Li/Li_21.vrp",
                                 "X/X-n101-k25.vrp"])
def test_reader_matches_reference_reader(rel):
    path = os.path.join(REF_DATASET, rel)
    if not os.path.exists(path):
        pytest.skip("instance missing")
    want = oracle.ref_read_instance(path)
    got = read_instance_file(path)
    assert got.num_node == want["n"] and got.vehicle_capacity == want["capacity"]
    assert np.array_equal(got.x, want["x"]) and np.array_equal(got.y, want["y"])
    assert np.array_equal(got.demand, want["demand"])
    assert got.optimum == np.float32(want["optimum"])
    assert got.max_distance == np.float32(want["max_distance"])
    assert got.service_time == np.float32(want["service_time"])
    d = compute_distances(got.x, got.y, got.dis_type)
    assert np.array_equal(d, want["dist"])
    nn = compute_nn_lists(d, got.num_node - 2, got.num_node - 2)
    assert np.array_equal(nn, want["nn"])
