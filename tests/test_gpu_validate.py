"""Device validation of every tour slot, the solution writer and the batch's
best-so-far records."""
import numpy as np
import pytest

from cvrp_aco_ocl_b200 import MODE_PARITY, MODE_THROUGHPUT, Batch, Problem, Solver, default_params
from cvrp_aco_ocl_b200 import instances as I
from cvrp_aco_ocl_b200.aco import compute_distances, tour_length

pytestmark = pytest.mark.gpu


def params(n, A, mode=MODE_THROUGHPUT, **kw):
    p = default_params(n)
    p.mode, p.n_ants, p.nn_ants, p.nn_ls = mode, A, min(25, n - 2), min(25, n - 2)
    p.seed_time, p.rnd_seed = 1796300000, 21
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize("mode", [MODE_PARITY, MODE_THROUGHPUT])
def test_all_tours_valid_after_iterations(gpu, mode):
    inst = I.gen_mixed(3, 150)
    prob = Problem.from_instance(inst)
    with Solver(prob, params(inst.n, 48, mode)) as S:
        S.init()
        S.iterate(3)
        flags, bad = S.validate()
        assert bad == 0 and flags.tolist() == [1] * 49


def test_corrupted_slots_are_flagged(gpu):
    inst = I.gen_mixed(4, 80)
    prob = Problem.from_instance(inst)
    n, T, A = inst.n, 2 * inst.n, 16
    with Solver(prob, params(n, A)) as S:
        S.init()
        S.iterate(2)
        sol, lens = S.solutions()
        sol, lens = sol.copy(), lens.copy()
        t3 = sol[3 * T:4 * T]
        size3 = t3[T - 1]
        j = next(p for p in range(2, size3) if t3[p] != 0 and t3[p - 1] != 0)
        t3[j] = t3[j - 1]                         # ant 3: a customer twice (and one missing)
        lens[5] = np.nextafter(lens[5], np.float32(np.inf))  # ant 5: stored length off by one ulp
        t7 = sol[7 * T:8 * T]                     # ant 7: all customers in one route (over capacity)
        cust = [c for c in t7[:t7[T - 1]] if c != 0]
        one = np.array([0] + cust + [0], np.int32)
        t7[:] = 0
        t7[:len(one)] = one
        t7[T - 1] = len(one)
        d = compute_distances(inst.x, inst.y)
        lens[7] = tour_length(d, one)[0]
        S.set_state(solutions=sol, lens=lens)
        flags, bad = S.validate()
        assert bad == 3
        assert [a for a in range(A + 1) if flags[a] == 0] == [3, 5, 7]


def test_writer_block_format(gpu, tmp_path):
    inst = I.gen_mixed(5, 60)
    prob = Problem.from_instance(inst)
    with Solver(prob, params(inst.n, 32)) as S:
        S.init()
        S.iterate(2)
        tour, length = S.best()
        path = tmp_path / "best.sol"
        S.write_solution(str(path))
    lines = path.read_text().splitlines()
    assert lines[0] == "Begin Solution" and lines[-1] == "End Solution"
    assert [int(v) for v in lines[1].split()] == tour.tolist()
    d = compute_distances(inst.x, inst.y)
    assert lines[2] == "Solution Length %f" % tour_length(d, tour)[0]


def test_batch_validate_write_and_records(gpu, tmp_path):
    probs = [Problem.from_instance(I.gen_mixed(60 + k, m)) for k, m in enumerate([50, 120, 90])]
    with Batch(probs, params(121, 24)) as B:
        B.init()
        B.iterate(4)
        inv, bad = B.validate()
        assert bad == 0 and inv.tolist() == [0, 0, 0]
        path = tmp_path / "batch.sol"
        B.write_solutions(str(path))
        text = path.read_text()
        assert text.count("Begin Solution") == 3 and text.startswith("Instance 0\n")
        for b in range(3):
            recs = B.records(b)
            assert recs and recs[-1][1] == B.best(b)[1]
            assert all(r2[1] < r1[1] for r1, r2 in zip(recs, recs[1:]))
