"""Checkpoint and resume: a solver (or batch) loaded from a checkpoint runs
the same iterations, bit for bit, as the one that saved it."""
import numpy as np
import pytest

from cvrp_aco_ocl_b200 import MODE_PARITY, MODE_THROUGHPUT, AcoError, Batch, Problem, Solver, default_params
from cvrp_aco_ocl_b200 import instances as I

pytestmark = pytest.mark.gpu


def params(n, A, mode, ls=1, **kw):
    p = default_params(n)
    p.mode, p.n_ants, p.ls_flag = mode, A, ls
    p.nn_ants, p.nn_ls = min(25, n - 2), min(25, n - 2)
    p.seed_time, p.rnd_seed = 1796300000, 8
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def state(S):
    sol, lens = S.solutions()
    tau, tot = S.pheromone()
    return sol, lens, tau, tot, S.seeds(), S.iteration(), [r[:2] for r in S.records()]


def same(a, b):
    for x, y in zip(a, b):
        if isinstance(x, np.ndarray):
            if not np.array_equal(x, y):
                return False
        elif x != y:
            return False
    return True


@pytest.mark.parametrize("mode,ls", [(MODE_PARITY, 1), (MODE_THROUGHPUT, 1), (MODE_THROUGHPUT, 3)])
def test_resume_is_bit_exact(gpu, tmp_path, mode, ls):
    inst = I.gen_mixed(12, 120)
    prob = Problem.from_instance(inst)
    path = str(tmp_path / "ck.bin")
    with Solver(prob, params(inst.n, 40, mode, ls)) as S:
        S.init()
        S.iterate(3)
        S.save_checkpoint(path)
        S.iterate(3)
        want = state(S)
    with Solver(prob, params(inst.n, 40, mode, ls)) as R:
        R.load_checkpoint(path)
        R.iterate(3)
        got = state(R)
    assert same(got, want)


def test_checkpoint_rejects_other_parameters_and_needs_init(gpu, tmp_path):
    inst = I.gen_mixed(13, 80)
    prob = Problem.from_instance(inst)
    path = str(tmp_path / "ck.bin")
    with Solver(prob, params(inst.n, 32, MODE_THROUGHPUT)) as S:
        with pytest.raises(AcoError):
            S.save_checkpoint(path)  # before init
        S.init()
        S.save_checkpoint(path)
    with Solver(prob, params(inst.n, 32, MODE_THROUGHPUT, rho=0.2)) as R, pytest.raises(AcoError):
        R.load_checkpoint(path)
    with Solver(prob, params(inst.n, 16, MODE_THROUGHPUT)) as R, pytest.raises(AcoError):
        R.load_checkpoint(path)
    with Solver(prob, params(inst.n, 32, MODE_THROUGHPUT)) as R, pytest.raises(AcoError):
        R.load_checkpoint(str(tmp_path / "missing.bin"))


def test_batch_resume_is_bit_exact(gpu, tmp_path):
    probs = [Problem.from_instance(I.gen_mixed(70 + k, m)) for k, m in enumerate([60, 140, 95])]
    path = str(tmp_path / "batch.bin")
    p = params(141, 24, MODE_THROUGHPUT)
    with Batch(probs, p) as B:
        B.init()
        B.iterate(2)
        B.save_checkpoint(path)
        B.iterate(2)
        want = [B.solutions(b) + B.pheromone(b) for b in range(3)]
    with Batch(probs, params(141, 24, MODE_THROUGHPUT)) as R:
        R.load_checkpoint(path)
        R.iterate(2)
        got = [R.solutions(b) + R.pheromone(b) for b in range(3)]
    assert all(np.array_equal(x, y) for g, w in zip(got, want) for x, y in zip(g, w))


def test_checkpoint_rejects_another_instance_seed_or_prior(gpu, tmp_path):
    """A checkpoint names the instance it was saved for (a hash of its data),
    its seeds, its stages and its prior: a solver for another instance of the
    same size, with other seeds, another local-search stage or another prior
    does not load it."""
    a, b = I.gen_mixed(21, 70), I.gen_mixed(22, 70)
    pa, pb = Problem.from_instance(a), Problem.from_instance(b)
    path = str(tmp_path / "ck.bin")
    with Solver(pa, params(a.n, 24, MODE_THROUGHPUT)) as S:
        S.init()
        S.save_checkpoint(path)
    for prob, kw in ((pb, {}), (pa, {"rnd_seed": 9}), (pa, {"ls_flag": 3})):
        with Solver(prob, params(a.n, 24, MODE_THROUGHPUT, **kw)) as R, pytest.raises(AcoError):
            R.load_checkpoint(path)
    with Solver(pa, params(a.n, 24, MODE_THROUGHPUT)) as R:  # prior set after the save: refused
        R.set_prior(np.full((a.n, a.n), 0.5, np.float32))
        with pytest.raises(AcoError):
            R.load_checkpoint(path)
        R.set_prior(None)  # back to the plain colony: accepted
        R.load_checkpoint(path)
