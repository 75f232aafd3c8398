"""Instance preprocessing on the device: distances and neighbour lists equal
to the host's (the reference's formulas and quicksort tie order), and
solvers built either way compute the same bits."""
import ctypes

import numpy as np
import pytest

from cvrp_aco_ocl_b200 import (MODE_PARITY, MODE_THROUGHPUT, Batch, Problem, Solver, compute_distances,
                               compute_nn_lists, default_params)
from cvrp_aco_ocl_b200 import instances as I
from cvrp_aco_ocl_b200._lib import check, lib

pytestmark = pytest.mark.gpu


def device_prep(x, y, dist_type, nn_ls, nn_ants):
    import torch
    n = len(x)
    ld = (n + 31) // 32 * 32
    dx = torch.tensor(np.asarray(x, np.float32), device="cuda")
    dy = torch.tensor(np.asarray(y, np.float32), device="cuda")
    dd = torch.zeros((n, ld), dtype=torch.float32, device="cuda")
    depth = ctypes.c_int()
    nn = torch.zeros(n * max(1, min(max(nn_ls, nn_ants), n - 1)), dtype=torch.int32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib().aco_compute_distances_device(n, dx.data_ptr(), dy.data_ptr(), dist_type, dd.data_ptr(), ld, st), "dist")
    check(lib().aco_compute_nn_lists_device(n, dd.data_ptr(), ld, nn_ls, nn_ants, nn.data_ptr(),
                                            ctypes.byref(depth), st), "nn")
    torch.cuda.synchronize()
    return dd[:, :n].cpu().numpy(), nn.cpu().numpy()[: n * depth.value].reshape(n, depth.value)


@pytest.mark.parametrize("maker,dist_type", [
    (lambda: I.gen_uniform_small(5), 0),        # integer coordinates: many equal distances
    (lambda: I.gen_uniform_small(6), 1),        # CEIL_2D
    (lambda: I.gen_uniform_small(7), 3),        # ATT
    (lambda: I.gen_mixed(8, 200), 0),
    (lambda: I.gen_large(9, 1000), 0),
])
def test_device_distances_and_lists_equal_host(gpu, maker, dist_type):
    inst = maker()
    n = inst.n
    host_d = compute_distances(inst.x, inst.y, dist_type)
    for nn_ls, nn_ants in ((25, 25), (10, 30), (n - 2, 25)):
        dev_d, dev_nn = device_prep(inst.x, inst.y, dist_type, nn_ls, nn_ants)
        assert np.array_equal(dev_d.view(np.uint32), host_d.view(np.uint32))
        assert np.array_equal(dev_nn, compute_nn_lists(host_d, nn_ls, nn_ants))


def test_device_lists_of_arbitrary_matrices(gpu):
    """The warp's fast path (distinct smallest values) and the quicksort fallback
    give the host's lists on matrices with negative values, -0, NaN and ties."""
    import torch
    rng = np.random.default_rng(5)
    n = 150
    ld = (n + 31) // 32 * 32
    cases = []
    m = rng.uniform(0, 100, (n, n)).astype(np.float32)
    cases.append(m.copy())                                   # distinct values: fast path on every row
    m2 = m.copy()
    m2[::3, 5] = -1.5                                        # negative entries
    m2[1::4, 7] = np.float32(-0.0)                           # -0 against +0
    m2[2::5, 9] = 0.0
    cases.append(m2)
    m3 = np.round(m / 10).astype(np.float32)                 # many ties
    cases.append(m3)
    m4 = m.copy()
    m4[::7, 11] = np.nan
    cases.append(m4)
    for hm in cases:
        dd = torch.zeros((n, ld), dtype=torch.float32, device="cuda")
        dd[:, :n] = torch.tensor(hm, device="cuda")
        depth = ctypes.c_int()
        nn = torch.zeros(n * 25, dtype=torch.int32, device="cuda")
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        check(lib().aco_compute_nn_lists_device(n, dd.data_ptr(), ld, 25, 25, nn.data_ptr(), ctypes.byref(depth),
                                                st), "nn")
        torch.cuda.synchronize()
        got = nn.cpu().numpy()[: n * depth.value].reshape(n, depth.value)
        assert np.array_equal(got, compute_nn_lists(hm, 25, 25))


def test_geo_is_left_to_the_host(gpu):
    from cvrp_aco_ocl_b200 import AcoError
    with pytest.raises(AcoError):
        device_prep([1.0, 2.0, 3.0], [1.0, 2.0, 3.0], 2, 1, 1)


def run(prob, p, iters=2):
    with Solver(prob, p) as S:
        S.init()
        S.iterate(iters)
        return S.solutions() + S.pheromone()


@pytest.mark.parametrize("mode", [MODE_PARITY, MODE_THROUGHPUT])
def test_solver_same_bits_with_device_or_host_prep(gpu, mode):
    inst = I.gen_uniform_small(11) if mode == MODE_PARITY else I.gen_mixed(12, 300)
    prob = Problem.from_instance(inst)
    outs = []
    for hp in (0, 1):
        p = default_params(inst.n)
        p.mode, p.n_ants, p.host_prep = mode, 40, hp
        p.nn_ants, p.nn_ls = min(25, inst.n - 2), min(25, inst.n - 2)
        p.seed_time, p.rnd_seed = 1796300000, 3
        outs.append(run(prob, p))
    assert all(np.array_equal(a, b) for a, b in zip(*outs))


def test_batch_same_bits_with_device_or_host_prep(gpu):
    probs = [Problem.from_instance(I.gen_mixed(40 + k, m)) for k, m in enumerate([90, 250, 140])]
    res = []
    for hp in (0, 1):
        p = default_params(251)
        p.mode, p.n_ants, p.host_prep, p.nn_ants, p.nn_ls = MODE_THROUGHPUT, 32, hp, 20, 20
        with Batch(probs, p) as B:
            B.init()
            B.iterate(2)
            res.append([B.solutions(b)[0] for b in range(3)])
    assert all(np.array_equal(a, b) for a, b in zip(*res))
