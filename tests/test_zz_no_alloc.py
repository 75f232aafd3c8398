"""aco_pheromone_update_noalloc against the allocating path.

The entry point is for callers that cannot let the library allocate device
memory (their memory manager owns it all, or their loop cannot take the
device-wide synchronisation of cudaMalloc / cudaFree).  The test hands it device
buffers it allocated itself (through torch), then checks two calls in a row
against aco_update_statistics + aco_pheromone_update of a solver holding the
same state, through the C ABI.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from cvrp_aco_ocl_b200 import MODE_THROUGHPUT, Problem, Solver, default_params
from cvrp_aco_ocl_b200 import instances as I
from cvrp_aco_ocl_b200._lib import lib

pytestmark = pytest.mark.gpu
# The allocating path applies the deposit in the same fixed elite order, so the
# two paths agree bit for bit; the parity tests' fp32 bar (1e-6 relative) is not
# needed here.


def close(a, b):
    return np.array_equal(a, b)


@pytest.mark.parametrize("mode,nc,ants,ranks,ls,alpha,beta", [
    (0, 60, 24, 6, 1, 1.0, 2.0),
    (MODE_THROUGHPUT, 200, 64, 6, 1, 1.0, 2.0),
    (MODE_THROUGHPUT, 150, 32, 6, 1, 1.5, 2.5),   # non-integer exponents: powf on both paths
    (MODE_THROUGHPUT, 120, 4, 8, 1, 1.0, 2.0),    # fewer ants than ranks - 1: repeated elites
    (MODE_THROUGHPUT, 4095, 12, 8, 0, 1.0, 2.0),  # n = 4096 with 8 ranks fills the scratch array
])
def test_noalloc_update_matches_allocating_path(gpu, mode, nc, ants, ranks, ls, alpha, beta):
    import torch

    inst = I.gen_mixed(77, nc)
    prob = Problem.from_instance(inst)
    p = default_params(inst.n)
    p.n_ants, p.nloc, p.seed_time, p.rnd_seed, p.mode = ants, 64, 1796300000, 9, mode
    p.nn_ls, p.nn_ants, p.ras_ranks, p.ls_flag, p.alpha, p.beta = 20, 20, ranks, ls, alpha, beta
    n = inst.n
    dev = torch.device("cuda", 0)
    with Solver(prob, p) as S:
        S.init()
        S.construct()
        if ls:
            S.local_search()
        S.update_statistics()  # best-so-far slot, elites, deposit lists of the allocating path
        tau0, _ = S.pheromone()
        sol, lens = S.solutions()
        dist = np.ascontiguousarray(prob_dist(inst), np.float32)
        # caller-owned device buffers: n rows, pitch ld > n to exercise the stride
        ld = n + 3
        def pitched(a):
            m = np.zeros((n, ld), np.float32)
            m[:, :n] = a.reshape(n, n)
            return torch.from_numpy(m).to(dev)
        tau_d, tot_d, dist_d = pitched(tau0), pitched(np.zeros(n * n, np.float32)), pitched(dist)
        sol_d = torch.from_numpy(sol).to(dev)
        lens_d = torch.from_numpy(lens).to(dev)
        el_d = torch.zeros(ranks, dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream(dev)
        for call in range(2):
            rc = lib().aco_pheromone_update_noalloc(
                n, ld, ants, ranks, ctypes.c_float(0.1), ctypes.c_float(alpha), ctypes.c_float(beta),
                ctypes.c_void_p(tau_d.data_ptr()), ctypes.c_void_p(tot_d.data_ptr()),
                ctypes.c_void_p(dist_d.data_ptr()), ctypes.c_void_p(sol_d.data_ptr()),
                ctypes.c_void_p(lens_d.data_ptr()), ctypes.c_void_p(el_d.data_ptr()),
                ctypes.c_void_p(stream.cuda_stream))
            assert rc == 0
            torch.cuda.synchronize(dev)
            S.pheromone_update()  # the existing entry point, same state
            want_tau, want_tot = S.pheromone()
            got_tau = tau_d.cpu().numpy()[:, :n].ravel()
            got_tot = tot_d.cpu().numpy()[:, :n].ravel()
            assert close(got_tau, want_tau), f"tau differs on call {call + 1}"
            assert close(got_tot, want_tot), f"total_info differs on call {call + 1}"
            assert np.array_equal(el_d.cpu().numpy(), S.elites())


def _update_np(tau, dist, sol, lens, n, ants, ranks, bad=()):
    """Evaporation, rank-based deposit in elite order and total_info for
    alpha = 1, beta = 2, in fp32 (kernel.cl:685-692,717-789); elites in `bad`
    deposit nothing."""
    f = np.float32
    T = 2 * n
    order = np.lexsort((np.arange(ants), lens[:ants]))  # ascending length, lowest index on ties
    elites = [ants] + [int(order[r - 1]) if r - 1 < ants else 0 for r in range(1, ranks)]
    v = (f(1.0) - f(0.1)) * tau.reshape(n, n)
    for r, e in enumerate(elites):
        if r in bad:
            continue
        d = f(ranks - r) / lens[e]
        tour = sol[e * T:(e + 1) * T]
        size = tour[T - 1]
        for k in range(size - 1):
            v[tour[k], tour[k + 1]] = v[tour[k], tour[k + 1]] + d
    eta = f(1.0) / (dist.reshape(n, n) + f(0.1))
    return v.ravel(), (v * (eta * eta)).ravel(), elites


def test_noalloc_rejects_malformed_elite_tours(gpu):
    """A caller's tour with a node id outside [0, n) or a size beyond 2n-1 is
    not read as indices: that elite deposits nothing and reads ACO_ERR_INVALID
    in elites_out; the other elites deposit as usual; nothing outside the
    scratch array is written."""
    import torch

    rng = np.random.default_rng(5)
    n, ants, ranks = 40, 10, 6
    T = 2 * n
    x, y = rng.uniform(0, 100, n).astype(np.float32), rng.uniform(0, 100, n).astype(np.float32)
    from cvrp_aco_ocl_b200 import compute_distances
    dist = compute_distances(x, y).astype(np.float32)
    sol = np.zeros(T * (ants + 1) + 1, np.int32)
    for a in range(ants + 1):
        perm = rng.permutation(np.arange(1, n)).astype(np.int32)
        tour = np.concatenate([[0], perm[:19], [0], perm[19:], [0]]).astype(np.int32)
        sol[a * T:a * T + tour.size] = tour
        sol[a * T + T - 1] = tour.size
    lens = rng.uniform(500, 900, ants + 1).astype(np.float32)
    lens[ants] = 400.0
    order = np.lexsort((np.arange(ants), lens[:ants]))
    e1, e3 = int(order[0]), int(order[2])
    sol[e1 * T + 5] = n + 7          # node id out of range in elite rank 1
    sol[e3 * T + T - 1] = T + 50     # tour size beyond 2n-1 in elite rank 3
    tau = rng.uniform(0.1, 1.0, n * n).astype(np.float32)
    want_tau, want_tot, elites = _update_np(tau, dist, sol, lens, n, ants, ranks, bad=(1, 3))
    dev = torch.device("cuda", 0)
    tau_d = torch.from_numpy(tau.copy()).to(dev)
    tot_d = torch.zeros(n * n, dtype=torch.float32, device=dev)
    dist_d, sol_d, lens_d = (torch.from_numpy(a).to(dev) for a in (dist.ravel(), sol, lens))
    el_d = torch.zeros(ranks, dtype=torch.int32, device=dev)
    rc = lib().aco_pheromone_update_noalloc(
        n, n, ants, ranks, ctypes.c_float(0.1), ctypes.c_float(1.0), ctypes.c_float(2.0),
        *(ctypes.c_void_p(t.data_ptr()) for t in (tau_d, tot_d, dist_d, sol_d, lens_d, el_d)), None)
    assert rc == 0
    torch.cuda.synchronize(dev)
    got_el = el_d.cpu().numpy()
    assert got_el[1] == -1 and got_el[3] == -1  # ACO_ERR_INVALID
    assert [int(got_el[r]) for r in (0, 2, 4, 5)] == [elites[r] for r in (0, 2, 4, 5)]
    assert np.array_equal(tau_d.cpu().numpy(), want_tau)
    assert np.allclose(tot_d.cpu().numpy(), want_tot, rtol=1e-6, atol=0)


def prob_dist(inst):
    from cvrp_aco_ocl_b200 import compute_distances
    return compute_distances(inst.x, inst.y)


def test_noalloc_rejects_sizes_beyond_scratch(gpu):
    import torch

    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float32, device=dev)
    ip = torch.zeros(16, dtype=torch.int32, device=dev)
    args = [ctypes.c_float(0.1), ctypes.c_float(1.0), ctypes.c_float(2.0)] + [ctypes.c_void_p(buf.data_ptr())] * 3 + \
        [ctypes.c_void_p(ip.data_ptr()), ctypes.c_void_p(buf.data_ptr()), None, None]
    assert lib().aco_pheromone_update_noalloc(4097, 4097, 8, 6, *args) == -10
    assert lib().aco_pheromone_update_noalloc(100, 100, 8, 9, *args) == -10
