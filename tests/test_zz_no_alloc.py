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
TAU_RTOL = 1e-6  # the tolerance the parity tests use for the fp32 pheromone matrix


def close(a, b):
    return np.array_equal(a, b) or np.allclose(a, b, rtol=TAU_RTOL, atol=0)


@pytest.mark.parametrize("mode,nc,ants", [(0, 60, 24), (MODE_THROUGHPUT, 200, 64)])
def test_noalloc_update_matches_allocating_path(gpu, mode, nc, ants):
    import torch

    inst = I.gen_mixed(77, nc)
    prob = Problem.from_instance(inst)
    p = default_params(inst.n)
    p.n_ants, p.nloc, p.seed_time, p.rnd_seed, p.mode = ants, 64, 1796300000, 9, mode
    p.nn_ls, p.nn_ants = 20, 20
    n = inst.n
    dev = torch.device("cuda", 0)
    with Solver(prob, p) as S:
        S.init()
        S.construct()
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
        el_d = torch.zeros(6, dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream(dev)
        for call in range(2):
            rc = lib().aco_pheromone_update_noalloc(
                n, ld, ants, 6, ctypes.c_float(0.1), ctypes.c_float(1.0), ctypes.c_float(2.0),
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
