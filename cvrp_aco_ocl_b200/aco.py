"""Python mirror of the reference's driver surface over the C ABI.

``Problem`` / ``read_instance_file`` / ``init_problem`` follow
cvrp_ocl/problem.h:82-140, io.cpp:334-517 and problem.cpp:43-56,186-220;
``GACO`` follows the g_ACO class (cvrp_ocl/gpu/g_aco.h:16-37) with the same
method names; ``termination_condition`` and ``run`` follow main.cpp:29-34,68-92.
All computation happens in libcvrp_aco.so on the GPU; errors raise
``AcoError`` instead of exiting the process.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import time
from typing import List, Optional, Tuple

import numpy as np

from . import _lib
from ._lib import AcoError, AcoInstance, AcoParams, AcoRecord, check, lib, ptr
from .instances import Instance

EPSILON = 0.001  # utilities.h:19


@dataclasses.dataclass
class Problem:
    """The fields of ``Problem`` (problem.h:82-140) the path uses, plus the
    parameter globals alpha/beta/rho/ras_ranks (problem.h:30-33)."""

    name: str
    x: np.ndarray
    y: np.ndarray
    demand: np.ndarray
    vehicle_capacity: int
    max_distance: float = math.inf
    service_time: float = 0.0
    dis_type: int = 0
    optimum: float = 0.0
    # set_default_parameters (problem.cpp:186-220)
    n_ants: int = 0
    nn_ants: int = 0
    nn_ls: int = 0
    ls_flag: bool = True
    max_iteration: int = 250
    max_runtime: float = 600.0
    rnd_seed: int = 0
    alpha: float = 1.0
    beta: float = 2.0
    rho: float = 0.1
    ras_ranks: int = 6
    iteration: int = 0
    distance: Optional[np.ndarray] = None
    nn_list: Optional[np.ndarray] = None
    best_tour: Optional[np.ndarray] = None
    best_length: float = math.inf

    @property
    def num_node(self) -> int:
        return int(self.x.shape[0])

    @classmethod
    def from_instance(cls, inst: Instance) -> "Problem":
        return cls(name=inst.name, x=inst.x, y=inst.y, demand=inst.demand, vehicle_capacity=inst.capacity,
                   max_distance=inst.max_distance, service_time=inst.service_time, dis_type=inst.dist_type,
                   optimum=inst.optimum)

    def c_instance(self) -> Tuple[AcoInstance, list]:
        keep = [np.ascontiguousarray(self.x, np.float32), np.ascontiguousarray(self.y, np.float32),
                np.ascontiguousarray(self.demand, np.int32)]
        ci = AcoInstance(self.num_node, keep[0].ctypes.data, keep[1].ctypes.data, keep[2].ctypes.data,
                         int(self.vehicle_capacity), float(self.max_distance), float(self.service_time),
                         int(self.dis_type), None)
        if self.distance is not None:
            d = np.ascontiguousarray(self.distance, np.float32)
            keep.append(d)
            ci.dist = d.ctypes.data
        return ci, keep


def read_instance_file(path: str) -> Problem:
    """read_instance_file (io.cpp:334-517) through aco_read_vrplib."""
    L = lib()
    n = ctypes.c_int(0)
    check(L.aco_read_vrplib(path.encode(), ctypes.byref(n), None, None, None, None, None, None, None, None,
                            None, 0), "read_instance_file")
    N = n.value
    x = np.zeros(N, np.float32)
    y = np.zeros(N, np.float32)
    dem = np.zeros(N, np.int32)
    cap, dt = ctypes.c_int(), ctypes.c_int()
    md, st, opt = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    name = ctypes.create_string_buffer(256)
    check(L.aco_read_vrplib(path.encode(), ctypes.byref(n), ptr(x), ptr(y), ptr(dem), ctypes.byref(cap),
                            ctypes.byref(md), ctypes.byref(st), ctypes.byref(dt), ctypes.byref(opt), name, 256),
          "read_instance_file")
    return Problem(name=name.value.decode(), x=x, y=y, demand=dem, vehicle_capacity=cap.value,
                   max_distance=md.value, service_time=st.value, dis_type=dt.value, optimum=opt.value)


def compute_distances(x, y, dist_type: int = 0) -> np.ndarray:
    """compute_distances (vrpHelper.cpp:160-184)."""
    xs = np.ascontiguousarray(x, np.float32)
    ys = np.ascontiguousarray(y, np.float32)
    n = xs.shape[0]
    d = np.zeros((n, n), np.float32)
    check(lib().aco_compute_distances(n, ptr(xs), ptr(ys), dist_type, ptr(d)), "compute_distances")
    return d


def compute_nn_lists(dist: np.ndarray, nn_ls: int, nn_ants: int) -> np.ndarray:
    """compute_nn_lists (vrpHelper.cpp:188-236)."""
    d = np.ascontiguousarray(dist, np.float32)
    n = d.shape[0]
    depth = max(nn_ls, nn_ants)
    depth = min(depth, n - 1)
    out = np.zeros(n * max(depth, 1), np.int32)
    got = ctypes.c_int()
    check(lib().aco_compute_nn_lists(n, ptr(d), nn_ls, nn_ants, ptr(out), ctypes.byref(got)), "compute_nn_lists")
    return out[: n * got.value].reshape(n, got.value)


def set_default_parameters(p: Problem) -> None:
    """set_default_parameters (problem.cpp:186-220); rnd_seed is left to the
    caller instead of time(NULL)."""
    n = p.num_node
    p.n_ants = n
    p.nn_ants = n - 2
    p.nn_ls = n - 2
    p.max_iteration = 250
    p.iteration = 0
    p.ls_flag = True
    p.alpha, p.beta, p.rho, p.ras_ranks = 1.0, 2.0, 0.1, 6
    p.max_runtime = 600.0


def init_problem(p: Problem) -> None:
    """init_problem (problem.cpp:43-56): defaults, distances, NN lists."""
    set_default_parameters(p)
    p.distance = compute_distances(p.x, p.y, p.dis_type)
    p.nn_list = compute_nn_lists(p.distance, p.nn_ls, p.nn_ants)


def check_solution(p: Problem, tour) -> bool:
    """check_solution (problem.cpp:226-319)."""
    ci, keep = p.c_instance()
    t = np.ascontiguousarray(tour, np.int32)
    rc = lib().aco_check_solution(ctypes.byref(ci), ptr(t), len(t))
    if rc < 0:
        raise AcoError(rc, "check_solution")
    return rc == 1


def tour_length(dist: np.ndarray, tour) -> Tuple[float, float]:
    """compute_tour_length (vrpHelper.cpp:244-253) in fp32, and in fp64."""
    d = np.ascontiguousarray(dist, np.float32)
    t = np.ascontiguousarray(tour, np.int32)
    l32, l64 = ctypes.c_float(), ctypes.c_double()
    check(lib().aco_tour_length(d.shape[0], ptr(d), ptr(t), len(t), ctypes.byref(l32), ctypes.byref(l64)),
          "tour_length")
    return l32.value, l64.value


def make_seeds(seed_time: int, rnd_seed: int, n_ants: int, nloc: int) -> Tuple[np.ndarray, int]:
    """The per-work-item seeds of create_memory_objects (g_aco.cpp:714-722)."""
    out = np.zeros(n_ants * nloc, np.int32)
    rs = ctypes.c_int(rnd_seed)
    check(lib().aco_make_seeds(seed_time, ctypes.byref(rs), n_ants, nloc, ptr(out)), "make_seeds")
    return out, rs.value


def default_params(n: int) -> AcoParams:
    p = AcoParams()
    check(lib().aco_params_default(ctypes.byref(p), n), "aco_params_default")
    return p


class Solver:
    """One solver handle: device state of one instance on one GPU."""

    def __init__(self, problem: Problem, params: Optional[AcoParams] = None, tune_table=None, **overrides):
        self.problem = problem
        p = params if params is not None else default_params(problem.num_node)
        for k, v in overrides.items():
            setattr(p, k, v)
        if tune_table is not None:  # fills the launch-shape fields left at 0
            tune_table.apply(p, problem.num_node)
        self.params = p
        ci, keep = problem.c_instance()
        h = ctypes.c_void_p()
        check(lib().aco_create(ctypes.byref(ci), ctypes.byref(p), ctypes.byref(h)), "aco_create")
        self.h = h
        n = problem.num_node
        self.n, self.A, self.T = n, p.n_ants, 2 * n
        self.nloc, self.R = p.nloc, p.ras_ranks

    # lifecycle
    def init(self):
        check(lib().aco_init(self.h), "aco_init")

    def iterate(self, n_iter: int = 1):
        check(lib().aco_iterate(self.h, n_iter), "aco_iterate")

    def run(self, optimum: float = 0.0) -> int:
        done = ctypes.c_int()
        check(lib().aco_run(self.h, optimum, ctypes.byref(done)), "aco_run")
        return done.value

    def close(self):
        if self.h:
            lib().aco_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # phases
    def construct(self):
        check(lib().aco_construct_solutions(self.h), "aco_construct_solutions")

    def local_search(self):
        check(lib().aco_local_search(self.h), "aco_local_search")

    def update_statistics(self):
        check(lib().aco_update_statistics(self.h), "aco_update_statistics")

    def pheromone_update(self):
        check(lib().aco_pheromone_update(self.h), "aco_pheromone_update")

    def pheromone_init(self, trail: float):
        check(lib().aco_pheromone_init(self.h, trail), "aco_pheromone_init")

    # state
    def best(self) -> Tuple[np.ndarray, float]:
        buf = np.zeros(self.T, np.int32)
        size, length = ctypes.c_int(), ctypes.c_float()
        check(lib().aco_get_best(self.h, ptr(buf), self.T, ctypes.byref(size), ctypes.byref(length)), "aco_get_best")
        return buf[: size.value].copy(), length.value

    def solutions(self) -> Tuple[np.ndarray, np.ndarray]:
        sol = np.zeros(self.T * (self.A + 1) + 1, np.int32)
        lens = np.zeros(self.A + 1, np.float32)
        check(lib().aco_get_solutions(self.h, ptr(sol), sol.size, ptr(lens), lens.size), "aco_get_solutions")
        return sol, lens

    def tour(self, sol: np.ndarray, a: int) -> np.ndarray:
        t = sol[a * self.T:(a + 1) * self.T]
        return t[: t[self.T - 1]].copy()

    def pheromone(self) -> Tuple[np.ndarray, np.ndarray]:
        tau = np.zeros(self.n * self.n, np.float32)
        tot = np.zeros(self.n * self.n, np.float32)
        check(lib().aco_get_pheromone(self.h, ptr(tau), ptr(tot), tau.size), "aco_get_pheromone")
        return tau, tot

    def seeds(self) -> np.ndarray:
        s = np.zeros(self.A * self.nloc, np.int32)
        check(lib().aco_get_seeds(self.h, ptr(s), s.size), "aco_get_seeds")
        return s

    def elites(self) -> np.ndarray:
        e = np.zeros(self.R, np.int32)
        check(lib().aco_get_elites(self.h, ptr(e), self.R), "aco_get_elites")
        return e

    def iteration(self) -> int:
        it = ctypes.c_int()
        check(lib().aco_get_iteration(self.h, ctypes.byref(it)), "aco_get_iteration")
        return it.value

    def records(self) -> List[Tuple[int, float, float]]:
        cnt = ctypes.c_int()
        check(lib().aco_get_bsf_records(self.h, None, 0, ctypes.byref(cnt)), "aco_get_bsf_records")
        k = min(cnt.value, self.params.record_cap)
        arr = (AcoRecord * max(k, 1))()
        if k:
            check(lib().aco_get_bsf_records(self.h, ctypes.cast(arr, ctypes.c_void_p), k, ctypes.byref(cnt)),
                  "aco_get_bsf_records")
        return [(arr[i].iter, arr[i].length, arr[i].time) for i in range(k)]

    def validate(self) -> Tuple[np.ndarray, int]:
        """Device check of every tour slot (ants, then best-so-far): flags (1 =
        valid) and the number of invalid slots."""
        flags = np.zeros(self.A + 1, np.int32)
        bad = ctypes.c_int()
        check(lib().aco_validate(self.h, ptr(flags), ctypes.byref(bad)), "aco_validate")
        return flags, bad.value

    def write_solution(self, path: str) -> None:
        """The best-so-far tour in print_solution_to_file's block format."""
        check(lib().aco_write_solution(self.h, path.encode()), "aco_write_solution")

    def save_checkpoint(self, path: str) -> None:
        check(lib().aco_save_checkpoint(self.h, path.encode()), "aco_save_checkpoint")

    def load_checkpoint(self, path: str) -> None:
        """Resume from a checkpoint of a solver with the same instance and parameters."""
        check(lib().aco_load_checkpoint(self.h, path.encode()), "aco_load_checkpoint")

    def set_prior(self, prior=None):
        """heur = eta^beta * prior (n x n, finite, >= 0); None restores eta^beta."""
        if prior is None:
            check(lib().aco_set_prior(self.h, None, 0), "aco_set_prior")
            return
        pr = np.ascontiguousarray(prior, np.float32)
        if pr.shape != (self.n, self.n):
            raise ValueError(f"prior must be {self.n} x {self.n}")
        check(lib().aco_set_prior(self.h, ptr(pr), self.n), "aco_set_prior")

    def set_state(self, tau=None, total=None, solutions=None, lens=None, seeds=None):
        def c(a, dt):
            return None if a is None else np.ascontiguousarray(a, dt)
        arrs = [c(tau, np.float32), c(total, np.float32), c(solutions, np.int32), c(lens, np.float32),
                c(seeds, np.int32)]
        check(lib().aco_set_state(self.h, *[ptr(a) if a is not None else None for a in arrs]), "aco_set_state")

    def status(self) -> int:
        return lib().aco_status(self.h)

    def clear_status(self) -> int:
        """The sticky device status, then reset to ACO_OK."""
        return lib().aco_clear_status(self.h)

    def set_wait_limit(self, polls: int) -> None:
        """Polls before a device wait gives up (0 = the default)."""
        check(lib().aco_set_wait_limit(self.h, polls), "aco_set_wait_limit")

    def stream(self) -> int:
        return lib().aco_get_stream(self.h)

    def launches_per_iteration(self) -> int:
        return lib().aco_launches_per_iteration(self.h)

    def time_iterations(self, n_iter: int) -> float:
        ms = ctypes.c_float()
        check(lib().aco_time_iterations(self.h, n_iter, ctypes.byref(ms)), "aco_time_iterations")
        return ms.value

    def enqueue(self, n_iter: int = 1):
        check(lib().aco_enqueue_iterations(self.h, n_iter), "aco_enqueue_iterations")

    def enqueue_lengths(self) -> int:
        """Queue a copy of the A+1 tour lengths as they stand after the work
        queued so far; returns a ticket for read_lengths (at most 4 outstanding)."""
        t = ctypes.c_longlong()
        check(lib().aco_enqueue_lengths(self.h, ctypes.byref(t)), "aco_enqueue_lengths")
        return t.value

    def read_lengths(self, ticket: int, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Wait for the copy of `ticket` only and return the lengths."""
        if out is None:
            out = np.empty(self.A + 1, np.float32)
        check(lib().aco_read_lengths(self.h, ticket, ptr(out), out.size), "aco_read_lengths")
        return out

    def time_phases(self, n_iter: int) -> np.ndarray:
        ms = np.zeros(4, np.float32)
        check(lib().aco_time_phases(self.h, n_iter, ptr(ms)), "aco_time_phases")
        return ms

    def config(self) -> Tuple[int, int, int]:
        a, w, f = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().aco_get_config(self.h, ctypes.byref(a), ctypes.byref(w), ctypes.byref(f)), "aco_get_config")
        return a.value, w.value, f.value


class Batch:
    """Many independent instances solved by the same launches (throughput mode).

    Instance ``b`` runs exactly the iteration a single ``Solver`` with
    ``rnd_seed + b`` runs on it; the batch only shares launches, the work
    queue of the construct kernel and one device arena."""

    def __init__(self, problems: List[Problem], params: Optional[AcoParams] = None, tune_table=None, **overrides):
        self.problems = list(problems)
        if params is None:
            params = default_params(max(p.num_node for p in self.problems))
            params.mode = _lib.MODE_THROUGHPUT
        for k, v in overrides.items():
            setattr(params, k, v)
        if tune_table is not None:  # one launch shape for the batch: the entry of the median size
            sizes = sorted(p.num_node for p in self.problems)
            tune_table.apply(params, sizes[len(sizes) // 2], batch=True)
        self.params = params
        cis, self._keep = [], []
        for p in self.problems:
            ci, keep = p.c_instance()
            cis.append(ci)
            self._keep.append(keep)
        arr = (AcoInstance * len(cis))(*cis)
        h = ctypes.c_void_p()
        check(lib().aco_batch_create(arr, len(cis), ctypes.byref(params), ctypes.byref(h)), "aco_batch_create")
        self.h = h
        self.A = params.n_ants

    def __len__(self) -> int:
        return len(self.problems)

    def init(self):
        check(lib().aco_batch_init(self.h), "aco_batch_init")

    def iterate(self, n_iter: int = 1):
        check(lib().aco_batch_iterate(self.h, n_iter), "aco_batch_iterate")

    def enqueue(self, n_iter: int = 1):
        check(lib().aco_batch_enqueue_iterations(self.h, n_iter), "aco_batch_enqueue_iterations")

    def status(self) -> int:
        return lib().aco_batch_status(self.h)

    def size(self) -> Tuple[int, int]:
        c, a = ctypes.c_int(), ctypes.c_int()
        check(lib().aco_batch_size(self.h, ctypes.byref(c), ctypes.byref(a)), "aco_batch_size")
        return c.value, a.value

    def launches_per_iteration(self) -> int:
        return lib().aco_batch_launches_per_iteration(self.h)

    def stream(self) -> int:
        return lib().aco_batch_get_stream(self.h)

    def best(self, b: int) -> Tuple[np.ndarray, float]:
        T = 2 * self.problems[b].num_node
        buf = np.zeros(T, np.int32)
        size, length = ctypes.c_int(), ctypes.c_float()
        check(lib().aco_batch_get_best(self.h, b, ptr(buf), T, ctypes.byref(size), ctypes.byref(length)),
              "aco_batch_get_best")
        return buf[: size.value].copy(), length.value

    def ants_of(self, b: int) -> int:
        return self.A if self.A > 0 else self.problems[b].num_node  # n_ants = 0: one ant per node

    def lengths_total(self) -> int:
        """Floats one lengths readback holds: every instance's ants and best-so-far."""
        return sum(self.ants_of(b) + 1 for b in range(len(self.problems)))

    def enqueue_lengths(self) -> int:
        """Queue a copy of every instance's lengths as the stream stands; returns its ticket."""
        t = ctypes.c_longlong()
        check(lib().aco_batch_enqueue_lengths(self.h, ctypes.byref(t)), "aco_batch_enqueue_lengths")
        return t.value

    def read_lengths(self, ticket: int, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Wait for a queued copy: instance b's A_b + 1 lengths (ants, best-so-far)
        follow those of instances 0..b-1."""
        if out is None:
            out = np.zeros(self.lengths_total(), np.float32)
        check(lib().aco_batch_read_lengths(self.h, ticket, ptr(out), out.size), "aco_batch_read_lengths")
        return out

    def best_all(self) -> Tuple[List[np.ndarray], np.ndarray]:
        """Every instance's best-so-far tour and length in one transfer."""
        Ts = [2 * p.num_node for p in self.problems]
        tours = np.zeros(sum(Ts), np.int32)
        sizes = np.zeros(len(Ts), np.int32)
        lens = np.zeros(len(Ts), np.float32)
        check(lib().aco_batch_get_best_all(self.h, ptr(tours), tours.size, ptr(sizes), ptr(lens)),
              "aco_batch_get_best_all")
        out, off = [], 0
        for T, s in zip(Ts, sizes):
            out.append(tours[off:off + s].copy())
            off += T
        return out, lens

    def solutions(self, b: int) -> Tuple[np.ndarray, np.ndarray]:
        T = 2 * self.problems[b].num_node
        sol = np.zeros(T * (self.A + 1) + 1, np.int32)
        lens = np.zeros(self.A + 1, np.float32)
        check(lib().aco_batch_get_solutions(self.h, b, ptr(sol), sol.size, ptr(lens), lens.size),
              "aco_batch_get_solutions")
        return sol, lens

    def pheromone(self, b: int) -> Tuple[np.ndarray, np.ndarray]:
        n = self.problems[b].num_node
        tau = np.zeros(n * n, np.float32)
        tot = np.zeros(n * n, np.float32)
        check(lib().aco_batch_get_pheromone(self.h, b, ptr(tau), ptr(tot), tau.size), "aco_batch_get_pheromone")
        return tau, tot

    def time_phases(self, n_iter: int) -> np.ndarray:
        ms = np.zeros(4, np.float32)
        check(lib().aco_batch_time_phases(self.h, n_iter, ptr(ms)), "aco_batch_time_phases")
        return ms

    def config(self) -> Tuple[int, int, int]:
        """(ants per construct CTA, warps per ant, staging flags) of the batch's launches."""
        a, w, f = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().aco_batch_get_config(self.h, ctypes.byref(a), ctypes.byref(w), ctypes.byref(f)),
              "aco_batch_get_config")
        return a.value, w.value, f.value

    def validate(self) -> Tuple[np.ndarray, int]:
        """Device check of every tour of every instance: invalid slots per
        instance and in total."""
        inv = np.zeros(len(self.problems), np.int32)
        bad = ctypes.c_int()
        check(lib().aco_batch_validate(self.h, ptr(inv), ctypes.byref(bad)), "aco_batch_validate")
        return inv, bad.value

    def write_solutions(self, path: str) -> None:
        check(lib().aco_batch_write_solutions(self.h, path.encode()), "aco_batch_write_solutions")

    def save_checkpoint(self, path: str) -> None:
        check(lib().aco_batch_save_checkpoint(self.h, path.encode()), "aco_batch_save_checkpoint")

    def load_checkpoint(self, path: str) -> None:
        check(lib().aco_batch_load_checkpoint(self.h, path.encode()), "aco_batch_load_checkpoint")

    def records(self, b: int) -> List[Tuple[int, float, float]]:
        cnt = ctypes.c_int()
        check(lib().aco_batch_get_bsf_records(self.h, b, None, 0, ctypes.byref(cnt)), "aco_batch_get_bsf_records")
        k = cnt.value
        arr = (AcoRecord * max(k, 1))()
        if k:
            check(lib().aco_batch_get_bsf_records(self.h, b, ctypes.cast(arr, ctypes.c_void_p), k, ctypes.byref(cnt)),
                  "aco_batch_get_bsf_records")
        return [(arr[i].iter, arr[i].length, arr[i].time) for i in range(k)]

    def set_prior(self, b: int, prior=None):
        """Prior of instance b (see Solver.set_prior)."""
        if prior is None:
            check(lib().aco_batch_set_prior(self.h, b, None, 0), "aco_batch_set_prior")
            return
        n = self.problems[b].num_node
        pr = np.ascontiguousarray(prior, np.float32)
        if pr.shape != (n, n):
            raise ValueError(f"prior must be {n} x {n}")
        check(lib().aco_batch_set_prior(self.h, b, ptr(pr), n), "aco_batch_set_prior")

    def close(self):
        if self.h:
            lib().aco_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class GACO:
    """The reference's g_ACO (g_aco.h:16-37) over a Problem: same method names."""

    def __init__(self, instance: Problem, *, nloc: int = 256, seed_time: int = 0, mode: int = _lib.MODE_PARITY,
                 device: int = 0, **extra):
        self.instance = instance
        p = default_params(instance.num_node)
        p.n_ants = instance.n_ants or instance.num_node
        p.alpha, p.beta, p.rho, p.ras_ranks = instance.alpha, instance.beta, instance.rho, instance.ras_ranks
        p.nn_ls = instance.nn_ls
        if instance.nn_ants and mode == _lib.MODE_THROUGHPUT:
            p.nn_ants = min(instance.nn_ants, 32)
        p.ls_flag = int(bool(instance.ls_flag))
        p.mode, p.nloc, p.seed_time, p.rnd_seed, p.device = mode, nloc, seed_time, instance.rnd_seed, device
        p.max_iteration, p.max_runtime = instance.max_iteration, instance.max_runtime
        for k, v in extra.items():
            setattr(p, k, v)
        self.solver = Solver(instance, p)
        self._t0 = None

    def init_aco(self):
        self._t0 = time.perf_counter()
        self.solver.init()
        self.instance.iteration = 1
        self.update_best_so_far_from_device()

    def run_aco_iteration(self):
        self.solver.iterate(1)

    def construct_solutions(self):
        self.solver.construct()

    def local_search(self):
        self.solver.local_search()

    def update_statistics(self):
        self.solver.update_statistics()

    def pheromone_update(self):
        self.solver.pheromone_update()

    def pheromone_init(self, trail_0: float):
        self.solver.pheromone_init(trail_0)

    def update_best_so_far_from_device(self):
        tour, length = self.solver.best()
        self.instance.best_tour, self.instance.best_length = tour, length

    def exit_aco(self):
        self.update_best_so_far_from_device()
        return self.solver.records()

    def termination_condition(self) -> bool:
        """main.cpp:29-34."""
        inst = self.instance
        return (inst.iteration >= inst.max_iteration
                or (time.perf_counter() - self._t0) >= inst.max_runtime
                or abs(inst.best_length - inst.optimum) < 10 * EPSILON)

    def run(self) -> int:
        """main.cpp:83-88: init, iterate until termination, exit."""
        self.init_aco()
        while not self.termination_condition():
            self.run_aco_iteration()
            self.instance.iteration += 1
            self.update_best_so_far_from_device()
        self.exit_aco()
        return self.instance.iteration
