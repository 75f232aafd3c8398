"""CPU oracle for the CVRP ACO iteration -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline and
``--impl reference`` legs may import this package.  It wraps two shared
libraries built from ``oracle/``:

* ``liboracle.so`` -- the C restatement of the reference's kernels and host
  sequencing (``aco_oracle.c``; every function cites cvrp_ocl/gpu/kernel.cl or
  g_aco.cpp by file:line);
* ``_ref/libcvrp_ref.so`` -- the reference's own code (kernel.cl, g_aco.cpp,
  g_type.cpp and the host .cpp files) on a fake CPU OpenCL runtime, used to pin
  the restatement.  It is built only where the reference sources exist.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
import tempfile
from typing import List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libcvrp_ref.so")

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class OrcRecord(ctypes.Structure):
    _fields_ = [("iter", ctypes.c_int), ("length", ctypes.c_float), ("time", ctypes.c_float)]


class OrcState(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("n_ants", ctypes.c_int), ("nloc", ctypes.c_int),
        ("nn_ls", ctypes.c_int), ("ras_ranks", ctypes.c_int),
        ("capacity", ctypes.c_int),
        ("max_dist", ctypes.c_float), ("serv_time", ctypes.c_float),
        ("alpha", ctypes.c_float), ("beta", ctypes.c_float), ("rho", ctypes.c_float),
        ("ls_flag", ctypes.c_int), ("step_limit_passes", ctypes.c_int),
        ("dist", ctypes.c_void_p), ("demand", ctypes.c_void_p), ("nn_list", ctypes.c_void_p),
        ("tau", ctypes.c_void_p), ("total", ctypes.c_void_p),
        ("seeds", ctypes.c_void_p), ("solutions", ctypes.c_void_p), ("lens", ctypes.c_void_p),
        ("elites", ctypes.c_void_p), ("records", ctypes.c_void_p),
        ("record_cap", ctypes.c_int), ("num_bsf", ctypes.c_int),
        ("iteration", ctypes.c_int), ("update_flag", ctypes.c_int), ("status", ctypes.c_int),
        ("ns_rounds", ctypes.c_int), ("ns_seed", ctypes.c_int),
    ]


# Root of the reference's source tree (its cvrp_ocl/ and dataset/ folders), read
# only by the recipes that compile or read the reference for the checker.
REFERENCE_ROOT = os.environ.get("CVRP_REFERENCE_DIR", "/root/reference")


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and _ref/libcvrp_ref.so where the reference sources
    are present) with the committed Makefile."""
    kw = dict(cwd=HERE, check=True)
    if quiet:
        kw.update(stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    subprocess.run(["make", "liboracle.so"], **kw)
    if os.path.isdir(os.path.join(REFERENCE_ROOT, "cvrp_ocl")):
        subprocess.run(["make", "ref", f"REF={REFERENCE_ROOT}"], **kw)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_ran01.restype = ctypes.c_float
        L.orc_ran01.argtypes = [ctypes.POINTER(ctypes.c_int)]
        L.orc_make_seeds.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int, _i32p]
        L.orc_compute_distances.argtypes = [ctypes.c_int, _f32p, _f32p, ctypes.c_int, _f32p]
        L.orc_compute_nn_lists.argtypes = [ctypes.c_int, _f32p, ctypes.c_int, ctypes.c_int, _i32p]
        L.orc_compute_nn_lists.restype = ctypes.c_int
        L.orc_swap.argtypes = [ctypes.c_int, _f32p, _i32p, ctypes.c_int, ctypes.c_float, ctypes.c_float, _i32p,
                               ctypes.c_int, ctypes.c_int]
        L.orc_swap.restype = ctypes.c_int
        L.orc_srandom.argtypes = [ctypes.c_void_p, ctypes.c_uint]
        L.orc_random.argtypes = [ctypes.c_void_p]
        L.orc_random.restype = ctypes.c_int32
        L.orc_ns_propose.argtypes = [ctypes.c_int, _f32p, _i32p, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                     _i32p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_ns_apply.argtypes = [_i32p, ctypes.c_void_p]
        L.orc_ns_seed.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_ns_seed.restype = ctypes.c_uint
        L.orc_ns_descent.argtypes = [ctypes.c_int, _f32p, _i32p, ctypes.c_int, ctypes.c_float, ctypes.c_float, _i32p,
                                     ctypes.c_int, ctypes.c_uint, ctypes.c_int]
        L.orc_ns_descent.restype = ctypes.c_int
        L.orc_tour_length.argtypes = [ctypes.c_int, _f32p, _i32p, ctypes.c_int]
        L.orc_tour_length.restype = ctypes.c_float
        L.orc_tour_length_f64.argtypes = [ctypes.c_int, _f32p, _i32p, ctypes.c_int]
        L.orc_tour_length_f64.restype = ctypes.c_double
        L.orc_check_solution.argtypes = [ctypes.c_int, _f32p, _i32p, ctypes.c_int, ctypes.c_float,
                                         ctypes.c_float, _i32p, ctypes.c_int]
        L.orc_tournament_priority.argtypes = [ctypes.c_int, _i32p]
        L.orc_pow_rule.argtypes = [ctypes.c_float, ctypes.c_float]
        L.orc_pow_rule.restype = ctypes.c_float
        L.orc_f2i_x86.argtypes = [ctypes.c_float]
        L.orc_race_exp1.argtypes = [ctypes.c_float]
        L.orc_race_exp1.restype = ctypes.c_float
        sp = ctypes.POINTER(OrcState)
        for name in ("orc_construct", "orc_local_search", "orc_init_aco", "orc_run_aco_iteration"):
            getattr(L, name).argtypes = [sp, ctypes.c_int]
        for name in ("orc_construct_nn", "orc_init_aco_nn", "orc_run_aco_iteration_nn"):
            getattr(L, name).argtypes = [sp, _i32p, ctypes.c_int, ctypes.c_int]
        for name in ("orc_find_best", "orc_get_elites", "orc_pheromone_evaporation",
                     "orc_pheromone_deposit", "orc_compute_total_info"):
            getattr(L, name).argtypes = [sp]
        L.orc_update_best_so_far.argtypes = [sp, ctypes.c_float]
        L.orc_pheromone_init.argtypes = [sp, ctypes.c_float]
        _lib = L
    return _lib


# ---- small functions ------------------------------------------------------
def ran01(seed: int):
    s = ctypes.c_int(seed)
    r = lib().orc_ran01(ctypes.byref(s))
    return r, s.value


def race_exp1(u: float) -> float:
    """-ln(u) as the throughput sampler computes it (fp32, own polynomial)."""
    return float(lib().orc_race_exp1(ctypes.c_float(u)))


def make_seeds(seed_time: int, rnd_seed: int, n_ants: int, nloc: int):
    out = np.zeros(n_ants * nloc, dtype=np.int32)
    rs = ctypes.c_int(rnd_seed)
    lib().orc_make_seeds(seed_time, ctypes.byref(rs), n_ants, nloc, out)
    return out, rs.value


def compute_distances(x, y, dist_type: int = 0):
    n = len(x)
    d = np.zeros(n * n, dtype=np.float32)
    lib().orc_compute_distances(n, np.ascontiguousarray(x, np.float32), np.ascontiguousarray(y, np.float32),
                                dist_type, d)
    return d.reshape(n, n)


def compute_nn_lists(dist: np.ndarray, nn_ls: int, nn_ants: int):
    n = dist.shape[0]
    depth = max(nn_ls, nn_ants)
    if depth >= n:
        depth = n - 1
    out = np.zeros(n * max(depth, 1), dtype=np.int32)
    got = lib().orc_compute_nn_lists(n, np.ascontiguousarray(dist, np.float32).ravel(), nn_ls, nn_ants, out)
    return out[: n * got].reshape(n, got)


def tournament_priority(n: int):
    p = np.zeros(n, dtype=np.int32)
    lib().orc_tournament_priority(n, p)
    return p


def tour_length(dist, tour):
    t = np.ascontiguousarray(tour, np.int32)
    return lib().orc_tour_length(dist.shape[0], np.ascontiguousarray(dist, np.float32).ravel(), t, len(t))


def tour_length_f64(dist, tour):
    t = np.ascontiguousarray(tour, np.int32)
    return lib().orc_tour_length_f64(dist.shape[0], np.ascontiguousarray(dist, np.float32).ravel(), t, len(t))


def check_solution(dist, demand, capacity, tour, max_dist=math.inf, serv_time=0.0) -> bool:
    t = np.ascontiguousarray(tour, np.int32)
    return bool(lib().orc_check_solution(dist.shape[0], np.ascontiguousarray(dist, np.float32).ravel(),
                                         np.ascontiguousarray(demand, np.int32), int(capacity),
                                         float(max_dist), float(serv_time), t, len(t)))


# ---- full state ------------------------------------------------------------
class Oracle:
    """The reference's device state and phases on the CPU (one instance)."""

    def __init__(self, dist: np.ndarray, demand, capacity: int, n_ants: int, nloc: int,
                 nn_list: np.ndarray, seeds: np.ndarray, *, ras_ranks: int = 6,
                 alpha: float = 1.0, beta: float = 2.0, rho: float = 0.1,
                 max_dist: float = math.inf, serv_time: float = 0.0, ls_flag: bool = False,
                 ls_pass_limit: int = 0, record_cap: int = 4096, nn_ants_list: Optional[np.ndarray] = None,
                 n_threads: int = 1, ns_rounds: int = 0, ns_seed: int = 0):
        n = dist.shape[0]
        self.n, self.A, self.T = n, n_ants, 2 * n
        self.n_threads = n_threads
        self.dist = np.ascontiguousarray(dist, np.float32).ravel().copy()
        self.demand = np.ascontiguousarray(demand, np.int32).copy()
        self.nn_list = np.ascontiguousarray(nn_list, np.int32).ravel().copy()
        self.nn_ls = nn_list.shape[1] if nn_list.ndim == 2 else 0
        self.nn_ants_list = None if nn_ants_list is None else np.ascontiguousarray(nn_ants_list, np.int32).copy()
        self.tau = np.zeros(n * n, np.float32)
        self.total = np.zeros(n * n, np.float32)
        self.seeds = np.ascontiguousarray(seeds, np.int32).copy()
        assert self.seeds.size == n_ants * nloc
        self.solutions = np.zeros(self.T * (n_ants + 1) + 1, np.int32)
        self.lens = np.zeros(n_ants + 1, np.float32)
        self.elites = np.zeros(ras_ranks, np.int32)
        self.records = (OrcRecord * record_cap)()
        st = OrcState()
        st.n, st.n_ants, st.nloc, st.nn_ls, st.ras_ranks = n, n_ants, nloc, self.nn_ls, ras_ranks
        st.capacity = int(capacity)
        st.max_dist, st.serv_time = float(max_dist), float(serv_time)
        st.alpha, st.beta, st.rho = alpha, beta, rho
        st.ls_flag = int(ls_flag)  # 1: 2-opt; 3: 2-opt then the swap stage
        st.step_limit_passes = int(ls_pass_limit)
        st.ns_rounds, st.ns_seed = int(ns_rounds), int(ns_seed)
        for name in ("dist", "demand", "nn_list", "tau", "total", "seeds", "solutions", "lens", "elites"):
            setattr(st, name, getattr(self, name).ctypes.data)
        st.records = ctypes.cast(self.records, ctypes.c_void_p)
        st.record_cap = record_cap
        self.st = st
        self._p = ctypes.byref(st)

    # phases
    def construct(self):
        return lib().orc_construct(self._p, self.n_threads)

    def construct_nn(self):
        K = self.nn_ants_list.shape[1]
        return lib().orc_construct_nn(self._p, self.nn_ants_list.ravel(), K, self.n_threads)

    def local_search(self):
        return lib().orc_local_search(self._p, self.n_threads)

    def find_best(self):
        lib().orc_find_best(self._p)

    def update_best_so_far(self, time: float = 0.0):
        lib().orc_update_best_so_far(self._p, time)

    def get_elites(self):
        lib().orc_get_elites(self._p)

    def pheromone_init(self, trail: float):
        lib().orc_pheromone_init(self._p, trail)

    def evaporation(self):
        lib().orc_pheromone_evaporation(self._p)

    def deposit(self):
        lib().orc_pheromone_deposit(self._p)

    def compute_total_info(self):
        lib().orc_compute_total_info(self._p)

    def init_aco(self, throughput: bool = False):
        if throughput:
            K = self.nn_ants_list.shape[1]
            return lib().orc_init_aco_nn(self._p, self.nn_ants_list.ravel(), K, self.n_threads)
        return lib().orc_init_aco(self._p, self.n_threads)

    def run_iteration(self, throughput: bool = False):
        if throughput:
            K = self.nn_ants_list.shape[1]
            return lib().orc_run_aco_iteration_nn(self._p, self.nn_ants_list.ravel(), K, self.n_threads)
        return lib().orc_run_aco_iteration(self._p, self.n_threads)

    # views
    def tour(self, a: int):
        t = self.solutions[a * self.T:(a + 1) * self.T]
        return t[: t[self.T - 1]].copy()

    @property
    def iteration(self):
        return self.st.iteration

    @property
    def num_bsf(self):
        return self.st.num_bsf

    @property
    def update_flag(self):
        return self.st.update_flag

    def record_list(self):
        k = min(self.st.num_bsf, self.st.record_cap)
        return [(self.records[i].iter, self.records[i].length) for i in range(k)]

    @property
    def iter_best(self):
        return int(self.solutions[self.T * (self.A + 1)])


# ---- the reference on the fake OpenCL runtime -------------------------------
_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_LIB_PATH)


def ref_lib():
    global _ref
    if _ref is None:
        L = ctypes.CDLL(REF_LIB_PATH)
        L.ref_open.argtypes = [ctypes.c_char_p, ctypes.c_char_p] + [ctypes.c_int] * 6
        L.ref_read.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_long]
        L.ref_read.restype = ctypes.c_long
        L.ref_problem_info.argtypes = [_i32p]
        L.ref_host_check_solution.argtypes = [_i32p, ctypes.c_int]
        L.ref_swap.argtypes = [ctypes.c_char_p, _i32p, ctypes.c_int]
        L.ref_ns.argtypes = [ctypes.c_char_p, _i32p, ctypes.c_int, ctypes.c_uint, ctypes.c_int, ctypes.c_int,
                             _i32p, _i32p, _f32p, _i32p, _i32p]
        L.ref_read_instance.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                        _f32p, _f32p, _i32p, _f32p, _i32p, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float),
                                        ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
        _ref = L
    return _ref


class RefSession:
    """One try of the reference (main.cpp:68-92) on the fake OpenCL runtime."""

    BUF = dict(seeds=0, solutions=1, lens=2, pheromone=3, total_info=4, elites=5, records=6,
               num_bsf=7, distance=8, nn_list=9, update_flag=10)

    def __init__(self, vrp_path: str, n_ants: int, nloc: int, seed_time: int, rnd_seed0: int,
                 nn_ls: int = 0, ls_flag: bool = False):
        self._tmp = tempfile.TemporaryDirectory()
        os.makedirs(os.path.join(self._tmp.name, "gpu"))
        open(os.path.join(self._tmp.name, "gpu", "kernel.cl"), "w").close()
        L = ref_lib()
        rc = L.ref_open(vrp_path.encode(), self._tmp.name.encode(), n_ants, nloc, seed_time, rnd_seed0,
                        nn_ls, int(bool(ls_flag)))
        if rc != 0:
            raise RuntimeError(f"ref_open failed: {rc}")
        info = np.zeros(4, np.int32)
        L.ref_problem_info(info)
        self.n, self.A, self.nn_ls, self.capacity = (int(v) for v in info)
        self.T = 2 * self.n

    def init_aco(self):
        ref_lib().ref_init_aco()

    def run_iteration(self):
        ref_lib().ref_run_iteration()

    def read(self, name: str, dtype=np.int32):
        L = ref_lib()
        size = L.ref_read(self.BUF[name], None, 0)
        item = np.dtype(dtype).itemsize
        out = np.zeros(max(size // item, 1), dtype=dtype)
        L.ref_read(self.BUF[name], out.ctypes.data, size)
        return out[: size // item]

    def close(self):
        ref_lib().ref_close()
        self._tmp.cleanup()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def ref_read_instance(vrp_path: str, cap_nodes: int = 2048):
    """The reference's read_instance_file + compute_distances + compute_nn_lists."""
    L = ref_lib()
    n = ctypes.c_int()
    cap = ctypes.c_int()
    depth = ctypes.c_int()
    opt, md, st = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    x = np.zeros(cap_nodes, np.float32)
    y = np.zeros(cap_nodes, np.float32)
    dem = np.zeros(cap_nodes, np.int32)
    dist = np.zeros(cap_nodes * cap_nodes, np.float32)
    nn = np.zeros(cap_nodes * cap_nodes, np.int32)
    L.ref_read_instance(vrp_path.encode(), ctypes.byref(n), ctypes.byref(cap), x, y, dem, dist, nn, cap_nodes,
                        ctypes.byref(depth), ctypes.byref(opt), ctypes.byref(md), ctypes.byref(st))
    N, D = n.value, depth.value
    return dict(n=N, capacity=cap.value, x=x[:N].copy(), y=y[:N].copy(), demand=dem[:N].copy(),
                dist=dist[: N * N].reshape(N, N).copy(), nn=nn[: N * D].reshape(N, D).copy(),
                optimum=opt.value, max_distance=md.value, service_time=st.value)


def swap(dist, demand, capacity: int, tour, max_dist: float = math.inf, serv_time: float = 0.0,
         max_swaps: int = 0):
    """LocalSearch::swap restated (orc_swap) on a copy of `tour`: (tour, swaps)."""
    d = np.ascontiguousarray(dist, np.float32)
    t = np.ascontiguousarray(tour, np.int32).copy()
    k = lib().orc_swap(d.shape[0], d.ravel(), np.ascontiguousarray(demand, np.int32), int(capacity), float(max_dist),
                       float(serv_time), t, len(t), int(max_swaps))
    return t, k


def ref_swap(vrp_path: str, tour) -> np.ndarray:
    """The reference's own LocalSearch::swap on a copy of `tour` (instance read from vrp_path)."""
    t = np.ascontiguousarray(tour, np.int32).copy()
    if ref_lib().ref_swap(vrp_path.encode(), t, len(t)) != 0:
        raise RuntimeError("ref_swap failed")
    return t


class OrcRng(ctypes.Structure):
    _fields_ = [("r", ctypes.c_uint32 * 31), ("f", ctypes.c_int), ("b", ctypes.c_int)]


class OrcMove(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("valid", ctypes.c_int), ("gain", ctypes.c_float), ("pos1", ctypes.c_int),
                ("pos2", ctypes.c_int)]


def random_stream(seed: int, count: int) -> List[int]:
    """glibc random() after srandom(seed), restated (orc_random)."""
    g = OrcRng()
    lib().orc_srandom(ctypes.byref(g), seed)
    return [lib().orc_random(ctypes.byref(g)) for _ in range(count)]


def ns_proposals(dist, demand, capacity, tour, seed: int, count: int, apply: bool, max_dist=math.inf, serv=0.0):
    """The restated NeighbourSearch proposals (and applications) on a copy of
    `tour`: list of (type, valid, gain, pos1, pos2) and the final tour."""
    d = np.ascontiguousarray(dist, np.float32)
    dem = np.ascontiguousarray(demand, np.int32)
    t = np.ascontiguousarray(tour, np.int32).copy()
    g = OrcRng()
    lib().orc_srandom(ctypes.byref(g), seed)
    out = []
    for _ in range(count):
        m = OrcMove()
        lib().orc_ns_propose(d.shape[0], d.ravel(), dem, int(capacity), float(max_dist), float(serv), t, len(t),
                             ctypes.byref(g), ctypes.byref(m))
        out.append((m.type, m.valid, np.float32(m.gain), m.pos1, m.pos2))
        if apply and m.type >= 0 and m.valid and np.float32(m.gain) < np.float32(-0.001):
            lib().orc_ns_apply(t, ctypes.byref(m))
    return out, t


def ref_ns_proposals(vrp_path: str, tour, seed: int, count: int, apply: bool):
    """The reference's own NeighbourSearch proposals on a copy of `tour`."""
    t = np.ascontiguousarray(tour, np.int32).copy()
    ty, va, p1, p2 = (np.zeros(count, np.int32) for _ in range(4))
    ga = np.zeros(count, np.float32)
    ref_lib().ref_ns(vrp_path.encode(), t, len(t), seed, count, int(apply), ty, va, ga, p1, p2)
    return [(int(a), int(b), np.float32(c), int(d), int(e)) for a, b, c, d, e in zip(ty, va, ga, p1, p2)], t


def ns_descent(dist, demand, capacity, tour, seed: int, rounds: int, max_dist=math.inf, serv=0.0):
    d = np.ascontiguousarray(dist, np.float32)
    t = np.ascontiguousarray(tour, np.int32).copy()
    k = lib().orc_ns_descent(d.shape[0], d.ravel(), np.ascontiguousarray(demand, np.int32), int(capacity),
                             float(max_dist), float(serv), t, len(t), seed, rounds)
    return t, k
