"""ctypes binding of the C ABI in include/cvrp_aco.h (libcvrp_aco.so, built in-tree).

There is no fallback: if the library is missing or cannot be loaded, every
entry point raises.  The library itself returns ACO_ERR_NO_DEVICE when no
sm_100 GPU is present.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libcvrp_aco.so")

ACO_OK = 0
ERRORS = {
    -1: "ACO_ERR_INVALID", -2: "ACO_ERR_INFEASIBLE", -3: "ACO_ERR_CUDA", -4: "ACO_ERR_NO_DEVICE",
    -5: "ACO_ERR_NOMEM", -6: "ACO_ERR_STATE", -7: "ACO_ERR_STEP_LIMIT", -8: "ACO_ERR_LS_LIMIT",
    -9: "ACO_ERR_RECORD_OVERFLOW", -10: "ACO_ERR_CAPACITY", -11: "ACO_ERR_IO", -12: "ACO_ERR_TIMEOUT",
}
MODE_PARITY, MODE_THROUGHPUT = 0, 1

# every symbol include/cvrp_aco.h declares
EXPORTED = [
    "aco_params_default", "aco_read_vrplib", "aco_compute_distances", "aco_compute_nn_lists",
    "aco_check_solution", "aco_tour_length", "aco_make_seeds", "aco_create", "aco_init", "aco_iterate",
    "aco_run", "aco_destroy", "aco_construct_solutions", "aco_local_search", "aco_update_statistics",
    "aco_pheromone_update", "aco_pheromone_init", "aco_get_best", "aco_get_bsf_records",
    "aco_get_solutions", "aco_get_pheromone", "aco_get_seeds", "aco_get_elites", "aco_get_iteration",
    "aco_set_state", "aco_status", "aco_strerror", "aco_get_stream", "aco_launches_per_iteration",
    "aco_time_iterations", "aco_enqueue_iterations", "aco_enqueue_lengths", "aco_read_lengths", "aco_time_phases", "aco_get_config",
    "aco_batch_get_config",
    "aco_pheromone_update_noalloc", "aco_batch_create", "aco_batch_init", "aco_batch_iterate",
    "aco_batch_enqueue_iterations", "aco_batch_status", "aco_batch_size", "aco_batch_get_best",
    "aco_batch_get_solutions", "aco_batch_get_pheromone", "aco_batch_time_phases", "aco_batch_get_stream",
    "aco_batch_destroy", "aco_batch_launches_per_iteration", "aco_autotune", "aco_batch_autotune", "aco_mpnn_param_count", "aco_mpnn_workspace_bytes",
    "aco_mpnn_forward", "aco_mpnn_grad", "aco_mpnn_adam", "aco_mpnn_status", "aco_set_prior", "aco_batch_set_prior",
    "aco_last_cuda_error", "aco_compute_distances_device", "aco_compute_nn_lists_device", "aco_validate",
    "aco_write_solution", "aco_batch_validate", "aco_batch_write_solutions", "aco_batch_get_bsf_records",
    "aco_save_checkpoint", "aco_load_checkpoint", "aco_batch_save_checkpoint", "aco_batch_load_checkpoint",
    "aco_batch_enqueue_lengths", "aco_batch_read_lengths", "aco_batch_get_best_all", "aco_clear_status",
    "aco_set_wait_limit",
]


class AcoError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        self.code = code
        super().__init__(f"{where}: {ERRORS.get(code, code)} ({code})")


class AcoInstance(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("demand", ctypes.c_void_p),
        ("capacity", ctypes.c_int), ("max_distance", ctypes.c_float), ("service_time", ctypes.c_float),
        ("dist_type", ctypes.c_int), ("dist", ctypes.c_void_p),
    ]


class AcoParams(ctypes.Structure):
    _fields_ = [
        ("n_ants", ctypes.c_int), ("alpha", ctypes.c_float), ("beta", ctypes.c_float), ("rho", ctypes.c_float),
        ("ras_ranks", ctypes.c_int), ("nn_ants", ctypes.c_int), ("nn_ls", ctypes.c_int), ("ls_flag", ctypes.c_int),
        ("mode", ctypes.c_int), ("nloc", ctypes.c_int), ("seed_time", ctypes.c_int), ("rnd_seed", ctypes.c_int),
        ("max_iteration", ctypes.c_int), ("max_runtime", ctypes.c_float), ("ls_pass_limit", ctypes.c_int),
        ("record_cap", ctypes.c_int), ("device", ctypes.c_int), ("use_graph", ctypes.c_int),
        ("ants_per_block", ctypes.c_int), ("warps_per_ant", ctypes.c_int), ("ls_warps", ctypes.c_int),
        ("stage_matrix", ctypes.c_int), ("host_prep", ctypes.c_int), ("fuse_ls", ctypes.c_int),
        ("ns_rounds", ctypes.c_int),
        ("ls_ants", ctypes.c_int),
        ("draw_warps", ctypes.c_int),
        ("route_ls", ctypes.c_int), ("wait_limit", ctypes.c_int), ("ls_best", ctypes.c_int),
        ("construct_ctas", ctypes.c_int),
    ]


class AcoRecord(ctypes.Structure):
    _fields_ = [("iter", ctypes.c_int), ("length", ctypes.c_float), ("time", ctypes.c_float)]


_lib = None


def lib() -> ctypes.CDLL:
    """Load libcvrp_aco.so (raises if it is missing: there is no CPU path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m cvrp_aco_ocl_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, fp = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.aco_params_default.argtypes = [ctypes.POINTER(AcoParams), ip]
        L.aco_read_vrplib.argtypes = [ctypes.c_char_p, ctypes.POINTER(ip), vp, vp, vp, ctypes.POINTER(ip),
                                      ctypes.POINTER(fp), ctypes.POINTER(fp), ctypes.POINTER(ip),
                                      ctypes.POINTER(fp), ctypes.c_char_p, ip]
        L.aco_compute_distances.argtypes = [ip, vp, vp, ip, vp]
        L.aco_compute_nn_lists.argtypes = [ip, vp, ip, ip, vp, ctypes.POINTER(ip)]
        L.aco_check_solution.argtypes = [ctypes.POINTER(AcoInstance), vp, ip]
        L.aco_tour_length.argtypes = [ip, vp, vp, ip, ctypes.POINTER(fp), ctypes.POINTER(ctypes.c_double)]
        L.aco_make_seeds.argtypes = [ip, ctypes.POINTER(ip), ip, ip, vp]
        L.aco_create.argtypes = [ctypes.POINTER(AcoInstance), ctypes.POINTER(AcoParams), ctypes.POINTER(vp)]
        for name in ("aco_init", "aco_construct_solutions", "aco_local_search", "aco_update_statistics",
                     "aco_pheromone_update", "aco_status", "aco_launches_per_iteration"):
            getattr(L, name).argtypes = [vp]
        L.aco_iterate.argtypes = [vp, ip]
        L.aco_run.argtypes = [vp, fp, ctypes.POINTER(ip)]
        L.aco_destroy.argtypes = [vp]
        L.aco_destroy.restype = None
        L.aco_pheromone_init.argtypes = [vp, fp]
        L.aco_get_best.argtypes = [vp, vp, ip, ctypes.POINTER(ip), ctypes.POINTER(fp)]
        L.aco_get_bsf_records.argtypes = [vp, vp, ip, ctypes.POINTER(ip)]
        L.aco_get_solutions.argtypes = [vp, vp, ctypes.c_size_t, vp, ctypes.c_size_t]
        L.aco_get_pheromone.argtypes = [vp, vp, vp, ctypes.c_size_t]
        L.aco_get_seeds.argtypes = [vp, vp, ctypes.c_size_t]
        L.aco_get_elites.argtypes = [vp, vp, ip]
        L.aco_get_iteration.argtypes = [vp, ctypes.POINTER(ip)]
        L.aco_set_state.argtypes = [vp, vp, vp, vp, vp, vp]
        L.aco_strerror.argtypes = [ip]
        L.aco_strerror.restype = ctypes.c_char_p
        L.aco_get_stream.argtypes = [vp]
        L.aco_get_stream.restype = vp
        L.aco_time_iterations.argtypes = [vp, ip, ctypes.POINTER(fp)]
        L.aco_enqueue_iterations.argtypes = [vp, ip]
        L.aco_batch_launches_per_iteration.argtypes = [vp]
        L.aco_enqueue_lengths.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        L.aco_read_lengths.argtypes = [vp, ctypes.c_longlong, vp, ctypes.c_size_t]
        L.aco_time_phases.argtypes = [vp, ip, vp]
        L.aco_pheromone_update_noalloc.argtypes = [ip, ip, ip, ip, fp, fp, fp, vp, vp, vp, vp, vp, vp, vp]
        L.aco_batch_create.argtypes = [ctypes.POINTER(AcoInstance), ip, ctypes.POINTER(AcoParams), ctypes.POINTER(vp)]
        for name in ("aco_batch_init", "aco_batch_status"):
            getattr(L, name).argtypes = [vp]
        L.aco_batch_iterate.argtypes = [vp, ip]
        L.aco_batch_enqueue_iterations.argtypes = [vp, ip]
        L.aco_batch_size.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip)]
        L.aco_batch_get_best.argtypes = [vp, ip, vp, ip, ctypes.POINTER(ip), ctypes.POINTER(fp)]
        L.aco_batch_get_solutions.argtypes = [vp, ip, vp, ctypes.c_size_t, vp, ctypes.c_size_t]
        L.aco_batch_get_pheromone.argtypes = [vp, ip, vp, vp, ctypes.c_size_t]
        L.aco_batch_time_phases.argtypes = [vp, ip, vp]
        L.aco_batch_get_stream.argtypes = [vp]
        L.aco_batch_get_stream.restype = vp
        L.aco_batch_destroy.argtypes = [vp]
        L.aco_batch_destroy.restype = None
        L.aco_autotune.argtypes = [ctypes.POINTER(AcoInstance), ctypes.POINTER(AcoParams), ip,
                                   ctypes.POINTER(AcoParams), ctypes.POINTER(fp)]
        L.aco_batch_autotune.argtypes = [ctypes.POINTER(AcoInstance), ip, ctypes.POINTER(AcoParams), ip,
                                         ctypes.POINTER(AcoParams), ctypes.POINTER(fp)]
        sz = ctypes.c_size_t
        L.aco_mpnn_param_count.argtypes = [ip]
        L.aco_mpnn_workspace_bytes.argtypes = [ip, ip, ip, ctypes.POINTER(sz)]
        L.aco_mpnn_forward.argtypes = [ip, ip, ip, vp, vp, vp, vp, vp, sz, vp, vp]
        L.aco_mpnn_grad.argtypes = [ip, ip, ip, vp, vp, vp, vp, vp, fp, vp, sz, vp, vp, vp, vp]
        L.aco_mpnn_adam.argtypes = [ip, vp, vp, vp, vp, fp, fp, fp, fp, ip, vp]
        L.aco_mpnn_status.argtypes = [vp, vp]
        L.aco_set_prior.argtypes = [vp, vp, ip]
        L.aco_batch_set_prior.argtypes = [vp, ip, vp, ip]
        L.aco_last_cuda_error.argtypes = []
        L.aco_last_cuda_error.restype = ctypes.c_char_p
        L.aco_compute_distances_device.argtypes = [ip, vp, vp, ip, vp, ip, vp]
        L.aco_compute_nn_lists_device.argtypes = [ip, vp, ip, ip, ip, vp, ctypes.POINTER(ip), vp]
        L.aco_validate.argtypes = [vp, vp, ctypes.POINTER(ip)]
        L.aco_write_solution.argtypes = [vp, ctypes.c_char_p]
        L.aco_batch_validate.argtypes = [vp, vp, ctypes.POINTER(ip)]
        L.aco_batch_write_solutions.argtypes = [vp, ctypes.c_char_p]
        L.aco_batch_get_bsf_records.argtypes = [vp, ip, vp, ip, ctypes.POINTER(ip)]
        for name in ("aco_save_checkpoint", "aco_load_checkpoint", "aco_batch_save_checkpoint",
                     "aco_batch_load_checkpoint"):
            getattr(L, name).argtypes = [vp, ctypes.c_char_p]
        L.aco_get_config.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ip)]
        L.aco_batch_get_config.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ip)]
        L.aco_batch_enqueue_lengths.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        L.aco_batch_read_lengths.argtypes = [vp, ctypes.c_longlong, vp, ctypes.c_size_t]
        L.aco_batch_get_best_all.argtypes = [vp, vp, ctypes.c_size_t, vp, vp]
        L.aco_clear_status.argtypes = [vp]
        L.aco_set_wait_limit.argtypes = [vp, ip]
        _lib = L
    return _lib


def check(rc: int, where: str = "") -> None:
    if rc != ACO_OK:
        if rc == -3:  # ACO_ERR_CUDA
            where = f"{where} [{lib().aco_last_cuda_error().decode()}]"
        raise AcoError(rc, where)


def ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None
