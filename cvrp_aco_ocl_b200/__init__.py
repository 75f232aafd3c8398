"""cvrp_aco_ocl_b200 -- the CVRP ant-colony iteration (construct, 2-opt,
rank-based pheromone update) as hand-written sm_100a CUDA kernels behind a C
ABI (include/cvrp_aco.h), with a Python mirror of the reference's driver
surface (Problem, read_instance_file, init_problem, g_ACO)."""
from ._lib import MODE_PARITY, MODE_THROUGHPUT, AcoError, AcoParams
from .aco import (GACO, Batch, Problem, Solver, check_solution, compute_distances, compute_nn_lists, default_params,
                  init_problem, make_seeds, read_instance_file, tour_length)
from .instances import Instance, gen_batch, gen_large, gen_mixed, gen_uniform_small, write_vrplib

__all__ = [
    "MODE_PARITY", "MODE_THROUGHPUT", "AcoError", "AcoParams", "GACO", "Batch", "Problem", "Solver", "check_solution",
    "compute_distances", "compute_nn_lists", "default_params", "init_problem", "make_seeds", "read_instance_file",
    "tour_length", "Instance", "gen_batch", "gen_large", "gen_mixed", "gen_uniform_small", "write_vrplib",
]
