"""Generate golden vectors from the reference's own code.

Runs the reference (cvrp_ocl/gpu/kernel.cl + g_aco.cpp + host .cpp files,
compiled for the CPU against oracle/refshim's fake OpenCL runtime by
oracle/build_ref.sh) on small seeded synthetic instances and stores every
device buffer after init_aco and after each iteration in an .npz per case.
It reads the reference sources under $CVRP_REFERENCE_DIR (default
/root/reference); the fixtures it writes are committed, so the tests read them
wherever the reference is absent.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from cvrp_aco_ocl_b200 import instances as I  # noqa: E402

# (name, generator, seed, customers, n_ants, nloc, seed_time, rnd_seed, ls_flag, nn_ls, iterations)
CASES = [
    ("c1_ls", "small", 11, 50, 50, 256, 1796300000, 4242, True, 0, 3),
    ("c1_nols", "small", 12, 50, 50, 256, 1796300000, 99, False, 0, 3),
    ("n21_nloc32", "small", 13, 20, 12, 32, 1700000000, 7, True, 0, 4),
    ("n70_nloc64_nn10", "mixed", 14, 69, 40, 64, 1234567, 555, True, 10, 3),
    ("n130_a33", "mixed", 15, 129, 33, 128, 1796300123, 31337, True, 25, 2),
]


def run_case(name, gen, seed, nc, A, nloc, T0, rs0, ls, nn_ls, iters, out_dir):
    inst = I.gen_uniform_small(seed, nc) if gen == "small" else I.gen_mixed(seed, nc)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, name + ".vrp")
        I.write_vrplib(inst, path)
        info = oracle.ref_read_instance(path)
        with oracle.RefSession(path, A, nloc, T0, rs0, nn_ls=nn_ls, ls_flag=ls) as R:
            n = R.n
            snap = dict(
                x=inst.x, y=inst.y, demand=inst.demand, capacity=np.int32(inst.capacity),
                meta=np.array([n, A, nloc, T0, rs0, int(ls), R.nn_ls, iters], np.int64),
                dist=info["dist"], nn=info["nn"],
            )
            R.init_aco()
            for it in range(iters + 1):
                tag = "init" if it == 0 else f"it{it}"
                snap[f"{tag}_seeds"] = R.read("seeds")
                snap[f"{tag}_solutions"] = R.read("solutions")
                snap[f"{tag}_lens"] = R.read("lens", np.float32)
                snap[f"{tag}_tau"] = R.read("pheromone", np.float32)
                snap[f"{tag}_total"] = R.read("total_info", np.float32)
                snap[f"{tag}_elites"] = R.read("elites")
                snap[f"{tag}_num_bsf"] = R.read("num_bsf")
                rec = R.read("records", np.float32).reshape(-1, 3)
                k = int(snap[f"{tag}_num_bsf"][0])
                snap[f"{tag}_rec_iter"] = rec[:k, 0].view(np.int32).copy()
                snap[f"{tag}_rec_len"] = rec[:k, 1].copy()
                if it < iters:
                    R.run_iteration()
    np.savez_compressed(os.path.join(out_dir, name + ".npz"), **snap)


def main():
    if not oracle.ref_available():
        oracle.build(quiet=False)
    for case in CASES:
        run_case(*case, out_dir=HERE)
        print("wrote", case[0])


if __name__ == "__main__":
    main()
