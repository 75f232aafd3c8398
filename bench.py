"""Benchmark: ant-tours/s of the ACO iteration (construct + 2-opt + update).

Workload (the single-instance GPU configuration): one synthetic CVRP instance
with 200 customers (201 nodes; half uniform in [0,1000]^2, half from 8 Gaussian
clusters, depot at the centre, demand U{1..100}, capacity for ~12 customers a
route), 200 ants, 25-nearest-neighbour candidate lists (throughput mode:
prefix-sum roulette), 2-opt over 25-NN lists, rank-based update with 6 ranks,
fp32 pheromone / choice_info / distances.  A step is one ACO iteration (200
ant-tours).  L2 is flushed (256 MiB write) before every timed iteration.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank runs an independent replica of the workload
(the single-instance path does not shard); `value` is the total over ranks
divided by the slowest rank's device time.  `--impl reference` times the CPU
port of the reference's path (the oracle, all host threads) on the same
workload; rank 0 alone runs it.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CUST, ANTS, NN_ANTS, NN_LS, NLOC = 200, 200, 25, 25, 256
SEED_INSTANCE, SEED_TIME, RND_SEED = 2026, 1796300000, 4242
BATCH_COUNT, BATCH_ANTS, BATCH_SEED = 512, 128, 512
KERNELS = ["construct_nn_kernel", "local_search_kernel", "stats_kernel", "rows_kernel"]
METRIC = "ant-tours/sec (construct+2-opt+update)"
UNIT = "ant-tours/s"
WORKLOAD = ("single CVRP instance, 200 customers (50% uniform, 50% 8 Gaussian clusters), 200 ants, "
            "25-NN candidate lists, 2-opt on 25-NN lists, rank-based pheromone update")


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def make_instance(rank: int = 0):
    from cvrp_aco_ocl_b200 import instances as I
    return I.gen_mixed(SEED_INSTANCE + rank, N_CUST)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summaries
    (a line 'dram_bytes_per_launch <kernel> <bytes>'), or None."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for f in sorted(os.listdir(d)):
        try:
            for line in open(os.path.join(d, f)):
                parts = line.split()
                if len(parts) == 3 and parts[0] == "dram_bytes_per_launch" and parts[1] == kernel:
                    return float(parts[2])
        except Exception:
            pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        time.sleep(0.25)
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------
def run_ours(args, ws, rank, local):
    import torch
    from cvrp_aco_ocl_b200 import MODE_THROUGHPUT, Problem, Solver, default_params

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    inst = make_instance(rank)
    prob = Problem.from_instance(inst)

    def params():
        p = default_params(inst.n)
        p.n_ants, p.nn_ants, p.nn_ls, p.nloc, p.mode = ANTS, NN_ANTS, NN_LS, NLOC, MODE_THROUGHPUT
        p.seed_time, p.rnd_seed, p.device, p.ls_flag = SEED_TIME, RND_SEED + rank, local, 1
        return p

    S = Solver(prob, params())
    S.init()
    stream = torch.cuda.ExternalStream(S.stream(), device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        with torch.cuda.stream(stream):
            flush.zero_()
        S.enqueue(1)
    S.status()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for e0, e1 in evs:
            with torch.cuda.stream(stream):
                flush.zero_()  # L2 flush between timed iterations (not timed)
                e0.record(stream)
            S.enqueue(1)
            with torch.cuda.stream(stream):
                e1.record(stream)
        torch.cuda.synchronize()
    rc = S.status()
    if rc != 0:
        raise RuntimeError(f"device status {rc}")
    ms = sum(e0.elapsed_time(e1) for e0, e1 in evs)
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = ws * ANTS * args.steps / (ms_max / 1e3)

    # per-kernel shares (device time, phase by phase, same workload and stream)
    phase_ms = S.time_phases(max(5, args.steps // 2))
    names = KERNELS
    share = phase_ms / phase_ms.sum()
    dom = int(np.argmax(phase_ms))
    n_phase = max(5, args.steps // 2)
    best_tour, best_len = S.best()
    sol, lens = S.solutions()
    draw = bool(S.config()[2] & 4)  # construct_nn_draw_kernel is the construct launched
    launches = S.launches_per_iteration()
    S.close()

    # roofline of the dominant kernel: algorithmic bytes per launch / launch time
    n = inst.n
    routes = int(np.count_nonzero(best_tour == 0)) - 1
    steps_per_tour = (n - 1) + routes
    algo = {
        "construct_nn_kernel": ANTS * steps_per_tour * NN_ANTS * 12,   # neighbour id + choice_info + distance
        "local_search_kernel": ANTS * 2 * (2 * n) * 4 * 4,              # tour read/write + edge lengths, 4 B each
        "stats_kernel": (ANTS + 1) * 4 + 6 * (2 * n) * 4,
        "rows_kernel": 16 * n * n,                                     # read tau, heur; write tau, total
    }
    peak, peak_kind = load_peaks()
    dk = names[dom]
    kname = "construct_nn_draw_kernel" if dk == "construct_nn_kernel" and draw else dk
    dur_s = phase_ms[dom] / n_phase / 1e3
    achieved = algo[dk] / dur_s / 1e9
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": profile_traffic(kname),
                "algorithmic_bytes_per_launch": algo[dk], "launch_ms": phase_ms[dom] / n_phase,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
                "fallback 6.65 TB/s", "kernel_share": {k: float(s) for k, s in zip(names, share)}}

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": WORKLOAD, "n_nodes": n, "ants": ANTS, "nn_ants": NN_ANTS, "nn_ls": NN_LS,
                   "mode": "throughput", "ras_ranks": 6, "parallelism": f"replicas x{ws}",
                   "l2": "flushed before every timed iteration (256 MiB write)", "instance_seed": SEED_INSTANCE},
        "clocks": clk.summary(), "roofline": roofline,
        "gpu_launches": args.steps * launches,  # construct, 2-opt, statistics, row pass per iteration
        "best_length": float(best_len),
    }
    if not args.no_batched:
        result["batched"] = run_batched(args, ws, rank, local, peak, peak_kind)
    # end to end through the public API with host buffers
    if rank == 0 or ws > 1:
        result["e2e"] = run_e2e(args, rank, local)
    if ws > 1:
        import torch.distributed as dist
        e = torch.tensor([result["e2e"]["value"]], device=dev, dtype=torch.float64)
        dist.all_reduce(e, op=dist.ReduceOp.MIN)
        result["e2e"]["value"] = float(e.item()) * ws
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        if ws == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(seconds=args.cpu_seconds)
        print(json.dumps(result, default=float))


def run_batched(args, ws, rank, local, peak, peak_kind):
    """Batched workload: BATCH_COUNT independent instances, customer count
    uniform in [100, 1000] (mixed and large generators alternately), 128 ants
    each, all served by the same four launches per iteration.  Instances are
    sharded over ranks by estimated cost (cvrp_aco_ocl_b200.shard; no
    collective on the data path).
    Reports ant-tours/s over the whole batch and the roofline of the fused
    pheromone pass, whose matrices (16 bytes per element over all instances)
    far exceed L2."""
    import torch
    from cvrp_aco_ocl_b200 import MODE_THROUGHPUT, Batch, Problem, default_params
    from cvrp_aco_ocl_b200 import instances as I

    from cvrp_aco_ocl_b200.shard import shard_of

    count_all = args.batch_count
    every = I.gen_batch(BATCH_SEED, count_all, 100, 1000)
    insts = [every[i] for i in shard_of([x.n for x in every], BATCH_ANTS, ws, rank)]
    probs = [Problem.from_instance(x) for x in insts]
    p = default_params(1001)
    p.mode, p.n_ants, p.nn_ants, p.nn_ls, p.nloc = MODE_THROUGHPUT, BATCH_ANTS, NN_ANTS, NN_LS, NLOC
    p.seed_time, p.rnd_seed, p.device, p.ls_flag = SEED_TIME, RND_SEED, local, 1
    t0 = time.perf_counter()
    B = Batch(probs, p)
    B.init()
    t_setup = time.perf_counter() - t0
    count, total_ants = B.size()
    for _ in range(max(3, args.batch_warmup)):
        B.enqueue(1)
    if B.status() != 0:
        raise RuntimeError("batched warm-up failed")
    dev = torch.device("cuda", local)
    stream = torch.cuda.ExternalStream(B.stream(), device=dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.batch_steps)]
    torch.cuda.synchronize()
    for e0, e1 in evs:  # inputs (about 3 GB of matrices) exceed L2: no flush needed
        with torch.cuda.stream(stream):
            e0.record(stream)
        B.enqueue(1)
        with torch.cuda.stream(stream):
            e1.record(stream)
    torch.cuda.synchronize()
    if B.status() != 0:
        raise RuntimeError("batched run failed")
    ms = sum(e0.elapsed_time(e1) for e0, e1 in evs)
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    tot = torch.tensor([float(total_ants)], device=dev, dtype=torch.float64)
    if ws > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    ms_max = float(t.item())
    phase = B.time_phases(args.batch_steps)
    launches = B.launches_per_iteration()  # the route-level 2-opt adds a kernel
    B.close()
    n_all = [pr.num_node for pr in probs]
    row_bytes = sum(16 * n * n for n in n_all)
    row_ms = float(phase[3]) / args.batch_steps
    achieved = row_bytes / (row_ms / 1e3) / 1e9
    return {
        "workload": f"{count_all} independent instances, 100-1000 customers (seeded, mixed/large generators), "
                    f"{BATCH_ANTS} ants each, {NN_ANTS}-NN lists, 2-opt on {NN_LS}-NN lists",
        "value": float(tot.item()) * args.batch_steps / (ms_max / 1e3), "unit": UNIT,
        "ms_per_step": ms_max / args.batch_steps, "steps": args.batch_steps, "instances_this_rank": count,
        "ants_this_rank": total_ants, "setup_s": t_setup,
        "gpu_launches": args.batch_steps * launches,
        "kernel_share": {k: float(v) for k, v in zip(KERNELS, phase / phase.sum())},
        "roofline": {"bound": "hbm", "kernel": "rows_kernel", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": profile_traffic("rows_kernel@batch"),
                     "algorithmic_bytes_per_launch": row_bytes, "launch_ms": row_ms,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
                     "fallback 6.65 TB/s"},
    }


def run_e2e(args, rank, local):
    """aco_create from host arrays (coordinates and demands copied host->device;
    distances, NN lists and seeds computed there), aco_init, then per
    step one iteration and a device->host read of its ant and best-so-far
    lengths (pipelined: iteration k is queued before iteration k-1's lengths
    are read), then the best tour read back: the reference's main.cpp loop
    through the C ABI, timed by the host clock."""
    import torch
    from cvrp_aco_ocl_b200 import MODE_THROUGHPUT, Problem, Solver, default_params
    from cvrp_aco_ocl_b200._lib import lib, ptr

    inst = make_instance(rank)
    prob = Problem.from_instance(inst)
    p = default_params(inst.n)
    p.n_ants, p.nn_ants, p.nn_ls, p.nloc, p.mode = ANTS, NN_ANTS, NN_LS, NLOC, MODE_THROUGHPUT
    p.seed_time, p.rnd_seed, p.device = SEED_TIME, RND_SEED + rank, local
    lens = np.zeros(ANTS + 1, np.float32)
    L = lib()
    ticket = ctypes.c_longlong()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    S = Solver(prob, p)
    S.init()
    prev = -1
    for _ in range(args.steps):
        # queue iteration k and the copy of its lengths, then read iteration k-1's:
        # the GPU runs iteration k while the host reads
        rc = L.aco_enqueue_iterations(S.h, 1) or L.aco_enqueue_lengths(S.h, ctypes.byref(ticket))
        if rc == 0 and prev >= 0:
            rc = L.aco_read_lengths(S.h, prev, ptr(lens), lens.size)
        if rc != 0:
            raise RuntimeError(rc)
        prev = ticket.value
    rc = L.aco_read_lengths(S.h, prev, ptr(lens), lens.size)
    if rc != 0:
        raise RuntimeError(rc)
    tour, length = S.best()
    t1 = time.perf_counter()
    S.close()
    n = inst.n
    # coordinates and demands, per-ant index tables and work items, argument blocks (about 1 KB); distances,
    # lists and the ants' seeds are computed on the device
    h2d = n * 4 * 3 + ANTS * 4 * 3 + 1024
    d2h = (ANTS + 1) * 4 + 4  # lengths and the status word
    return {"value": ANTS * args.steps / (t1 - t0), "unit": UNIT,
            "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h + (2 * n * 4 + 4) / args.steps,
            "note": "create+init+iterations+readbacks, host wall clock"}


# --------------------------------------------------------------------------
def oracle_run(n_threads: int, warmup: int, steps: int, max_seconds: float):
    import oracle

    inst = make_instance(0)
    dist = oracle.compute_distances(inst.x, inst.y)
    nn = oracle.compute_nn_lists(dist, NN_LS, NN_ANTS)
    seeds, _ = oracle.make_seeds(SEED_TIME, RND_SEED, ANTS, NLOC)
    O = oracle.Oracle(dist, inst.demand, inst.capacity, ANTS, NLOC, nn, seeds, ls_flag=True, nn_ants_list=nn,
                      n_threads=n_threads)
    O.init_aco(throughput=True)
    for _ in range(warmup):
        O.run_iteration(throughput=True)
    done = 0
    t0 = time.perf_counter()
    while done < steps:
        O.run_iteration(throughput=True)
        done += 1
        if time.perf_counter() - t0 > max_seconds:
            break
    dt = time.perf_counter() - t0
    return ANTS * done / dt, done, dt


def cpu_baseline(seconds: float = 15.0):
    cores = os.cpu_count() or 1
    value, done, dt = oracle_run(cores, 1, 10**9, seconds)
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{done} iterations of the same workload ({done * ANTS} ant-tours) in {dt:.1f} s, "
                      f"CPU port of the path (oracle/aco_oracle.c), {cores} threads over ants"}


def run_reference(args, ws, rank):
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    value, done, dt = oracle_run(cores, args.warmup, args.steps, max_seconds=240.0)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": ws, "steps": done,
            "warmup": args.warmup, "ms_per_step": dt * 1e3 / max(done, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": WORKLOAD, "n_nodes": N_CUST + 1, "ants": ANTS, "nn_ants": NN_ANTS,
                       "nn_ls": NN_LS, "mode": "throughput", "ras_ranks": 6},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{done} iterations ({done * ANTS} ant-tours) in {dt:.1f} s"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-workload section")
    ap.add_argument("--batch-steps", type=int, default=5)
    ap.add_argument("--batch-count", type=int, default=BATCH_COUNT,
                    help="instances of the batched section (smaller counts for profiling captures)")
    ap.add_argument("--only-batched", action="store_true",
                    help="run the batched section alone and print it as the line")
    ap.add_argument("--batch-warmup", type=int, default=3)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    ws, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    if args.only_batched:
        import torch
        torch.cuda.set_device(local)
        peak, peak_kind = load_peaks()
        line = run_batched(args, 1, 0, local, peak, peak_kind)
        print(json.dumps(line, default=float))
        return
    run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
