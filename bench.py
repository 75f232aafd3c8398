"""Benchmark: ant-tours/s of the ACO iteration (construct + 2-opt + update).

Headline workload (the batched configuration, the largest that fits one GPU):
512 independent synthetic CVRP instances per GPU, customer count uniform in
[100, 1000], drawn alternately from the mixed generator (half uniform in
[0,1000]^2, half from 8 Gaussian clusters, sigma 40, depot at the centre,
demand U{1..100}, ~12 customers a route) and the large generator (uniform or
clustered, depot random/centre/corner, uniform or 80/20 small/large demand,
~15 customers a route); 128 ants each, 25-nearest-neighbour candidate lists,
2-opt on 25-NN lists, rank-based update with 6 ranks, fp32 state.  All
instances advance together: one iteration is one replay of a CUDA graph of five
kernel launches for the whole batch.  A step is one iteration (65,536
ant-tours).  The matrices (3.4 GB) exceed L2, so no flush is needed between
timed iterations.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Extra keys of the line: `single` (200 customers, 200 ants), `large` (1000
customers, 256 ants, 30-NN lists), `parity` (the reference's own algorithm:
50 customers, 50 ants, full-row I-Roulette, 2-opt on full lists, 800
iterations, bit-compared with the CPU restatement of the reference's kernels)
and `learned_vs_plain` (time for the learned-prior colony to come within 1% of
the plain colony's FP64-checked best on held-out 1000-customer instances).

Under torchrun (N > 1) the global batch is 512 x N instances, partitioned over
the ranks by estimated cost (cvrp_aco_ocl_b200.shard; no collective on the data
path): weak scaling, `value` = all ranks' ant-tours / the slowest rank's device
time.  `--impl reference` times the CPU port of the reference's path (the
oracle, all host threads) on a stratified sample of the same batch at the same
iteration offsets; rank 0 alone runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ant-tours/sec (construct+2-opt+update)"
UNIT = "ant-tours/s"
SEED_TIME, RND_SEED, NLOC = 1796300000, 4242, 256
# headline: the batch
BATCH_COUNT, BATCH_ANTS, BATCH_SEED, NN_ANTS, NN_LS, RANKS = 512, 128, 512, 25, 25, 6
CPU_SAMPLE_STRIDE = 16  # the CPU legs run every 16th instance of the size-sorted batch (32 of 512)
# extra sections
SINGLE_CUST, SINGLE_ANTS, SINGLE_SEED = 200, 200, 2026
LARGE_CUST, LARGE_ANTS, LARGE_K, LARGE_SEED = 1000, 256, 30, 3031
# 800 iterations: on this configuration the reference's algorithm stops working at iteration 866.  With
# rho = 0.1 and no lower bound on tau, tau * eta^beta of the unused edges underflows to 0 in fp32.  Every
# choice value is then 0, and kernel.cl:461 sends the ant back to the depot forever.  The reference hangs
# there; this build reports ACO_ERR_STEP_LIMIT.
PARITY_CUST, PARITY_ANTS, PARITY_ITERS, PARITY_SEED = 50, 50, 800, 2024
LEARNED_N, LEARNED_COUNT, LEARNED_PLAIN_ITERS, LEARNED_ANTS = 1001, 8, 500, 256
PHASES = ["construct", "two_opt", "stats", "rows"]
PHASE_KERNELS = {"construct": "construct_nn_kernel", "two_opt": "route_opt_kernel+local_search_kernel",
                 "stats": "stats_kernel", "rows": "rows_kernel"}


def construct_kernel(flags: int) -> str:
    """The throughput construct kernel a colony launches, from aco_batch_get_config's flags."""
    return "construct_nn_wide_kernel" if flags & 8 else "construct_nn_draw_kernel" if flags & 4 else "construct_nn_kernel"


def dist_env():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def batch_workload(ws: int, rank: int):
    """This rank's shard of the global batch (512 x ws instances) and their
    indices in it."""
    from cvrp_aco_ocl_b200 import instances as I
    from cvrp_aco_ocl_b200.shard import shard_of

    every = I.gen_batch(BATCH_SEED, BATCH_COUNT * ws, 100, 1000)
    idx = shard_of([x.n for x in every], BATCH_ANTS, ws, rank)
    return [every[i] for i in idx], idx


def batch_params(local: int):
    from cvrp_aco_ocl_b200 import MODE_THROUGHPUT, default_params
    p = default_params(1001)
    p.mode, p.n_ants, p.nn_ants, p.nn_ls, p.nloc, p.ras_ranks = MODE_THROUGHPUT, BATCH_ANTS, NN_ANTS, NN_LS, NLOC, RANKS
    p.seed_time, p.rnd_seed, p.device, p.ls_flag = SEED_TIME, RND_SEED, local, 1
    return p


def tune_table():
    """The committed launch-shape table of this GPU (cvrp_aco_ocl_b200/tune_b200.json); its 0
    fields leave the choice to the library's create-time model."""
    from cvrp_aco_ocl_b200.tune import DEFAULT_TABLE, TuneTable
    return TuneTable.load(DEFAULT_TABLE) if os.path.exists(DEFAULT_TABLE) else None


def config(ws: int):
    return {"workload": f"{BATCH_COUNT} independent CVRP instances per GPU, 100-1000 customers each (mixed and large "
                        f"generators alternately), {BATCH_ANTS} ants each, {NN_ANTS}-NN candidate lists, 2-opt on "
                        f"{NN_LS}-NN lists, rank-based pheromone update ({RANKS} ranks), one batched iteration per step",
            "instances": BATCH_COUNT * ws, "ants": BATCH_ANTS, "nn_ants": NN_ANTS, "nn_ls": NN_LS,
            "mode": "throughput", "ras_ranks": RANKS, "batch_seed": BATCH_SEED,
            "parallelism": f"instances sharded by cost over {ws} GPU(s)",
            "l2": "inputs exceed L2 (about 3.4 GB of matrices per GPU): no flush",
            "launch_shapes": "tune table (cvrp_aco_ocl_b200/tune_b200.json)"}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


def profile_figure(key: str, name: str):
    """A machine-readable figure `<key> <name> <value>` from the committed ncu
    summaries under profiles/, or None."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for f in sorted(os.listdir(d)):
        try:
            for line in open(os.path.join(d, f)):
                parts = line.split()
                if len(parts) == 3 and parts[0] == key and parts[1] == name:
                    return float(parts[2])
        except (OSError, ValueError):
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
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        time.sleep(0.25)
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
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


def timed_launches(enqueue, stream, steps, dev):
    """Device time of `steps` calls of enqueue(), each bracketed by CUDA events
    recorded on the solver's own stream (milliseconds, summed)."""
    import torch
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for e0, e1 in evs:
        e0.record(stream)
        enqueue()
        e1.record(stream)
    torch.cuda.synchronize(dev)
    return sum(e0.elapsed_time(e1) for e0, e1 in evs)


# --------------------------------------------------------------------------
def kernel_rooflines(phase_ms, steps, row_bytes, clk, peak_hbm, peak_src, workload_tag, kernels=None):
    """Per phase: launch time, share and the bound that limits it.  The pheromone
    pass is HBM-bound (16 bytes per matrix element); the construct and the 2-opt
    are issue-bound (many independent warp-serial chains, no bandwidth near a
    limit): achieved = warp instructions per launch (ncu, committed under
    profiles/) / the live launch time, against 148 SMs x 4 schedulers x the SM
    clock sampled during the timed region."""
    out = {}
    kernels = dict(PHASE_KERNELS, **(kernels or {}))
    total = float(sum(phase_ms))
    mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0
    issue_peak = 148 * 4 * mhz * 1e6 / 1e9  # G warp-instructions/s
    for k, name in enumerate(PHASES):
        launch_ms = float(phase_ms[k]) / steps
        e = {"kernel": kernels[name], "launch_ms": launch_ms, "share": float(phase_ms[k]) / total}
        if name == "rows":
            ach = row_bytes / (launch_ms / 1e3) / 1e9
            e.update({"bound": "hbm", "achieved": ach, "peak": peak_hbm, "unit": "GB/s", "frac": ach / peak_hbm,
                      "algorithmic_bytes_per_launch": row_bytes, "peak_source": peak_src,
                      "traffic": profile_figure("dram_bytes_per_launch", f"rows_kernel@{workload_tag}")})
        elif name in ("construct", "two_opt"):
            ks = kernels[name].split("+")
            insts = [profile_figure("warp_inst_per_launch", f"{k2}@{workload_tag}") for k2 in ks]
            inst = sum(insts) if all(v is not None for v in insts) else None
            ach = inst / (launch_ms / 1e3) / 1e9 if inst is not None else None
            e.update({"bound": "issue", "achieved": ach, "peak": issue_peak, "unit": "G warp-instructions/s",
                      "frac": ach / issue_peak if ach is not None else None,
                      "warp_instructions_per_launch": inst,
                      "peak_source": f"148 SMs x 4 issue slots x {mhz:.0f} MHz (sampled)",
                      # fractions of the same kernel on the 64-instance cut of the batch (multi-pass capture)
                      "smem_frac_ncu": profile_figure("smem_pipe_frac", f"{ks[0]}@batch64"),
                      "issue_active_ncu": profile_figure("issue_active_frac", f"{ks[0]}@batch64"),
                      "traffic": sum(v for v in (profile_figure("dram_bytes_per_launch", f"{k2}@{workload_tag}")
                                                 for k2 in ks) if v is not None) or None})
        else:
            e.update({"bound": "latency"})
        out[name] = e
    return out


def run_ours(args, ws, rank, local):
    import torch
    from cvrp_aco_ocl_b200 import Batch, Problem

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    insts, _ = batch_workload(ws, rank)
    probs = [Problem.from_instance(x) for x in insts]
    B = Batch(probs, batch_params(local), tune_table=tune_table())
    B.init()
    count, total_ants = B.size()
    stream = torch.cuda.ExternalStream(B.stream(), device=dev)
    for _ in range(args.warmup):
        B.enqueue(1)
    if B.status() != 0:
        raise RuntimeError("batched warm-up failed")
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        ms = timed_launches(lambda: B.enqueue(1), stream, args.steps, dev)
    rc = B.status()
    if rc != 0:
        raise RuntimeError(f"device status {rc}")
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    tot = torch.tensor([float(total_ants)], device=dev, dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    ms_max = float(t.item())
    value = float(tot.item()) * args.steps / (ms_max / 1e3)
    launches = B.launches_per_iteration()
    # per-phase device time, same batch and stream, phase by phase with events between
    n_phase = max(3, args.steps // 2)
    phase_ms = B.time_phases(n_phase)
    ckern = construct_kernel(B.config()[2])
    B.close()
    row_bytes = sum(16 * p.num_node * p.num_node for p in probs)
    peak, peak_src = load_peaks()
    clocks = clk.summary()
    kern = kernel_rooflines(phase_ms, n_phase, row_bytes, clocks, peak, peak_src, "batch512",
                            {"construct": ckern})
    dom = max(kern, key=lambda k: kern[k]["share"])
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded generators, no dataset)", "config": config(ws),
        "clocks": clocks, "roofline": dict(kern[dom], phase=dom), "kernels": kern,
        "roofline_hbm": dict(kern["rows"], phase="rows"),
        "gpu_launches": args.steps * launches, "launches_per_iteration": launches,
        "instances_this_rank": count, "ants_this_rank": total_ants,
    }
    # end to end through the public API, host buffers in, results out
    e2e = run_e2e(args, ws, rank, local)
    if dist is not None:
        e = torch.tensor([e2e["seconds"]], device=dev, dtype=torch.float64)
        dist.all_reduce(e, op=dist.ReduceOp.MAX)
        e2e["value"] = float(tot.item()) * args.steps / float(e.item())
        dist.barrier()
        dist.destroy_process_group()
    result["e2e"] = e2e
    if rank != 0:
        return
    if not args.no_extras:
        result["single"] = run_single(args, local)
        result["large"] = run_large(args, local)
        result["parity"] = run_parity(args, local)
        if not args.no_learned:
            result["learned_vs_plain"] = run_learned(args)
    if ws == 1 and not args.no_cpu_baseline:
        v, done, dt, sample = oracle_batch_run(os.cpu_count() or 1, args.warmup, args.steps, args.cpu_seconds)
        result["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                                  "sample": sample}
    print(json.dumps(result, default=float))


def run_e2e(args, ws, rank, local):
    """aco_batch_create from host arrays (coordinates and demands copied
    host->device; distances, NN lists and seeds computed there), aco_batch_init,
    then per step one iteration and a device->host read of every instance's ant
    and best-so-far lengths (pipelined: iteration k is queued before iteration
    k-1's lengths are read), then every best tour read back in one transfer:
    the reference's main.cpp loop through the C ABI, for the whole batch, timed
    by the host clock."""
    import torch
    from cvrp_aco_ocl_b200 import Batch, Problem

    insts, _ = batch_workload(ws, rank)
    probs = [Problem.from_instance(x) for x in insts]
    table = tune_table()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    B = Batch(probs, batch_params(local), tune_table=table)
    B.init()
    buf = np.zeros(B.lengths_total(), np.float32)
    prev = -1
    for _ in range(args.steps):
        # queue iteration k and the copy of its lengths, then read iteration k-1's
        B.enqueue(1)
        tk = B.enqueue_lengths()
        if prev >= 0:
            B.read_lengths(prev, buf)
        prev = tk
    B.read_lengths(prev, buf)
    tours, best = B.best_all()
    t1 = time.perf_counter()
    count, total_ants = B.size()
    B.close()
    h2d = sum(p.num_node * 4 * 3 for p in probs) + count * 1024  # coordinates, demands; tables and argument blocks
    d2h_step = buf.size * 4 + 4  # lengths and the status word
    d2h_end = sum(2 * p.num_node * 4 + 8 for p in probs)
    return {"value": total_ants * args.steps / (t1 - t0), "unit": UNIT, "seconds": t1 - t0,
            "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h_step + d2h_end / args.steps,
            "best_length_mean": float(np.mean(best)),
            "note": "batch create + init + iterations with per-step length readback + best tours, host wall clock"}


def single_params(n, ants, k, local, seed):
    from cvrp_aco_ocl_b200 import MODE_THROUGHPUT, default_params
    p = default_params(n)
    p.n_ants, p.nn_ants, p.nn_ls, p.nloc, p.mode = ants, k, k, NLOC, MODE_THROUGHPUT
    p.seed_time, p.rnd_seed, p.device, p.ls_flag = SEED_TIME, seed, local, 1
    return p


def run_one_instance(args, local, inst, ants, k, label):
    """Device time of one instance's iterations (L2 flushed before each)."""
    import torch
    from cvrp_aco_ocl_b200 import Problem, Solver

    dev = torch.device("cuda", local)
    S = Solver(Problem.from_instance(inst), single_params(inst.n, ants, k, local, RND_SEED), tune_table=tune_table())
    S.init()
    stream = torch.cuda.ExternalStream(S.stream(), device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        S.enqueue(1)
    S.status()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize(dev)
    for e0, e1 in evs:
        with torch.cuda.stream(stream):
            flush.zero_()  # L2 flush between timed iterations (not timed)
        e0.record(stream)
        S.enqueue(1)
        e1.record(stream)
    torch.cuda.synchronize(dev)
    if S.status() != 0:
        raise RuntimeError(f"{label}: device status")
    ms = sum(e0.elapsed_time(e1) for e0, e1 in evs)
    phase = S.time_phases(max(3, args.steps // 2))
    _, best = S.best()
    S.close()
    return {"value": ants * args.steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / args.steps,
            "n_nodes": inst.n, "ants": ants, "nn_ants": k, "nn_ls": k, "best_length": float(best),
            "phase_share": {nm: float(v) for nm, v in zip(PHASES, phase / phase.sum())},
            "l2": "flushed before every timed iteration (256 MiB write)"}


def run_single(args, local):
    from cvrp_aco_ocl_b200 import instances as I
    r = run_one_instance(args, local, I.gen_mixed(SINGLE_SEED, SINGLE_CUST), SINGLE_ANTS, NN_ANTS, "single")
    r["workload"] = (f"one instance, {SINGLE_CUST} customers (50% uniform, 50% 8 Gaussian clusters), "
                     f"{SINGLE_ANTS} ants, {NN_ANTS}-NN lists, 2-opt on {NN_ANTS}-NN lists")
    return r


def run_large(args, local):
    from cvrp_aco_ocl_b200 import instances as I
    r = run_one_instance(args, local, I.gen_large(LARGE_SEED, LARGE_CUST), LARGE_ANTS, LARGE_K, "large")
    r["workload"] = (f"one instance, {LARGE_CUST} customers (large generator), {LARGE_ANTS} ants, "
                     f"{LARGE_K}-NN lists, 2-opt on {LARGE_K}-NN lists")
    return r


def run_parity(args, local):
    """The reference's algorithm bit for bit: 50 customers (integer coordinates
    in [0,100]^2, demand U{1..30}, capacity 160), 50 ants, alpha 1, beta 2,
    rho 0.1, full-row I-Roulette with the reference's RNG stream (nloc 256),
    2-opt on full neighbour lists, 800 iterations after init_aco (the
    reference's algorithm itself breaks down at iteration 866 here, see
    PARITY_ITERS).  Device time
    of the iterations, end-to-end time through the C ABI (create, init,
    iterations with per-iteration length readback, best tour), and the CPU
    restatement of the reference's kernels (the oracle) timed on the host's
    cores; the final state of both is compared bit for bit."""
    import torch

    import oracle
    from cvrp_aco_ocl_b200 import MODE_PARITY, Problem, Solver, default_params
    from cvrp_aco_ocl_b200 import instances as I

    inst = I.gen_uniform_small(PARITY_SEED, PARITY_CUST)
    n, A = inst.n, PARITY_ANTS
    prob = Problem.from_instance(inst)

    def params():
        p = default_params(n)
        p.n_ants, p.nloc, p.seed_time, p.rnd_seed, p.mode, p.device = A, NLOC, SEED_TIME, RND_SEED, MODE_PARITY, local
        p.nn_ls, p.ls_flag = n - 2, 1
        return p

    S = Solver(prob, params())
    S.init()
    dev_ms = S.time_iterations(PARITY_ITERS)
    sol, lens = S.solutions()
    tau, tot = S.pheromone()
    seeds = S.seeds()
    _, best = S.best()
    S.close()
    # end to end
    lens_buf = np.zeros(A + 1, np.float32)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    S = Solver(prob, params())
    S.init()
    prev = -1
    for _ in range(PARITY_ITERS):
        S.enqueue(1)
        tk = S.enqueue_lengths()
        if prev >= 0:
            S.read_lengths(prev, lens_buf)
        prev = tk
    S.read_lengths(prev, lens_buf)
    S.best()
    e2e_s = time.perf_counter() - t0
    S.close()
    # the oracle: same seeds, same iterations
    cores = os.cpu_count() or 1
    dist = oracle.compute_distances(inst.x, inst.y)
    nn = oracle.compute_nn_lists(dist, n - 2, n - 2)
    sd, _ = oracle.make_seeds(SEED_TIME, RND_SEED, A, NLOC)
    O = oracle.Oracle(dist, inst.demand, inst.capacity, A, NLOC, nn, sd, ls_flag=True, n_threads=cores)
    O.init_aco()
    c0 = time.perf_counter()
    for _ in range(PARITY_ITERS):
        O.run_iteration()
    cpu_s = time.perf_counter() - c0
    same = {"solutions": bool(np.array_equal(sol, O.solutions)), "lengths": bool(np.array_equal(lens, O.lens)),
            "pheromone": bool(np.array_equal(tau, O.tau)), "total_info": bool(np.array_equal(tot, O.total)),
            "seeds": bool(np.array_equal(seeds, O.seeds))}
    if not all(same.values()):
        print(f"bench: parity run differs from the oracle after {PARITY_ITERS} iterations: {same}", file=sys.stderr)
    return {"workload": f"one instance, {PARITY_CUST} customers (integer coordinates in [0,100]^2, demand U{{1..30}}, "
                        f"capacity 160), {A} ants, full-row I-Roulette with the reference's RNG stream (nloc {NLOC}), "
                        f"2-opt on full lists, {PARITY_ITERS} iterations",
            "value": A * PARITY_ITERS / (dev_ms / 1e3), "unit": UNIT, "ms_per_step": dev_ms / PARITY_ITERS,
            "e2e": {"value": A * PARITY_ITERS / e2e_s, "unit": UNIT, "seconds": e2e_s},
            "cpu_reference_port": {"value": A * PARITY_ITERS / cpu_s, "unit": UNIT, "cores": cores,
                                   "seconds": cpu_s, "kind": "port (oracle/aco_oracle.c, kernel.cl restated)"},
            "bit_exact_after_run": all(same.values()), "compared": same, "best_length": float(best)}


def run_learned(args):
    from cvrp_aco_ocl_b200 import learned_eval as LE
    from cvrp_aco_ocl_b200 import prior as PR

    scorer = PR.EdgeScorer.load(PR.DEFAULT_WEIGHTS)
    t0 = time.perf_counter()
    res = LE.time_to_equal_cost(scorer, LEARNED_N, args.learned_count, LEARNED_PLAIN_ITERS, LEARNED_ANTS, NN_ANTS)
    res["seconds"] = time.perf_counter() - t0
    res["workload"] = (f"{args.learned_count} held-out instances of {LEARNED_N - 1} customers (mixed and large "
                       f"generators), {LEARNED_ANTS} ants, {NN_ANTS}-NN candidate lists in both arms, plain = "
                       f"{LEARNED_PLAIN_ITERS} iterations; learned wall time includes graph build, network forward "
                       f"and prior upload")
    res["gate"] = "median ratio <= 0.5"
    return res


# --------------------------------------------------------------------------
def oracle_batch_run(n_threads: int, warmup: int, steps: int, max_seconds: float):
    """The CPU port of the path (oracle/aco_oracle.c) on a stratified sample of
    rank 0's batch: every 16th instance by size (32 of 512, 100-1000 customers),
    with the same parameters and per-instance seeds as on the GPU; after
    init_aco, `warmup` iterations, then `steps` timed iterations (the GPU arm's
    offsets), each iteration over every sampled instance.  Threads split each
    instance's ants."""
    import oracle

    insts, _ = batch_workload(1, 0)
    order = sorted(range(len(insts)), key=lambda i: (insts[i].n, i))
    picked = order[::CPU_SAMPLE_STRIDE]
    colonies = []
    for b in picked:
        inst = insts[b]
        d = oracle.compute_distances(inst.x, inst.y)
        k = min(NN_ANTS, inst.n - 2)
        nn = oracle.compute_nn_lists(d, min(NN_LS, inst.n - 2), k)
        seeds, _ = oracle.make_seeds(SEED_TIME, RND_SEED + b, BATCH_ANTS, NLOC)
        O = oracle.Oracle(d, inst.demand, inst.capacity, BATCH_ANTS, NLOC, nn, seeds, ls_flag=True,
                          nn_ants_list=nn, n_threads=n_threads)
        O.init_aco(throughput=True)
        colonies.append(O)
    for _ in range(warmup):
        for O in colonies:
            O.run_iteration(throughput=True)
    done = 0
    t0 = time.perf_counter()
    while done < steps:
        for O in colonies:
            O.run_iteration(throughput=True)
        done += 1
        if time.perf_counter() - t0 > max_seconds:
            break
    dt = time.perf_counter() - t0
    ants = BATCH_ANTS * len(colonies)
    sample = (f"{len(colonies)} of the batch's {len(insts)} instances (every {CPU_SAMPLE_STRIDE}th by size, "
              f"{insts[picked[0]].n}-{insts[picked[-1]].n} nodes), iterations {warmup + 1}-{warmup + done} after "
              f"init ({done * ants} ant-tours) in {dt:.1f} s, {n_threads} threads over each instance's ants")
    return ants * done / dt, done, dt, sample


def run_reference(args, ws, rank):
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    value, done, dt, sample = oracle_batch_run(cores, args.warmup, args.steps, max_seconds=240.0)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": ws, "steps": done,
            "warmup": args.warmup, "ms_per_step": dt * 1e3 / max(done, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators, no dataset)",
            "config": config(ws),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    global BATCH_COUNT
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=120.0, help="bound on the timed CPU iterations")
    ap.add_argument("--no-extras", action="store_true", help="only the headline batch (profiling captures)")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-vs-plain section")
    ap.add_argument("--learned-count", type=int, default=LEARNED_COUNT)
    ap.add_argument("--batch-count", type=int, default=BATCH_COUNT,
                    help="instances per GPU of the headline batch (smaller counts for profiling captures)")
    ap.add_argument("--only", choices=["single", "large", "parity", "learned"],
                    help="run this extra section alone and print it as the line (profiling captures)")
    args = ap.parse_args()
    BATCH_COUNT = args.batch_count
    if args.impl == "ours":
        args.warmup = max(args.warmup, 3)
    ws, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    if args.only:
        import torch
        torch.cuda.set_device(local)
        fn = {"single": run_single, "large": run_large, "parity": run_parity}.get(args.only)
        line = fn(args, local) if fn else run_learned(args)
        print(json.dumps(line, default=float))
        return
    run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
