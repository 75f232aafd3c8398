"""Autotuner front end: launch configurations per instance size, kept in a table.

``aco_autotune`` / ``aco_batch_autotune`` (C ABI) time the launch shapes on
the device -- ants per construct CTA, matrix staging (throughput) or warps per
ant (parity), ants and warps per 2-opt CTA -- and return the fastest.  Every shape
computes the same result bit for bit, so the choice is a pure speed question.
This module runs them over a ladder of sizes, stores the winners as a JSON
table keyed by mode, node-count range and ant count, and fills the ``0 =
autotuned`` fields of ``aco_params`` from it.

The candidate-list length (``nn_ants``) changes the search, not only its
speed; ``tune_candidate_length`` picks it by solution quality at equal wall
time instead.

    python -m cvrp_aco_ocl_b200.tune --sizes 101,201,501,1001 --ants 128 --out tune.json
"""
from __future__ import annotations

import argparse
import ctypes
import dataclasses
import json
import time
from typing import Dict, List, Optional, Sequence, Tuple

from . import _lib
from ._lib import AcoInstance, AcoParams, check, lib

SHAPE_FIELDS = ("ants_per_block", "warps_per_ant", "ls_warps", "stage_matrix", "ls_ants", "draw_warps", "route_ls",
                "construct_ctas")


@dataclasses.dataclass
class TuneEntry:
    mode: int
    n_lo: int
    n_hi: int
    ants: int
    ants_per_block: int
    warps_per_ant: int
    ls_warps: int
    stage_matrix: int
    ms_per_iter: float
    nn_ants: int = 0  # list length the entry was timed with (0 = not recorded)
    ls_ants: int = 0  # ants per 2-opt CTA (0 = the library's default)
    draw_warps: int = 0  # helper draw warps (0 = the library's default)
    route_ls: int = 0    # route-level 2-opt (0 = the library's default)
    batch: int = 0       # 1: tuned on a batch of instances in [n_lo, n_hi] (for Batch), 0: on one instance
    construct_ctas: int = 0  # construct CTAs per SM (0 = the library's default)


class TuneTable:
    """Tuned launch shapes by (mode, node-count range, ants)."""

    def __init__(self, entries: Optional[List[TuneEntry]] = None, device: str = ""):
        self.entries: List[TuneEntry] = list(entries or [])
        self.device = device

    def save(self, path: str) -> None:
        with open(path, "w") as f:
            json.dump({"version": 1, "device": self.device,
                       "entries": [dataclasses.asdict(e) for e in self.entries]}, f, indent=1)

    @classmethod
    def load(cls, path: str) -> "TuneTable":
        with open(path) as f:
            d = json.load(f)
        if d.get("version") != 1:
            raise ValueError(f"{path}: unknown tune table version {d.get('version')}")
        return cls([TuneEntry(**e) for e in d["entries"]], d.get("device", ""))

    def add(self, e: TuneEntry) -> None:
        self.entries = [x for x in self.entries
                        if not (x.mode == e.mode and x.n_lo == e.n_lo and x.n_hi == e.n_hi and x.ants == e.ants)]
        self.entries.append(e)
        self.entries.sort(key=lambda x: (x.mode, x.n_lo, x.ants))

    def lookup(self, n: int, mode: int, ants: int, batch: bool = False) -> Optional[TuneEntry]:
        """The entry of this mode and kind (batch or single instance) whose node
        range holds n, with the nearest ant count (ratio distance); None when no
        range holds n."""
        hits = [e for e in self.entries
                if e.mode == mode and bool(e.batch) == batch and e.n_lo <= n <= e.n_hi]
        if not hits:
            return None
        return min(hits, key=lambda e: abs((e.ants / max(ants, 1)) - 1.0))

    def apply(self, params: AcoParams, n: int, batch: bool = False) -> AcoParams:
        """Fill the launch-shape fields the caller left at 0 (autotuned) from the
        entry for n (a batch: its median size); fields set by the caller are kept."""
        e = self.lookup(n, params.mode, params.n_ants if params.n_ants > 0 else n, batch)
        if e is None:
            return params
        for f in SHAPE_FIELDS:
            if getattr(params, f) == 0:
                setattr(params, f, getattr(e, f))
        return params


def autotune(problem, params: AcoParams, iters: int = 3) -> Tuple[AcoParams, float]:
    """Fastest launch shape for one instance (aco_autotune)."""
    ci, _keep = problem.c_instance()
    out = AcoParams()
    ms = ctypes.c_float()
    check(lib().aco_autotune(ctypes.byref(ci), ctypes.byref(params), iters, ctypes.byref(out), ctypes.byref(ms)),
          "aco_autotune")
    return out, ms.value


def autotune_batch(problems, params: AcoParams, iters: int = 2) -> Tuple[AcoParams, float]:
    """Fastest launch shape for a batch (aco_batch_autotune)."""
    cis, keep = [], []
    for p in problems:
        ci, k = p.c_instance()
        cis.append(ci)
        keep.append(k)
    arr = (AcoInstance * len(cis))(*cis)
    out = AcoParams()
    ms = ctypes.c_float()
    check(lib().aco_batch_autotune(arr, len(cis), ctypes.byref(params), iters, ctypes.byref(out),
                                   ctypes.byref(ms)), "aco_batch_autotune")
    return out, ms.value


def size_ranges(sizes: Sequence[int]) -> List[Tuple[int, int]]:
    """Node-count ranges around a ladder of tuned sizes: each size covers up to
    the geometric midpoint with its neighbours; the ends are open."""
    s = sorted(set(int(v) for v in sizes))
    out = []
    for k, n in enumerate(s):
        lo = 3 if k == 0 else int((s[k - 1] * n) ** 0.5) + 1
        hi = 1 << 30 if k == len(s) - 1 else int((n * s[k + 1]) ** 0.5)
        out.append((lo, hi))
    return out


def build_table(sizes: Sequence[int], ants: int, mode: int = _lib.MODE_THROUGHPUT, iters: int = 3,
                seed: int = 1, nn_ants: int = 25, table: Optional[TuneTable] = None, log=None) -> TuneTable:
    """Tune two synthetic instances per size (the mixed and the large
    generator) and record, over the size ranges of `size_ranges`, the fields
    both choose alike; a field they choose differently stays 0 (the library's
    create-time model), since the shape depends on the instance there."""
    from .aco import Problem, default_params
    from .instances import gen_large, gen_mixed

    table = table or TuneTable()
    for (lo, hi), n in zip(size_ranges(sizes), sorted(set(int(v) for v in sizes))):
        t0 = time.perf_counter()
        outs, mss = [], []
        for gen in (gen_mixed, gen_large):
            prob = Problem.from_instance(gen(seed + n, n - 1))
            p = default_params(n)
            p.mode, p.n_ants = mode, ants
            p.nn_ants = min(nn_ants, n - 2)
            p.nn_ls = min(p.nn_ls, 25)
            p.seed_time, p.rnd_seed = 1796300000, seed
            out, ms = autotune(prob, p, iters)
            outs.append(out)
            mss.append(ms)
        agree = {f: (getattr(outs[0], f) if getattr(outs[0], f) == getattr(outs[1], f) else 0) for f in SHAPE_FIELDS}
        ms = sum(mss) / len(mss)
        e = TuneEntry(mode, lo, hi, ants, agree["ants_per_block"], agree["warps_per_ant"], agree["ls_warps"],
                      agree["stage_matrix"], ms, min(nn_ants, n - 2), agree["ls_ants"], agree["draw_warps"],
                      agree["route_ls"], construct_ctas=agree["construct_ctas"])
        table.add(e)
        if log:
            log(f"n={n} [{lo},{hi}] ants={ants}: apc={e.ants_per_block} wpa={e.warps_per_ant} "
                f"ls_warps={e.ls_warps} ls_ants={e.ls_ants} stage={e.stage_matrix} ctas={e.construct_ctas} {ms:.3f} ms/iter ({time.perf_counter() - t0:.1f} s)")
    return table


def build_batch_entry(seed: int, count: int, n_min: int, n_max: int, ants: int, nn_ants: int = 25, iters: int = 3,
                      table: Optional[TuneTable] = None, log=None) -> TuneTable:
    """Tune the launch shape of a batch (gen_batch(seed, count, n_min, n_max),
    the batched workload's generator) and record it as the batch entry for
    customer counts in [n_min, n_max]."""
    from .aco import Problem, default_params
    from .instances import gen_batch

    table = table or TuneTable()
    probs = [Problem.from_instance(x) for x in gen_batch(seed, count, n_min, n_max)]
    p = default_params(n_max + 1)
    p.mode, p.n_ants, p.nn_ants, p.nn_ls = _lib.MODE_THROUGHPUT, ants, nn_ants, min(25, n_min - 1)
    p.seed_time, p.rnd_seed = 1796300000, seed
    t0 = time.perf_counter()
    out, ms = autotune_batch(probs, p, iters)
    e = TuneEntry(_lib.MODE_THROUGHPUT, n_min + 1, n_max + 1, ants, out.ants_per_block, out.warps_per_ant,
                  out.ls_warps, out.stage_matrix, ms, nn_ants, out.ls_ants, out.draw_warps, out.route_ls, batch=1,
                  construct_ctas=out.construct_ctas)
    table.entries = [x for x in table.entries if not (x.batch and x.n_lo == e.n_lo and x.n_hi == e.n_hi
                                                      and x.ants == e.ants)]
    table.entries.append(e)
    table.entries.sort(key=lambda x: (x.mode, x.batch, x.n_lo, x.ants))
    if log:
        log(f"batch of {count} [{e.n_lo},{e.n_hi}] ants={ants}: apc={e.ants_per_block} stage={e.stage_matrix} "
            f"draw={e.draw_warps} route_ls={e.route_ls} ctas={e.construct_ctas} {ms:.3f} ms/iter ({time.perf_counter() - t0:.1f} s)")
    return table


def tune_candidate_length(problem, params: AcoParams, ks: Sequence[int] = (16, 20, 25, 32),
                          seconds: float = 2.0) -> Tuple[int, Dict[int, float]]:
    """Candidate-list length by solution quality at equal wall time: plain
    throughput-mode ACO runs `seconds` with each K from the same seeds; the K
    with the lowest best-so-far length wins (ties: the smaller K)."""
    from .aco import Solver

    costs: Dict[int, float] = {}
    for k in ks:
        k = min(int(k), problem.num_node - 2)
        if k in costs or k < 1:
            continue
        p = AcoParams.from_buffer_copy(params)
        p.mode, p.nn_ants = _lib.MODE_THROUGHPUT, k
        with Solver(problem, p) as S:
            S.init()
            t0 = time.perf_counter()
            while time.perf_counter() - t0 < seconds:
                S.iterate(5)
            costs[k] = S.best()[1]
    best = min(costs, key=lambda k: (costs[k], k))
    return best, costs


DEFAULT_TABLE = __import__("os").path.join(__import__("os").path.dirname(__file__), "tune_b200.json")


def compare(table: TuneTable, iters: int = 20) -> Dict[str, Dict[str, float]]:
    """Device ms per iteration of three workloads with the table's shapes and
    with the library's create-time model (every shape field 0): one instance of
    200 customers with 200 ants (25-NN lists), one of 1000 customers with 256
    ants (30-NN), and the batch of 512 instances of 100-1000 customers with 128
    ants each (25-NN).  Same seeds and iterations for both; results are
    bit-identical, only time differs."""
    from . import instances as I
    from .aco import Batch, Problem, Solver, default_params

    def single(inst, ants, k, tuned):
        p = default_params(inst.n)
        p.mode, p.n_ants, p.nn_ants, p.nn_ls = _lib.MODE_THROUGHPUT, ants, k, k
        p.seed_time, p.rnd_seed = 1796300000, 4242
        with Solver(Problem.from_instance(inst), p, tune_table=table if tuned else None) as S:
            S.init()
            S.iterate(3)
            return S.time_iterations(iters) / iters

    def batch(tuned):
        p = default_params(1001)
        p.mode, p.n_ants, p.nn_ants, p.nn_ls = _lib.MODE_THROUGHPUT, 128, 25, 25
        p.seed_time, p.rnd_seed = 1796300000, 4242
        probs = [Problem.from_instance(x) for x in I.gen_batch(512, 512, 100, 1000)]
        with Batch(probs, p, tune_table=table if tuned else None) as B:
            B.init()
            B.iterate(3)
            return float(B.time_phases(5).sum()) / 5

    c2, c3 = I.gen_mixed(2026, 200), I.gen_large(3031, 1000)
    out = {}
    for name, fn in (("single_200x200", lambda t: single(c2, 200, 25, t)),
                     ("large_1000x256", lambda t: single(c3, 256, 30, t)),
                     ("batch_512x128", batch)):
        model, tuned = fn(False), fn(True)
        out[name] = {"model_ms": model, "table_ms": tuned, "table_over_model": tuned / model}
    return out


def main():
    ap = argparse.ArgumentParser(description="Build a launch-shape table for this GPU, or compare one with the "
                                             "library's create-time model.")
    ap.add_argument("--sizes", default="101,201,501,1001")
    ap.add_argument("--ants", type=int, default=128)
    ap.add_argument("--mode", choices=["throughput", "parity"], default="throughput")
    ap.add_argument("--iters", type=int, default=6)
    ap.add_argument("--batch", type=int, default=0,
                    help="tune a batch of this many instances of 100-1000 customers instead of single sizes")
    ap.add_argument("--compare", action="store_true", help="time the table against the model and print JSON")
    ap.add_argument("--out", default=DEFAULT_TABLE)
    a = ap.parse_args()
    mode = _lib.MODE_THROUGHPUT if a.mode == "throughput" else _lib.MODE_PARITY
    import os
    table = TuneTable.load(a.out) if os.path.exists(a.out) else TuneTable()
    if a.compare:
        print(json.dumps(compare(table), indent=1))
        return
    try:
        import torch
        table.device = torch.cuda.get_device_name(0)
    except Exception:
        pass
    if a.batch > 0:
        build_batch_entry(512, a.batch, 100, 1000, a.ants, iters=a.iters, table=table, log=print)
    else:
        build_table([int(v) for v in a.sizes.split(",")], a.ants, mode, a.iters, table=table, log=print)
    table.save(a.out)


if __name__ == "__main__":
    main()
