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

SHAPE_FIELDS = ("ants_per_block", "warps_per_ant", "ls_warps", "stage_matrix", "ls_ants")


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

    def lookup(self, n: int, mode: int, ants: int) -> Optional[TuneEntry]:
        """The entry of this mode whose node range holds n, with the nearest ant
        count (ratio distance); None when no range holds n."""
        hits = [e for e in self.entries if e.mode == mode and e.n_lo <= n <= e.n_hi]
        if not hits:
            return None
        return min(hits, key=lambda e: abs((e.ants / max(ants, 1)) - 1.0))

    def apply(self, params: AcoParams, n: int) -> AcoParams:
        """Fill the launch-shape fields the caller left at 0 (autotuned) from the
        entry for n; fields set by the caller are kept."""
        e = self.lookup(n, params.mode, params.n_ants if params.n_ants > 0 else n)
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
    """Tune one synthetic instance (the mixed generator) per size and record
    the winners over the size ranges of `size_ranges`."""
    from .aco import Problem, default_params
    from .instances import gen_mixed

    table = table or TuneTable()
    for (lo, hi), n in zip(size_ranges(sizes), sorted(set(int(v) for v in sizes))):
        prob = Problem.from_instance(gen_mixed(seed + n, n - 1))
        p = default_params(n)
        p.mode, p.n_ants = mode, ants
        p.nn_ants = min(nn_ants, n - 2)
        p.nn_ls = min(p.nn_ls, 25)
        p.seed_time, p.rnd_seed = 1796300000, seed
        t0 = time.perf_counter()
        out, ms = autotune(prob, p, iters)
        e = TuneEntry(mode, lo, hi, ants, out.ants_per_block, out.warps_per_ant, out.ls_warps, out.stage_matrix,
                      ms, p.nn_ants, out.ls_ants)
        table.add(e)
        if log:
            log(f"n={n} [{lo},{hi}] ants={ants}: apc={e.ants_per_block} wpa={e.warps_per_ant} "
                f"ls_warps={e.ls_warps} ls_ants={e.ls_ants} stage={e.stage_matrix} {ms:.3f} ms/iter ({time.perf_counter() - t0:.1f} s)")
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


def main():
    ap = argparse.ArgumentParser(description="Build a launch-shape table for this GPU.")
    ap.add_argument("--sizes", default="101,201,501,1001")
    ap.add_argument("--ants", type=int, default=128)
    ap.add_argument("--mode", choices=["throughput", "parity"], default="throughput")
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    mode = _lib.MODE_THROUGHPUT if a.mode == "throughput" else _lib.MODE_PARITY
    import os
    table = TuneTable.load(a.out) if os.path.exists(a.out) else TuneTable()
    try:
        import torch
        table.device = torch.cuda.get_device_name(0)
    except Exception:
        pass
    build_table([int(v) for v in a.sizes.split(",")], a.ants, mode, a.iters, table=table, log=print)
    table.save(a.out)


if __name__ == "__main__":
    main()
