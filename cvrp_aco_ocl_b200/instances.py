"""Seeded synthetic CVRP instances and VRPLIB text I/O.

The reference ships public VRPLIB files and reads them with
``read_instance_file`` (cvrp_ocl/io.cpp:334-517).  The benchmark workloads here
are synthetic stand-ins with the shapes and value distributions of the five
workload configurations (plain ACO n=50; n=200 clustered; n=1000; a batch of 512
instances n in [100, 1000]; the learned-prior training set).  Node 0 is the
depot, nodes 1..n are customers, distances are EUC_2D in fp32 without rounding
(cvrp_ocl/vrpHelper.cpp:67-81), there is no maximum route distance and no
service time.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

EUC_2D, CEIL_2D, GEO, ATT = 0, 1, 2, 3
DIST_TYPES = {"EUC_2D": EUC_2D, "CEIL_2D": CEIL_2D, "GEO": GEO, "ATT": ATT}


@dataclasses.dataclass
class Instance:
    """Host-side CVRP instance (the fields of ``Problem`` the path reads,
    cvrp_ocl/problem.h:82-99)."""

    name: str
    x: np.ndarray  # float32 [n], node 0 = depot
    y: np.ndarray  # float32 [n]
    demand: np.ndarray  # int32 [n], demand[0] = 0
    capacity: int
    max_distance: float = math.inf
    service_time: float = 0.0
    dist_type: int = EUC_2D
    optimum: float = 0.0
    seed: Optional[int] = None

    @property
    def n(self) -> int:
        """Number of nodes, depot included (``num_node``)."""
        return int(self.x.shape[0])


def _finish(name, xs, ys, dem, capacity, seed) -> Instance:
    return Instance(
        name=name,
        x=np.ascontiguousarray(xs, dtype=np.float32),
        y=np.ascontiguousarray(ys, dtype=np.float32),
        demand=np.ascontiguousarray(dem, dtype=np.int32),
        capacity=int(capacity),
        seed=seed,
    )


def gen_uniform_small(seed: int, n_customers: int = 50, coord_max: int = 100,
                      demand_max: int = 30, capacity: int = 160) -> Instance:
    """Plain-ACO CPU workload: integer coordinates uniform in [0, coord_max]^2 for
    the depot and the customers, integer demand uniform in [1, demand_max]."""
    rng = np.random.default_rng(seed)
    n = n_customers + 1
    xs = rng.integers(0, coord_max + 1, size=n).astype(np.float32)
    ys = rng.integers(0, coord_max + 1, size=n).astype(np.float32)
    dem = rng.integers(1, demand_max + 1, size=n).astype(np.int32)
    dem[0] = 0
    return _finish(f"U{n_customers}_s{seed}", xs, ys, dem, capacity, seed)


def _clustered_coords(rng, k: int, n_clusters: int = 8, sigma: float = 40.0, side: float = 1000.0):
    centres = rng.uniform(0.0, side, size=(n_clusters, 2))
    which = rng.integers(0, n_clusters, size=k)
    pts = centres[which] + rng.normal(0.0, sigma, size=(k, 2))
    return np.clip(pts, 0.0, side)


def gen_mixed(seed: int, n_customers: int = 200, customers_per_route: float = 12.0) -> Instance:
    """Single-instance GPU workload: half the customers uniform in [0, 1000]^2,
    half from 8 Gaussian clusters (sigma 40, clipped), depot at the centre,
    integer demand uniform in [1, 100], capacity = round(customers_per_route *
    mean demand)."""
    rng = np.random.default_rng(seed)
    k_uni = n_customers // 2
    uni = rng.uniform(0.0, 1000.0, size=(k_uni, 2))
    clu = _clustered_coords(rng, n_customers - k_uni)
    pts = np.concatenate([uni, clu], axis=0)
    xs = np.concatenate([[500.0], pts[:, 0]])
    ys = np.concatenate([[500.0], pts[:, 1]])
    dem = np.concatenate([[0], rng.integers(1, 101, size=n_customers)])
    cap = int(round(customers_per_route * float(dem[1:].mean())))
    return _finish(f"M{n_customers}_s{seed}", xs, ys, dem, max(cap, int(dem.max())), seed)


def gen_large(seed: int, n_customers: int = 1000, customers_per_route: float = 15.0) -> Instance:
    """Large-instance workload: coordinates uniform or clustered (seeded choice),
    depot random / centre / corner, demand uniform [1, 100] or 80% small [1, 10]
    and 20% large [50, 100], capacity = round(customers_per_route * mean demand)."""
    rng = np.random.default_rng(seed)
    if rng.integers(0, 2) == 0:
        pts = rng.uniform(0.0, 1000.0, size=(n_customers, 2))
        kind = "u"
    else:
        pts = _clustered_coords(rng, n_customers)
        kind = "c"
    depot_kind = int(rng.integers(0, 3))
    if depot_kind == 0:
        depot = rng.uniform(0.0, 1000.0, size=2)
    elif depot_kind == 1:
        depot = np.array([500.0, 500.0])
    else:
        depot = np.array([0.0, 0.0])
    if rng.integers(0, 2) == 0:
        dem = rng.integers(1, 101, size=n_customers)
    else:
        small = rng.random(n_customers) < 0.8
        dem = np.where(small, rng.integers(1, 11, size=n_customers), rng.integers(50, 101, size=n_customers))
    dem = np.concatenate([[0], dem])
    cap = int(round(customers_per_route * float(dem[1:].mean())))
    xs = np.concatenate([[depot[0]], pts[:, 0]])
    ys = np.concatenate([[depot[1]], pts[:, 1]])
    return _finish(f"L{n_customers}{kind}{depot_kind}_s{seed}", xs, ys, dem, max(cap, int(dem.max())), seed)


def gen_batch(seed: int, count: int = 512, n_min: int = 100, n_max: int = 1000) -> List[Instance]:
    """Batched workload: `count` independent instances, customer count uniform in
    [n_min, n_max], drawn alternately from the mixed and the large generators."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(count):
        nc = int(rng.integers(n_min, n_max + 1))
        s = int(rng.integers(0, 2**31 - 1))
        out.append(gen_mixed(s, nc) if b % 2 == 0 else gen_large(s, nc))
    return out


def write_vrplib(inst: Instance, path: str) -> None:
    """Write an instance in the VRPLIB text layout ``read_instance_file`` parses
    (cvrp_ocl/io.cpp:353-512).  Coordinates are printed with 9 significant
    digits, which round-trips every fp32 value.  DISTANCE, SERVICE_TIME and
    COMMENT must carry an attached colon: the reader scans a float right after
    the key token (io.cpp:365-372, 459-474)."""
    lines = [  # "KEY: value" with the colon attached, as the reference's own datasets write it
        f"NAME: {inst.name}",
        f"COMMENT: {inst.optimum:.9g}",
        "TYPE: CVRP",
        f"DIMENSION: {inst.n}",
        "EDGE_WEIGHT_TYPE: " + {v: k for k, v in DIST_TYPES.items()}[inst.dist_type],
        f"CAPACITY: {inst.capacity}",
    ]
    if math.isfinite(inst.max_distance):
        lines.append(f"DISTANCE: {inst.max_distance:.9g}")
    if inst.service_time:
        lines.append(f"SERVICE_TIME: {inst.service_time:.9g}")
    lines.append("NODE_COORD_SECTION")
    for i in range(inst.n):
        lines.append(f"{i + 1} {float(inst.x[i]):.9g} {float(inst.y[i]):.9g}")
    lines.append("DEMAND_SECTION")
    for i in range(inst.n):
        lines.append(f"{i + 1} {int(inst.demand[i])}")
    lines.append("DEPOT_SECTION")
    lines.append("1")
    lines.append("-1")
    lines.append("EOF")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
