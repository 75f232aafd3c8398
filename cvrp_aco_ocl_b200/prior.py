"""Learned sampling prior: an edge-scoring message-passing network whose output
multiplies eta^beta in the ant colony's choice weights.

* ``build_graph``: the k-nearest-customer graph of an instance (the
  reference's neighbour-list rule, cvrp_ocl/vrpHelper.cpp:188-236) with node
  features (x, y, demand/capacity, is_depot, distance to the depot) and edge
  feature distance, all lengths divided by the bounding box's longer side.
* ``EdgeScorer``: parameters on the device; forward, gradient and Adam steps
  are the hand-written kernels of csrc/mpnn.cu (tcgen05 BF16 products, FP32
  accumulation) called through the C ABI.  PyTorch only holds device memory.
* ``make_training_set`` labels edges with the best tours the GPU colony itself
  finds (batched plain ACO); ``train`` fits the network to them.
* ``prior_matrix`` turns edge logits into the dense prior ``aco_set_prior``
  takes: sigmoid(score)^gamma on graph edges, ``floor`` elsewhere.  Feasibility
  and tour lengths are untouched; the plain colony (no prior) stays the
  fallback and the yardstick.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import os
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import AcoError, check, lib

K_GRAPH = 20
LAYERS = 3
DEFAULT_GAMMA = 2.0  # prior exponent: the best final lengths of the 0.5 / 1 / 2 sweep on held-out instances
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "edge_prior_k20_l3.npz")
HIDDEN = 64
NODE_FEATURES = 5


@dataclasses.dataclass
class Graph:
    n: int
    k: int
    node_feat: np.ndarray   # (n, 5) float32
    edge_feat: np.ndarray   # (n*k,) float32
    nbr: np.ndarray         # (n*k,) int32, local node ids
    dist: np.ndarray        # (n, n) float32 (the instance's distances)


def build_graph(problem, k: int = K_GRAPH, keep_dist: bool = True) -> Graph:
    """k nearest customers of every node (depot and self excluded) with the
    network's input features (keep_dist=False drops the n x n distances)."""
    from .aco import compute_distances, compute_nn_lists

    n = problem.num_node
    if n - 2 < k:
        raise ValueError(f"graph degree {k} needs at least {k + 2} nodes, the instance has {n}")
    x = np.asarray(problem.x, np.float32)
    y = np.asarray(problem.y, np.float32)
    dist = problem.distance if problem.distance is not None else compute_distances(x, y, problem.dis_type)
    nn = compute_nn_lists(dist, k, k)[:, :k]
    xmin, ymin = float(x.min()), float(y.min())
    s = max(float(x.max()) - xmin, float(y.max()) - ymin)
    s = s if s > 0 else 1.0
    nf = np.zeros((n, NODE_FEATURES), np.float32)
    nf[:, 0] = (x - xmin) / s
    nf[:, 1] = (y - ymin) / s
    nf[:, 2] = np.asarray(problem.demand, np.float32) / float(problem.vehicle_capacity)
    nf[0, 3] = 1.0
    nf[:, 4] = dist[:, 0] / s
    rows = np.repeat(np.arange(n), k)
    ef = (dist[rows, nn.ravel()] / s).astype(np.float32)
    return Graph(n, k, nf, ef, nn.ravel().astype(np.int32), dist if keep_dist else None)


def route_labels(g: Graph, tour) -> np.ndarray:
    """1 for graph edges (i, j) whose undirected edge {i, j} joins consecutive
    nodes of the tour (depot hops included), else 0."""
    t = np.asarray(tour, np.int64)
    a, b = t[:-1], t[1:]
    keys = np.concatenate([a * g.n + b, b * g.n + a])
    rows = np.repeat(np.arange(g.n, dtype=np.int64), g.k)
    return np.isin(rows * g.n + g.nbr.astype(np.int64), keys).astype(np.float32)


class GraphBatch:
    """Graphs concatenated node-wise on the device (global neighbour ids)."""

    def __init__(self, graphs: Sequence[Graph], labels: Optional[Sequence[np.ndarray]] = None, device: int = 0):
        import torch

        k = graphs[0].k
        if any(g.k != k for g in graphs):
            raise ValueError("all graphs of a batch need the same degree")
        offs = np.cumsum([0] + [g.n for g in graphs])
        self.k, self.n_nodes, self.offsets = k, int(offs[-1]), offs
        dev = torch.device("cuda", device)
        self.node_feat = torch.from_numpy(np.concatenate([g.node_feat for g in graphs])).to(dev)
        self.edge_feat = torch.from_numpy(np.concatenate([g.edge_feat for g in graphs])).to(dev)
        nbr = np.concatenate([g.nbr + o for g, o in zip(graphs, offs[:-1])]).astype(np.int32)
        self.nbr = torch.from_numpy(nbr).to(dev)
        self.labels = None
        if labels is not None:
            self.labels = torch.from_numpy(np.concatenate(labels).astype(np.float32)).to(dev)

    @property
    def n_edges(self) -> int:
        return self.n_nodes * self.k


def init_params(seed: int, layers: int = LAYERS) -> np.ndarray:
    """Weights uniform in +-1/sqrt(fan_in), biases zero, in the packed order of
    aco_mpnn_param_count (embeddings, layers (W, b, A, a), head)."""
    rng = np.random.default_rng(seed)
    H, F = HIDDEN, NODE_FEATURES
    parts = []

    def w(rows, cols):
        b = 1.0 / math.sqrt(cols)
        parts.append(rng.uniform(-b, b, size=rows * cols))

    def z(m):
        parts.append(np.zeros(m))

    w(H, F); z(H); w(H, 1); z(H)
    for _ in range(layers):
        w(4 * H, H); z(4 * H); w(H, H); z(H)
    w(H, H); z(H); w(1, H); z(1)
    flat = np.concatenate(parts).astype(np.float32)
    assert flat.size == lib().aco_mpnn_param_count(layers)
    return flat


class EdgeScorer:
    """Parameters (FP32 master copy) and optimiser state on one GPU."""

    def __init__(self, layers: int = LAYERS, seed: int = 0, params: Optional[np.ndarray] = None, device: int = 0):
        import torch

        self.layers, self.device = layers, device
        self.count = lib().aco_mpnn_param_count(layers)
        if self.count <= 0:
            raise AcoError(self.count, "aco_mpnn_param_count")
        p = init_params(seed, layers) if params is None else np.asarray(params, np.float32)
        if p.size != self.count:
            raise ValueError(f"expected {self.count} parameters, got {p.size}")
        dev = torch.device("cuda", device)
        self.params = torch.from_numpy(p.copy()).to(dev)
        self.grad = torch.zeros(self.count, dtype=torch.float32, device=dev)
        self.m = torch.zeros_like(self.grad)
        self.v = torch.zeros_like(self.grad)
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)
        self.step = 0
        self._ws = None
        self._ws_bytes = 0

    # -- device plumbing
    def _workspace(self, n_nodes: int, k: int):
        import torch

        b = ctypes.c_size_t()
        check(lib().aco_mpnn_workspace_bytes(n_nodes, k, self.layers, ctypes.byref(b)), "aco_mpnn_workspace_bytes")
        if self._ws is None or self._ws_bytes < b.value:
            self._ws = torch.empty(b.value, dtype=torch.uint8, device=torch.device("cuda", self.device))
            self._ws_bytes = b.value
        return self._ws

    @staticmethod
    def _stream():
        import torch

        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def _status(self):
        rc = lib().aco_mpnn_status(ctypes.c_void_p(self._ws.data_ptr()), self._stream())
        if rc != 0:
            raise AcoError(rc, "edge-scoring network")

    # -- inference and training steps
    def scores(self, batch: GraphBatch):
        """Edge logits (device tensor, n_edges)."""
        import torch

        ws = self._workspace(batch.n_nodes, batch.k)
        out = torch.empty(batch.n_edges, dtype=torch.float32, device=self.params.device)
        check(lib().aco_mpnn_forward(batch.n_nodes, batch.k, self.layers, self.params.data_ptr(),
                                     batch.node_feat.data_ptr(), batch.edge_feat.data_ptr(), batch.nbr.data_ptr(),
                                     ctypes.c_void_p(ws.data_ptr()), ws.numel(), out.data_ptr(), self._stream()),
              "aco_mpnn_forward")
        self._status()
        return out

    def compute_grad(self, batch: GraphBatch, pos_weight: float, sync: bool = True):
        """Loss gradient into self.grad, loss into self.loss; returns the logits."""
        import torch

        ws = self._workspace(batch.n_nodes, batch.k)
        out = torch.empty(batch.n_edges, dtype=torch.float32, device=self.params.device)
        check(lib().aco_mpnn_grad(batch.n_nodes, batch.k, self.layers, self.params.data_ptr(),
                                  batch.node_feat.data_ptr(), batch.edge_feat.data_ptr(), batch.nbr.data_ptr(),
                                  batch.labels.data_ptr(), float(pos_weight), ctypes.c_void_p(ws.data_ptr()),
                                  ws.numel(), self.grad.data_ptr(), self.loss.data_ptr(), out.data_ptr(),
                                  self._stream()), "aco_mpnn_grad")
        if sync:
            self._status()
        return out

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
        self.step += 1
        check(lib().aco_mpnn_adam(self.count, self.params.data_ptr(), self.grad.data_ptr(), self.m.data_ptr(),
                                  self.v.data_ptr(), lr, beta1, beta2, eps, self.step, self._stream()),
              "aco_mpnn_adam")

    # -- persistence
    def state(self) -> np.ndarray:
        return self.params.detach().cpu().numpy().copy()

    def save(self, path: str, meta: Optional[Dict] = None) -> None:
        np.savez(path, params=self.state(), layers=self.layers, k=K_GRAPH,
                 meta=np.array(json_dumps(meta or {})))

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS, device: int = 0) -> "EdgeScorer":
        """Weights saved by ``save`` (default: the network trained on 20k
        colony-labelled instances with 100-500 nodes, shipped with the package)."""
        d = np.load(path)
        return cls(layers=int(d["layers"]), params=d["params"], device=device)

    # -- prior for the colony
    def prior(self, problem, gamma: float = DEFAULT_GAMMA, floor: float = 1e-3, k: int = K_GRAPH,
              graph: Optional[Graph] = None) -> np.ndarray:
        g = graph or build_graph(problem, k)
        s = self.scores(GraphBatch([g], device=self.device)).cpu().numpy()
        return prior_matrix(g, s, gamma, floor)


def json_dumps(d) -> str:
    import json

    return json.dumps(d)


def prior_matrix(g: Graph, scores: np.ndarray, gamma: float = DEFAULT_GAMMA, floor: float = 1e-3) -> np.ndarray:
    """Dense n x n prior: sigmoid(score)^gamma on graph edges (at least floor),
    floor elsewhere (the diagonal and non-graph pairs)."""
    pr = np.full((g.n, g.n), floor, np.float32)
    sig = 1.0 / (1.0 + np.exp(-np.asarray(scores, np.float64)))
    val = np.maximum(sig ** gamma, floor).astype(np.float32)
    rows = np.repeat(np.arange(g.n), g.k)
    pr[rows, g.nbr] = val
    return pr


# ---------------------------------------------------------------------------
def make_training_set(count: int, n_min: int, n_max: int, seed: int, iters: int = 100, ants: int = 128,
                      chunk: int = 512, k: int = K_GRAPH, log=None):
    """Generated instances (mixed and large generators alternately) labelled
    with the best tour plain batched GPU ACO finds in `iters` iterations."""
    from . import instances as I
    from ._lib import MODE_THROUGHPUT
    from .aco import Batch, Problem, default_params

    insts = I.gen_batch(seed, count, n_min - 1, n_max - 1)
    graphs, labels, costs = [], [], []
    t0 = time.perf_counter()
    for c0 in range(0, count, chunk):
        probs = [Problem.from_instance(x) for x in insts[c0:c0 + chunk]]
        p = default_params(max(pr.num_node for pr in probs))
        p.mode, p.n_ants, p.nn_ants, p.nn_ls = MODE_THROUGHPUT, ants, 25, 25
        p.seed_time, p.rnd_seed = 1796300000, seed + c0
        with Batch(probs, p) as B:
            B.init()
            B.iterate(iters)
            for b, pr in enumerate(probs):
                tour, length = B.best(b)
                g = build_graph(pr, k, keep_dist=False)
                graphs.append(g)
                labels.append(route_labels(g, tour))
                costs.append(length)
        if log:
            log(f"labelled {min(c0 + chunk, count)}/{count} instances ({time.perf_counter() - t0:.1f} s)")
    return graphs, labels, costs


def train(scorer: EdgeScorer, graphs: List[Graph], labels: List[np.ndarray], epochs: int = 10,
          graphs_per_step: int = 32, lr: float = 1e-3, pos_weight: Optional[float] = None, seed: int = 0,
          log=None) -> List[float]:
    """Adam on the weighted BCE over shuffled mini-batches of whole graphs;
    returns the mean loss of every epoch."""
    import torch

    if pos_weight is None:  # balance the ~2/k positive rate
        pos = float(np.mean(np.concatenate(labels)))
        pos_weight = (1.0 - pos) / max(pos, 1e-6)
    rng = np.random.default_rng(seed)
    hist = []
    # batches are built once and reused (device copies), shuffled by batch each epoch
    order = rng.permutation(len(graphs))
    batches = [GraphBatch([graphs[i] for i in order[s:s + graphs_per_step]],
                          [labels[i] for i in order[s:s + graphs_per_step]], device=scorer.device)
               for s in range(0, len(graphs), graphs_per_step)]
    for ep in range(epochs):
        tot = torch.zeros(1, dtype=torch.float32, device=scorer.params.device)
        for bi in rng.permutation(len(batches)):
            scorer.compute_grad(batches[bi], pos_weight, sync=False)
            tot += scorer.loss
            scorer.adam(lr)
        scorer._status()
        hist.append(float(tot.item()) / len(batches))
        if log:
            log(f"epoch {ep + 1}/{epochs}: loss {hist[-1]:.4f}")
    return hist
