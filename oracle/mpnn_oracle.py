"""CPU oracle of the edge-scoring message-passing network (test infrastructure).

The network has no reference counterpart (the reference has no learned
component); this is the FP64 restatement the device kernels are checked
against.  Only tests import it.

Graph: every node i has k out-edges to its k nearest customers (the
reference's neighbour-list rule, cvrp_ocl/vrpHelper.cpp:188-236: the depot and
i itself excluded).  Node features f_i = (x, y, demand/capacity, is_depot,
d(i, depot)), coordinates shifted to the bounding-box corner and divided by its
longer side s; edge feature d_ij / s.

    h0 = W_n f + b_n                      e0 = W_e d + b_e
    per layer l:
      P   = h W_l^T + b_l                 (columns U | V | B | C, 64 each)
      q   = e A_l^T + a_l + B_i + C_j
      e'  = e + relu(q)
      g   = sigmoid(e')
      u_i = U_i + (1/k) sum_j g_ij * V_j
      h'  = h + relu(u)
    z = relu(e W_h^T + b_h);  s = z . w_o + b_o          (edge logit)
    loss = mean over edges of  -(w_pos y log sig(s) + (1 - y) log(1 - sig(s)))

With ``bf16=True`` every GEMM operand (activation and weight) is rounded to
bfloat16 (round to nearest even) before the FP64 product, as the tensor-core
kernels do; everything else stays FP64.
"""
from __future__ import annotations

import numpy as np

H = 64
F_NODE = 5
LAYERS = 3


def param_shapes(layers: int = LAYERS):
    """Named parameter shapes in the packed order of the device buffer."""
    s = [("W_n", (H, F_NODE)), ("b_n", (H,)), ("W_e", (H, 1)), ("b_e", (H,))]
    for l in range(layers):
        s += [(f"W{l}", (4 * H, H)), (f"b{l}", (4 * H,)), (f"A{l}", (H, H)), (f"a{l}", (H,))]
    s += [("W_h", (H, H)), ("b_h", (H,)), ("w_o", (H,)), ("b_o", (1,))]
    return s


def param_count(layers: int = LAYERS) -> int:
    return int(sum(np.prod(sh) for _, sh in param_shapes(layers)))


def unpack(flat: np.ndarray, layers: int = LAYERS):
    out, o = {}, 0
    for name, sh in param_shapes(layers):
        m = int(np.prod(sh))
        out[name] = flat[o:o + m].reshape(sh)
        o += m
    return out


def pack(d, layers: int = LAYERS) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in param_shapes(layers)])


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float64."""
    x = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    lsb = (x >> 16) & 1
    r = ((x + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _mm(x, w, bf16):
    """x @ w.T with optional bfloat16 operands."""
    if bf16:
        x = bf16_round(x.astype(np.float32))
        w = bf16_round(w.astype(np.float32))
    return x @ w.T


def sigmoid(x):
    return 0.5 * (1.0 + np.tanh(0.5 * x))


def forward(flat, node_feat, edge_feat, nbr, k, layers: int = LAYERS, bf16: bool = False):
    """Edge logits s (E,) and the saved activations for backward.

    node_feat (N, 5), edge_feat (E,) with E = N*k, nbr (E,) global node ids;
    the out-edges of node i are rows i*k .. i*k+k-1."""
    p = unpack(np.asarray(flat, np.float64), layers)
    N = node_feat.shape[0]
    src = np.repeat(np.arange(N), k)
    h = node_feat.astype(np.float64) @ p["W_n"].T + p["b_n"]
    e = edge_feat.astype(np.float64)[:, None] * p["W_e"][:, 0][None, :] + p["b_e"]
    saved = {"h": [h], "e": [e], "P": [], "q": [], "g": [], "u": []}
    for l in range(layers):
        P = _mm(h, p[f"W{l}"], bf16) + p[f"b{l}"]
        U, V, B, C = P[:, :H], P[:, H:2 * H], P[:, 2 * H:3 * H], P[:, 3 * H:]
        q = _mm(e, p[f"A{l}"], bf16) + p[f"a{l}"] + B[src] + C[nbr]
        e = e + np.maximum(q, 0.0)
        g = sigmoid(e)
        agg = (g * V[nbr]).reshape(N, k, H).sum(axis=1) / k
        u = U + agg
        h = h + np.maximum(u, 0.0)
        saved["P"].append(P); saved["q"].append(q); saved["g"].append(g); saved["u"].append(u)
        saved["h"].append(h); saved["e"].append(e)
    zpre = _mm(e, p["W_h"], bf16) + p["b_h"]
    z = np.maximum(zpre, 0.0)
    s = z @ p["w_o"] + p["b_o"][0]
    saved.update(zpre=zpre, z=z, src=src)
    return s, saved


def loss_and_dlogit(s, y, w_pos: float):
    """Mean weighted BCE with logits and its derivative with respect to s."""
    s = np.asarray(s, np.float64)
    y = np.asarray(y, np.float64)
    E = s.shape[0]
    ls = -np.logaddexp(0.0, -s)        # log sig(s)
    l1s = -np.logaddexp(0.0, s)        # log (1 - sig(s))
    loss = -(w_pos * y * ls + (1.0 - y) * l1s).sum() / E
    sg = sigmoid(s)
    ds = (w_pos * y * (sg - 1.0) + (1.0 - y) * sg) / E
    return loss, ds


def backward(flat, node_feat, edge_feat, nbr, k, saved, ds, layers: int = LAYERS, bf16: bool = False):
    """Gradient of the loss with respect to the packed parameters, given
    dL/ds.  With bf16, the weight operands of the input-gradient GEMMs and
    both operands of the weight-gradient GEMMs are rounded as on the device."""
    p = unpack(np.asarray(flat, np.float64), layers)
    gr = {name: np.zeros(sh) for name, sh in param_shapes(layers)}
    N = node_feat.shape[0]
    src = saved["src"]
    r = (lambda a: bf16_round(a.astype(np.float32))) if bf16 else (lambda a: a)

    # head
    z, zpre, eL = saved["z"], saved["zpre"], saved["e"][-1]
    gr["b_o"][0] = ds.sum()
    gr["w_o"] = z.T @ ds
    dz = ds[:, None] * p["w_o"][None, :] * (zpre > 0)
    gr["b_h"] = dz.sum(0)
    gr["W_h"] = r(dz).T @ r(eL)
    de = r(dz) @ r(p["W_h"])
    dh = np.zeros((N, H))
    for l in reversed(range(layers)):
        P, q, g, u = saved["P"][l], saved["q"][l], saved["g"][l], saved["u"][l]
        e_in = saved["e"][l]
        h_in = saved["h"][l]
        V = P[:, H:2 * H]
        du = dh * (u > 0)                   # h' = h + relu(u); dh passes through the residual
        dP = np.zeros((N, 4 * H))
        dP[:, :H] = du
        du_e = du[src] / k                  # per edge
        dg = du_e * V[nbr]
        np.add.at(dP[:, H:2 * H], nbr, du_e * g)
        de_tot = de + dg * g * (1.0 - g)    # e' feeds the gate and later layers
        dq = de_tot * (q > 0)
        gr[f"a{l}"] = dq.sum(0)
        gr[f"A{l}"] = r(dq).T @ r(e_in)
        de = de_tot + r(dq) @ r(p[f"A{l}"])
        dP[:, 2 * H:3 * H] = dq.reshape(N, k, H).sum(1)
        np.add.at(dP[:, 3 * H:], nbr, dq)
        gr[f"b{l}"] = dP.sum(0)
        gr[f"W{l}"] = r(dP).T @ r(h_in)
        dh = dh + r(dP) @ r(p[f"W{l}"])
    gr["b_n"] = dh.sum(0)
    gr["W_n"] = dh.T @ node_feat.astype(np.float64)
    gr["b_e"] = de.sum(0)
    gr["W_e"][:, 0] = de.T @ edge_feat.astype(np.float64)
    return pack(gr, layers)


def init_params(seed: int, layers: int = LAYERS) -> np.ndarray:
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, sh in param_shapes(layers):
        if len(sh) == 2:
            b = 1.0 / np.sqrt(sh[1])
            d[name] = rng.uniform(-b, b, size=sh)
        elif name == "w_o":
            b = 1.0 / np.sqrt(H)
            d[name] = rng.uniform(-b, b, size=sh)
        else:
            d[name] = np.zeros(sh)
    return pack(d, layers)
