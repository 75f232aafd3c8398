"""The FP64 oracle of the edge-scoring network: its analytic gradient against
central finite differences, and the bf16 operand rounding it emulates."""
import numpy as np

from oracle import mpnn_oracle as M


def tiny_graph(seed, N=9, k=3):
    rng = np.random.default_rng(seed)
    nf = rng.uniform(0, 1, size=(N, M.F_NODE))
    nbr = np.array([rng.choice([j for j in range(N) if j != i], size=k, replace=False) for i in range(N)]).ravel()
    ef = rng.uniform(0, 1, size=N * k)
    y = (rng.uniform(size=N * k) < 0.3).astype(np.float64)
    return nf, ef, nbr, y


def loss_of(flat, nf, ef, nbr, k, y, w_pos):
    s, _ = M.forward(flat, nf, ef, nbr, k)
    return M.loss_and_dlogit(s, y, w_pos)[0]


def test_gradient_matches_finite_differences():
    k = 3
    nf, ef, nbr, y = tiny_graph(1, k=k)
    flat = M.init_params(7)
    rng = np.random.default_rng(3)
    flat = flat + rng.normal(0, 0.05, size=flat.shape)  # nonzero biases too
    s, saved = M.forward(flat, nf, ef, nbr, k)
    _, ds = M.loss_and_dlogit(s, y, 2.5)
    g = M.backward(flat, nf, ef, nbr, k, saved, ds)
    idx = rng.choice(flat.size, size=300, replace=False)
    eps = 1e-6
    for i in idx:
        fp = flat.copy(); fp[i] += eps
        fm = flat.copy(); fm[i] -= eps
        num = (loss_of(fp, nf, ef, nbr, k, y, 2.5) - loss_of(fm, nf, ef, nbr, k, y, 2.5)) / (2 * eps)
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(num), (i, num, g[i])


def test_param_layout_roundtrip():
    flat = M.init_params(2)
    assert flat.size == M.param_count()
    d = M.unpack(flat)
    assert np.array_equal(M.pack(d), flat)
    assert d["W0"].shape == (4 * M.H, M.H) and d["w_o"].shape == (M.H,)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-8, 1.0 + 2**-9, -2.5, 3.0e38], np.float32)
    r = M.bf16_round(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                       # halfway, ties to even (mantissa ...0)
    assert r[2] == 1.0 + 4 * 2**-8           # halfway, ties to even (rounds up)
    assert r[3] == 1.0                       # below half
    assert r[4] == -2.5
    assert np.isfinite(r[5])


def test_bf16_forward_close_to_fp64():
    k = 3
    nf, ef, nbr, _ = tiny_graph(4, N=12, k=k)
    flat = M.init_params(5)
    s64, _ = M.forward(flat, nf, ef, nbr, k)
    s16, _ = M.forward(flat, nf, ef, nbr, k, bf16=True)
    assert np.max(np.abs(s64 - s16)) < 0.05 * (1 + np.max(np.abs(s64)))
