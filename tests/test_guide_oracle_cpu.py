"""The float64 restatement of the learned proposal's network
(oracle/guide_fp64.py) checked by central finite differences: its analytic
gradients of the weighted log-likelihood of the blend of the phase function
and the von Mises-Fisher mixture (with its selection probability) are the
derivatives of its own loss (the GPU kernels implement the same formulas and
are checked against this restatement on a B200)."""
import numpy as np

import guide_fp64 as G


def test_analytic_gradient_equals_finite_differences():
    rng = np.random.default_rng(7)
    rows = 6
    X = np.stack([G.encode(rng.random(3), (lambda v: v / np.linalg.norm(v))(rng.normal(size=3)), 1)
                  for _ in range(rows)])
    d = rng.normal(size=(rows, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    T = np.concatenate([d, rng.uniform(0.5, 2.0, (rows, 1)), rng.uniform(0.02, 1.0, (rows, 1))], axis=1)
    w_off, b_off, n = G.param_layout()
    P = rng.normal(0, 0.2, n)
    _, _, g = G.forward_backward(P, X, T, fp16_like_gpu=False)
    idx = list(rng.integers(0, n, 60)) + [b_off[3] + j for j in range(41)]
    h = 1e-6
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        lp = G.forward_backward(Pp, X, T, fp16_like_gpu=False)[1]
        lm = G.forward_backward(Pm, X, T, fp16_like_gpu=False)[1]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_encoding_layout():
    x = G.encode(np.array([0.25, 0.5, 0.75]), np.array([0.0, 0.0, 1.0]), 3)
    assert x.shape == (G.IN,)
    assert np.isclose(x[0], np.sin(np.pi * 0.25)) and np.isclose(x[1], np.cos(np.pi * 0.25))
    assert x[72:75].tolist() == [0.0, 0.0, 1.0]
    assert x[75 + 3] == 1.0 and x[75:95].sum() == 1.0 and x[95] == 0.0


def test_selection_probability_follows_the_fit():
    """Where the phase function explains the target better than the mixture
    the loss pushes the selection probability down, and up where the
    mixture explains it better."""
    o = np.zeros(G.OUT)
    o[G.LOBES:4 * G.LOBES] = np.tile([0.0, 0.0, 1.0], G.LOBES)   # every lobe along +z
    o[4 * G.LOBES:5 * G.LOBES] = np.log(50.0)                    # sharp lobes
    toward = np.array([0.0, 0.0, 1.0, 1.0, 0.01])   # target along the lobes, phase pdf low
    away = np.array([1.0, 0.0, 0.0, 1.0, 0.5])      # target off the lobes, phase pdf high
    assert G.row_loss_grad(o, toward, 1.0)[1][G.ALPHA_COL] < 0    # descent raises a
    assert G.row_loss_grad(o, away, 1.0)[1][G.ALPHA_COL] > 0      # descent lowers a
