"""The learned proposal for scattering in media (-guide <n>).

* Its FP16 tensor-core forward and backward kernels against the float64
  restatement (oracle/guide_fp64.py) on the same parameters and batch: the
  outputs, the loss and the gradient of every parameter matrix.
* Online training on the light subpaths' medium records lowers the loss.
* Unbiasedness: the converged guided image equals the plain method's within
  the noise of two independent plain renders (the proposal changes only
  which directions camera paths sample and, through the MIS recursion, how
  techniques are weighted -- never the expected value).
"""
import ctypes

import numpy as np
import pytest

from gpuupbp_b200 import scenes

pytestmark = pytest.mark.gpu


def _batch(rows, seed):
    import guide_fp64 as G
    rng = np.random.default_rng(seed)
    X = np.stack([G.encode(rng.random(3), (lambda v: v / np.linalg.norm(v))(rng.normal(size=3)), int(rng.integers(3)))
                  for _ in range(rows)])
    d = rng.normal(size=(rows, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    T = np.concatenate([d, rng.uniform(0.1, 2.0, size=(rows, 1)), rng.uniform(0.02, 1.0, size=(rows, 1))], axis=1)
    return X.astype(np.float32), T.astype(np.float32)


def _params(seed):
    import guide_fp64 as G
    rng = np.random.default_rng(seed)
    _, _, n = G.param_layout()
    p = np.zeros(n)
    w_off, b_off, _ = G.param_layout()
    for l, (i, o) in enumerate(G.LAYERS):
        p[w_off[l]:w_off[l] + i * o] = rng.normal(0, np.sqrt(2.0 / i), i * o) * (0.3 if l == 3 else 1.0)
        p[b_off[l]:b_off[l] + o] = rng.normal(0, 0.1, o)
    return p.astype(np.float32)


def test_tensor_core_training_kernels_match_float64():
    import guide_fp64 as G
    from gpuupbp_b200 import upbp
    L = upbp.load_library()
    rows = 2048
    X, T = _batch(rows, 3)
    P = _params(4)
    grads = np.zeros(len(P), np.float32)
    out = np.zeros((rows, G.OUT), np.float32)
    loss = ctypes.c_float()
    assert L.upbp_guide_gradients(P.ctypes.data, len(P), X.ctypes.data, T.ctypes.data, rows, grads.ctypes.data,
                                  out.ctypes.data, ctypes.byref(loss)) == 0
    # a parameter vector of another size is refused, not read past
    assert L.upbp_guide_gradients(P.ctypes.data, len(P) - 1, X.ctypes.data, T.ctypes.data, rows, grads.ctypes.data,
                                  out.ctypes.data, ctypes.byref(loss)) == -1
    O, loss64, g64 = G.forward_backward(P, X, T, fp16_like_gpu=True)
    # outputs: FP32 accumulation of FP16 products, same roundings of the
    # hidden activations
    assert np.abs(out - O).max() <= 2e-3 * (np.abs(O).max() + 1e-3)
    assert abs(loss.value - loss64) <= 1e-3 * abs(loss64)
    w_off, b_off, n = G.param_layout()
    bounds = [(w_off[l], w_off[l] + i * o) for l, (i, o) in enumerate(G.LAYERS)] + \
             [(b_off[l], b_off[l] + o) for l, (_, o) in enumerate(G.LAYERS)]
    for a, b in bounds:
        gg, gr = grads[a:b].astype(np.float64), g64[a:b]
        err = np.linalg.norm(gg - gr) / max(np.linalg.norm(gr), 1e-12)
        assert err <= 1e-2, (a, b, err)
    # and against the network without FP16 roundings, the same to ~FP16 precision
    _, _, g_exact = G.forward_backward(P, X, T, fp16_like_gpu=False)
    assert np.linalg.norm(grads - g_exact) / np.linalg.norm(g_exact) <= 5e-2


def _render(args, iterations, scene_dir, offset=0):
    """Mean of iterations 0..iterations-1 (the radius schedule's), with the
    random streams of iteration index + offset (-ioff)."""
    from gpuupbp_b200 import upbp
    path = scenes.write_workload("box_medium", scene_dir)
    r = upbp.Renderer(["-s", "-1", path] + args + ["-ioff", str(offset)])
    acc = np.zeros((r.height, r.width, 3))
    for it in range(iterations):
        r.run_iteration(it)
        acc += r.iteration_image()
    info = np.zeros(9, np.float32)
    r._L.upbp_guide_info(r._ctx, info.ctypes.data, 9)
    st = r.stats()
    r.close()
    return acc / iterations, info, st


BOX = ["-a", "upbp_all", "-l", "8", "-r", "64x64", "-r_initial", "-0.02", "-r_alpha", "0.75"]


def test_training_lowers_the_loss(scene_dir):
    from gpuupbp_b200 import upbp
    path = scenes.write_workload("box_medium", scene_dir)
    r = upbp.Renderer(["-s", "-1", path] + BOX + ["-guide", "4"])
    losses = []
    for it in range(4):
        r.run_iteration(it)
        info = np.zeros(9, np.float32)
        r._L.upbp_guide_info(r._ctx, info.ctypes.data, 9)
        losses.append(float(info[2]))
    assert info[1] == 4 * 4 and info[3] > 1000 and info[8] >= 0
    r.close()
    assert losses[-1] < losses[0] - 0.05, losses


def test_guided_render_is_unbiased(scene_dir):
    n = 128
    plain_a, _, _ = _render(BOX, n, scene_dir)
    plain_b, _, _ = _render(BOX, n, scene_dir, offset=100000)
    guided, info, st = _render(BOX + ["-guide", "8"], n, scene_dir, offset=200000)
    assert st["status"] == 0 and np.isfinite(guided).all()
    assert info[8] >= 0  # a table was in use

    def relmse(x, ref):
        return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))

    noise = relmse(plain_a, plain_b)
    # the guided image is as close to a plain one as two plain ones are
    assert relmse(guided, plain_a) <= 2.5 * noise + 1e-6, (relmse(guided, plain_a), noise)
    # and the image means agree to the noise of the mean
    assert abs(guided.mean() - plain_a.mean()) <= 4 * abs(plain_a.mean() - plain_b.mean()) + 1e-3 * plain_a.mean()
