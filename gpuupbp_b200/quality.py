"""Image error and equal-time comparisons of render methods.

relMSE (relative mean squared error) of an image x against a reference r is
the mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2).  An
equal-time comparison renders a converged reference with the plain method,
then renders each method for the same device time and compares their
relMSE: a method that reaches a k times lower relMSE in the same time is k
times as efficient.
"""
from __future__ import annotations

import numpy as np


def relmse(x: np.ndarray, ref: np.ndarray) -> float:
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


def _timed_render(args: list[str], iterations: int | None, budget_ms: float | None, start: int = 0):
    """Renders with a fresh renderer until `iterations` are done or
    `budget_ms` of device time (CUDA events on the library's stream, around
    every iteration including any training it does) is spent; returns
    (mean image, iterations, device ms)."""
    import torch

    from gpuupbp_b200 import upbp
    r = upbp.Renderer(args)
    stream = torch.cuda.ExternalStream(r.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms, it = 0.0, 0
    while (iterations is None or it < iterations) and (budget_ms is None or ms < budget_ms):
        e0.record(stream)
        r.run_iteration(start + it)
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        it += 1
    img = r.accumulated()
    r.close()
    return img, it, ms


def equal_time(plain_args: list[str], other_args: list[str], reference_iterations: int, other_iterations: int,
               reference_start: int = 100000) -> dict:
    """The plain method's converged reference (reference_iterations, on
    iteration indices from reference_start, so its random streams are
    independent of the compared renders), the other method for
    other_iterations, the plain method for the same device time, and both
    relMSEs."""
    ref, _, ref_ms = _timed_render(plain_args, reference_iterations, None, start=reference_start)
    other, n_other, t_other = _timed_render(other_args, other_iterations, None)
    plain, n_plain, t_plain = _timed_render(plain_args, None, t_other)
    e_other, e_plain = relmse(other, ref), relmse(plain, ref)
    return {"reference_iterations": reference_iterations, "reference_ms": ref_ms,
            "other_iterations": n_other, "other_ms": t_other, "plain_iterations": n_plain, "plain_ms": t_plain,
            "relmse_other": e_other, "relmse_plain": e_plain,
            "relmse_ratio_plain_over_other": e_plain / e_other if e_other > 0 else None}
