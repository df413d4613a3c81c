"""Image error and equal-time comparisons of render methods.

relMSE (relative mean squared error) of an image x against a reference r is
the mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2).  An
equal-time comparison renders a converged reference with the plain method,
then renders each method for the same device time and compares their
relMSE: a method that reaches a k times lower relMSE in the same time is k
times as efficient.

The reference runs the same radius schedule from iteration 0 (the radii
shrink with the iteration index, so later indices are noisier per
iteration) on independent random streams: -ioff shifts only the random
numbers' iteration index.
"""
from __future__ import annotations

import numpy as np

REFERENCE_IOFF = ["-ioff", "1000000"]


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


def equal_time(plain_args: list[str], other_args: list[str], reference_iterations: int,
               other_iterations: int) -> dict:
    """The plain method's converged reference (reference_iterations on
    random streams independent of the compared renders), the other method
    for other_iterations, the plain method for the same device time, and
    both relMSEs."""
    ref, _, ref_ms = _timed_render(plain_args + REFERENCE_IOFF, reference_iterations, None)
    other, n_other, t_other = _timed_render(other_args, other_iterations, None)
    plain, n_plain, t_plain = _timed_render(plain_args, None, t_other)
    e_other, e_plain = relmse(other, ref), relmse(plain, ref)
    return {"reference_iterations": reference_iterations, "reference_ms": ref_ms,
            "other_iterations": n_other, "other_ms": t_other, "plain_iterations": n_plain, "plain_ms": t_plain,
            "relmse_other": e_other, "relmse_plain": e_plain,
            "relmse_ratio_plain_over_other": e_plain / e_other if e_other > 0 else None}


def _batch_images(b) -> list:
    return [r.accumulated() for r in b.renderers]


def batch_equal_time(jobs: list, method_extra: list, reference_iterations: int, method_iterations: int) -> dict:
    """Equal-time comparison on many jobs (config 3 of the benchmark spec).

    * reference: every job's converged plain render, reference_iterations
      batch iterations on independent random streams;
    * method: the jobs with `method_extra` appended to their command lines
      (e.g. the learned proposal), rendered together by upbp_run_batch with
      the autotuner's choice, method_iterations iterations; its wall time T
      (the autotuning iterations are part of the method's work and time);
    * plain: the plain single-scene renderer taking the jobs one after
      another (one worker, no launch cap), whole iterations of all jobs
      until it has used the time T.
    Returns per-job relMSEs, the mean relMSE of both, and their ratio."""
    import time

    import torch

    from gpuupbp_b200 import batch as B

    ref = B.Batch([j + REFERENCE_IOFF for j in jobs])
    tune = B.autotune(ref, 0)
    it = tune["next_iteration"]
    while ref.renderers[0].iterations < reference_iterations:
        ref.run_iteration(it)
        it += 1
    refs = _batch_images(ref)
    ref.close()

    m = B.Batch([j + method_extra for j in jobs])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tune_m = B.autotune(m, 0)
    it = tune_m["next_iteration"]
    while m.renderers[0].iterations < method_iterations:
        m.run_iteration(it)
        it += 1
    torch.cuda.synchronize()
    t_method = time.perf_counter() - t0
    imgs_m = _batch_images(m)
    n_method = m.renderers[0].iterations
    m.close()

    p = B.Batch(jobs)
    p.set_grid_limit(0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    it, t_plain = 0, 0.0
    while t_plain < t_method:
        p.run_iteration(it, workers=1)
        it += 1
        torch.cuda.synchronize()
        t_plain = time.perf_counter() - t0
    imgs_p = _batch_images(p)
    n_plain = it
    p.close()

    e_m = [relmse(x, r) for x, r in zip(imgs_m, refs)]
    e_p = [relmse(x, r) for x, r in zip(imgs_p, refs)]
    mean_m, mean_p = float(np.mean(e_m)), float(np.mean(e_p))
    return {"jobs": len(jobs), "reference_iterations": reference_iterations,
            "method_iterations": n_method, "method_s": t_method, "method_autotune": tune_m,
            "plain_iterations": n_plain, "plain_s": t_plain,
            "relmse_method_mean": mean_m, "relmse_plain_mean": mean_p,
            "relmse_ratio_plain_over_method": mean_p / mean_m if mean_m > 0 else None,
            "per_job_ratio_median": float(np.median(np.array(e_p) / np.maximum(np.array(e_m), 1e-30))),
            "relmse_method": e_m, "relmse_plain": e_p}
