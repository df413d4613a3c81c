"""Batched rendering of many independent scene/view jobs (config 3 of the
benchmark spec): 64 jobs drawn from seeds, each with its own resolution
(64^2 .. 512^2), path length (4 .. 16), scene (1k .. 200k triangles of
displaced icospheres bounding 1-3 media in a box) and renderer context.

`Batch.run_iteration` renders one iteration of every job through
upbp_run_batch: host worker threads drive the jobs' contexts concurrently,
each on its own CUDA stream and launch-parameter slot.  `autotune` picks the
number of workers and the per-job cap on launch blocks (upbp_set_grid_limit)
by timing batch iterations.
"""
from __future__ import annotations

import ctypes
import time

from gpuupbp_b200 import scenes, upbp

JOB_TECH = "upbp_all"   # BPT + SURF + PP3D + PB2D + BB1D, the plain method of config 1
JOB_RADIUS = ["-r_initial", "-0.02", "-r_alpha", "0.75"]


def job_args(seed: int, scene_dir: str, tiny: bool = False, res_cap: int | None = None) -> list[str]:
    """Command line of batched job `seed` (its scene written into scene_dir)."""
    cfg = scenes.batch_job_config(seed)
    w, h = cfg["res"]
    if res_cap:
        w, h = min(w, res_cap), min(h, res_cap)
    path = scenes.write_workload("batch_job", scene_dir, seed=seed, tiny=tiny)
    return ["-s", "-1", path, "-a", JOB_TECH, "-l", str(cfg["length"]), "-r", f"{w}x{h}"] + JOB_RADIUS


class Batch:
    def __init__(self, jobs: list[list[str]], library: str = upbp.LIB_PATH):
        self.renderers = [upbp.Renderer(a, library=library) for a in jobs]
        self._L = self.renderers[0]._L
        self._ctxs = (ctypes.c_void_p * len(jobs))(*[r._ctx.value for r in self.renderers])
        self.workers = 16
        self.grid_limit = 0

    def __len__(self):
        return len(self.renderers)

    def paths_per_iteration(self) -> int:
        return sum(r.width * r.height + int(r.config.path_count_per_iter) for r in self.renderers)

    def set_grid_limit(self, blocks: int):
        self.grid_limit = blocks
        for r in self.renderers:
            self._L.upbp_set_grid_limit(r._ctx, blocks)

    def run_iteration(self, iteration: int, workers: int | None = None) -> int:
        rc = self._L.upbp_run_batch(self._ctxs, len(self._ctxs), iteration, workers or self.workers)
        if rc < 0:
            upbp._check(rc, f"batch iteration {iteration}", self._L)
        for r in self.renderers:
            r.iterations += 1
        return rc

    def close(self):
        for r in self.renderers:
            r.close()


def autotune(batch: Batch, first_iteration: int, workers=(4, 8, 16, 32), limits=(0, 148 * 2)) -> dict:
    """Times one batch iteration for every (workers, grid limit) pair, after
    one untimed iteration, and keeps the fastest; the jobs one after another
    (one worker, no cap) is always among the candidates, so the choice is
    never slower than that.
    The iterations rendered while tuning are real ones (first_iteration
    onward), so the caller continues after them.  Returns the choice, its
    timings and the next iteration index."""
    it = first_iteration
    # one untimed iteration first: a job's first iteration grows its buffers
    batch.run_iteration(it, max(workers))
    it += 1
    timings = {}
    pairs = [(1, 0)] + [(w, lim) for lim in limits for w in workers if (w, lim) != (1, 0)]
    for w, lim in pairs:
        batch.set_grid_limit(lim)
        t0 = time.perf_counter()
        batch.run_iteration(it, w)
        timings[(w, lim)] = time.perf_counter() - t0
        it += 1
    best = min(timings, key=timings.get)
    batch.workers, _ = best
    batch.set_grid_limit(best[1])
    return {"workers": best[0], "grid_limit": best[1], "next_iteration": it,
            "timings_s": {f"{w}x{lim}": t for (w, lim), t in timings.items()}}
