"""Batched rendering (upbp_run_batch): jobs of uneven resolution, path
length, triangle count and media, rendered concurrently by worker threads on
their own streams and launch-parameter slots, each agree with the same job
rendered alone by the plain single-scene renderer: equal light-vertex and
beam counts and status, pixels within the parity bar (the order of float
additions is all that differs)."""
import numpy as np
import pytest

from cases import MEAN_BAR, PIXEL_BAR

pytestmark = pytest.mark.gpu


def test_batched_jobs_equal_single_scene_renders(scene_dir):
    from gpuupbp_b200 import batch, upbp
    jobs = [batch.job_args(j, scene_dir, res_cap=128) for j in range(8)]
    assert len({a[a.index("-r") + 1] for a in jobs}) > 1   # uneven resolutions
    assert len({a[a.index("-l") + 1] for a in jobs}) > 1   # uneven path lengths
    b = batch.Batch(jobs)
    b.set_grid_limit(148)
    status = b.run_iteration(0, workers=8)
    got = []
    for r in b.renderers:
        st = r.stats()
        got.append((r.iteration_image(), st))
    b.close()
    for j, args in enumerate(jobs):
        r = upbp.Renderer(args)
        s_alone = r.run_iteration(0)
        img = r.iteration_image()
        st = r.stats()
        r.close()
        bimg, bst = got[j]
        for k in ("light_vertices", "surface_vertices", "medium_vertices", "light_beams"):
            assert bst[k] == st[k], (j, k)
        assert bst["status"] == st["status"] == s_alone
        rel = np.abs(bimg - img) / (np.abs(img) + 1e-3)
        assert float(np.mean(np.all(rel < 1e-3, axis=-1))) >= PIXEL_BAR, j
        assert abs(bimg.mean() - img.mean()) <= MEAN_BAR * abs(img.mean()) + 1e-9, j
    assert status >= 0


def test_autotuner_picks_a_measured_configuration(scene_dir):
    from gpuupbp_b200 import batch
    jobs = [batch.job_args(j, scene_dir, res_cap=64, tiny=True) for j in range(6)]
    b = batch.Batch(jobs)
    choice = batch.autotune(b, 0, workers=(1, 4), limits=(0, 64))
    assert (choice["workers"], choice["grid_limit"]) in {(1, 0), (4, 0), (1, 64), (4, 64)}
    assert choice["next_iteration"] == 5 and len(choice["timings_s"]) == 4
    b.run_iteration(choice["next_iteration"])
    b.close()
