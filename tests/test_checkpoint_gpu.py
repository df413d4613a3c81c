"""Checkpoint / resume (upbp_save_checkpoint, upbp_load_checkpoint) and the
-assert event report.

* A render checkpointed after 3 iterations, resumed in a new context and
  continued to 6 equals the uninterrupted 6-iteration render: the random
  numbers and radii depend only on the iteration index, so the only
  difference is the order of float additions (the image parity bar).
* With the learned proposal the resumed context continues the training from
  the saved network, Adam state and records: the Adam steps and records
  match the uninterrupted run's and the image agrees in the mean.
* A checkpoint loads only into a context of the same scene and
  configuration.
* -assert: the failed-path events of an iteration are counted and reported
  as the reference's exception program names them."""
import numpy as np
import pytest

from cases import MEAN_BAR, PIXEL_BAR
from gpuupbp_b200 import scenes

pytestmark = pytest.mark.gpu

BOX = ["-a", "upbp_all", "-l", "8", "-r", "48x48", "-r_initial", "-0.02", "-r_alpha", "0.75"]


def _render(args, its, start=0, load=None, save=None):
    from gpuupbp_b200 import upbp
    r = upbp.Renderer(args)
    if load:
        assert r.load_checkpoint(load) == start
    for it in range(start, its):
        r.run_iteration(it)
    if save:
        r.save_checkpoint(save)
    img = r.accumulated()
    info = np.zeros(9, np.float32)
    r._L.upbp_guide_info(r._ctx, info.ctypes.data, 9)
    r.close()
    return img, info


def _agree(a, b):
    rel = np.abs(a - b) / (np.abs(b) + 1e-3)
    frac = float(np.mean(np.all(rel < 1e-3, axis=-1)))
    return frac, abs(float(a.mean()) - float(b.mean())) / (abs(float(b.mean())) + 1e-9)


def test_resumed_render_equals_uninterrupted(scene_dir, tmp_path):
    args = ["-s", "-1", scenes.write_workload("box_medium", scene_dir, tiny=True)] + BOX
    straight, _ = _render(args, 6)
    ck = str(tmp_path / "box.ckpt")
    _render(args, 3, save=ck)
    resumed, _ = _render(args, 6, start=3, load=ck)
    frac, mean_rel = _agree(resumed, straight)
    assert frac >= PIXEL_BAR and mean_rel <= MEAN_BAR, (frac, mean_rel)


def test_resumed_guided_render_continues_training(scene_dir, tmp_path):
    args = ["-s", "-1", scenes.write_workload("box_medium", scene_dir, tiny=True)] + BOX + ["-guide", "4"]
    straight, info_s = _render(args, 6)
    ck = str(tmp_path / "guided.ckpt")
    _, info_3 = _render(args, 3, save=ck)
    resumed, info_r = _render(args, 6, start=3, load=ck)
    assert info_3[1] == 3 * 4 and info_r[1] == info_s[1] == 4 * 4  # Adam steps
    assert info_r[3] == info_s[3]                                  # training records
    assert info_r[8] >= 0 and info_s[8] >= 0                       # a table in use
    _, mean_rel = _agree(resumed, straight)
    assert mean_rel <= 2e-2, mean_rel


def test_checkpoint_refuses_another_configuration(scene_dir, tmp_path):
    from gpuupbp_b200 import upbp
    path = scenes.write_workload("box_medium", scene_dir, tiny=True)
    ck = str(tmp_path / "a.ckpt")
    _render(["-s", "-1", path] + BOX, 1, save=ck)
    other = ["-s", "-1", path] + [a if a != "8" else "6" for a in BOX]  # path length 6
    r = upbp.Renderer(other)
    with pytest.raises(upbp.UpbpError, match="fingerprint"):
        r.load_checkpoint(ck)
    r.close()


def test_assert_reports_failed_path_events(scene_dir, capfd):
    from gpuupbp_b200 import upbp
    path = scenes.write_workload("media_field", scene_dir)
    args = ["-s", "-1", path, "-a", "upbp_all", "-l", "12", "-r", "64x36", "-pcpi", "200000", "-assert"]
    r = upbp.Renderer(args)
    status = r.run_iteration(0)
    r.close()
    err = capfd.readouterr().err
    # rays through the full media field cross more than 8 imaginary
    # boundaries of its 20 icospheres (status bit 3)
    assert status & 8
    assert "[ 5][            USER]: intersection_stack too small (" in err, err[-2000:]
