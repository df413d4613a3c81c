"""The failure path of the bounded per-ray arrays against the reference's
own code: a scene built to overflow them, rendered by the reference's render
loop compiled for the host (oracle/_ref) and by the GPU library on the same
files, command line and random stream.

* media_row: 12 fog spheres along the view axis; a camera ray along the row
  meets more imaginary boundaries than the reference keeps between two real
  hits (MAX_IMAGINARY_INTERSECTIONS 8, ERR_INTERSECTION_STACK).

The reference gathers every imaginary crossing up to a ray's next real hit
before it samples free flight, so that limit is met first: the
medium-segment array (10) and the boundary stack (20) cannot overflow while
it holds (a ray splits into at most 9 segments, and a path that would push
20 boundaries crosses more than 8 of them on its way to a real surface --
24 nested shells of a dense forward-scattering medium raised only this code
in the reference's build as well).

The iteration's status bits equal the codes the reference raised, the
overflow happened, the light-vertex, surface, medium and beam counts agree
within COUNT_TOL, and the image agrees within the parity bar."""
import numpy as np
import pytest

from gpuupbp_b200 import scenes

pytestmark = pytest.mark.gpu

COUNT_TOL = 1e-3
ALL6 = "upbp_bpt+surf+pp3d+pb2d+bb1d+bp2d"
CASES = {
    # name: (workload, args, the status bit the scene must raise)
    "media_row": ("media_row", ["-a", ALL6, "-l", "8", "-r", "48x48"], 1 << 3),
}


def _status_of_codes(delta):
    return sum(1 << (code - 1) for code in range(1, 5) if delta[code] > 0)


@pytest.mark.parametrize("case", list(CASES))
def test_overflow_matches_reference(case, scene_dir):
    import ref_cpu
    from gpuupbp_b200 import upbp
    assert ref_cpu.available(), "oracle/_ref/libupbp_ref_cpu.so is not built (make -C oracle)"
    workload, extra, bit = CASES[case]
    args = ["-s", "-1", scenes.write_workload(workload, scene_dir)] + extra
    ref = ref_cpu.RefRenderer(args, threads=0)
    before = ref_cpu.RefRenderer.exception_counts()
    ref_img = ref.run_iteration(0)
    delta = [a - b for a, b in zip(ref_cpu.RefRenderer.exception_counts(), before)]
    rst = ref.stats()
    ref.close()
    r = upbp.Renderer(args)
    status = r.run_iteration(0)
    img = r.iteration_image()
    st = r.stats()
    r.close()
    assert status == _status_of_codes(delta), (case, status, delta)
    assert status & bit, (case, status)
    for k, kr in (("light_vertices", "vertices"), ("surface_vertices", "surface"), ("medium_vertices", "medium"),
                  ("light_beams", "beams")):
        assert abs(st[k] - rst[kr]) <= COUNT_TOL * max(1, rst[kr]), (case, k, st[k], rst[kr])
    rel = np.abs(img - ref_img) / (np.abs(ref_img) + 1e-3)
    frac = float(np.mean(np.all(rel < 1e-3, axis=-1)))
    mean_rel = abs(float(img.mean()) - float(ref_img.mean())) / (abs(float(ref_img.mean())) + 1e-9)
    assert frac >= 0.99 and mean_rel <= 1e-4, (case, frac, mean_rel)
