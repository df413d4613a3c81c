"""The FP64 full-path MIS oracle on its own (no GPU): on a hand-made path
through an area light, a diffuse wall, two vertices in a Henyey-Greenstein
medium and the camera, the balance-heuristic weights of every technique that
can sample the path -- BPT splits s = 0..k and the five photon density
estimators at each inner vertex -- sum to one, and the reference's form of
the weights (its three departures) does not."""
import math

import numpy as np

import mis_fp64 as M

L_PATHS = 1000.0


def _scene(exact=1):
    lights = [{"type": 0, "p0": [-0.1, 1.0, -0.1], "p1": [0.1, 1.0, -0.1], "p2": [0.1, 1.0, 0.1]}]
    materials = [{"diffuse": [0.5, 0.6, 0.7], "phong": [0.0, 0.0, 0.0], "mirror": [0.0, 0.0, 0.0], "ior": -1.0}]
    media = [{"absorption": [0.1, 0.1, 0.1], "scattering": [0.8, 0.8, 0.8], "mean_cosine": 0.4,
              "continuation_prob": 0.9},
             {"absorption": [0.0, 0.0, 0.0], "scattering": [0.0, 0.0, 0.0], "mean_cosine": 0.0,
              "continuation_prob": 1.0}]
    h = np.zeros(64)
    h[0:8] = [9, L_PATHS, 100, 0, 1 << 20, 15, 15, 10]
    h[8:11] = [0.0, 0.0, 3.0]
    h[11:14] = [0.0, 0.0, -1.0]
    h[14] = 20.0
    r = 0.02
    h[17:22] = [math.pi * r * r * L_PATHS, 4 / 3 * math.pi * r ** 3 * L_PATHS, math.pi * r * r * L_PATHS,
                math.pi * r * r * L_PATHS, 0.5 * r * 300]
    h[22:29] = [1.0, L_PATHS, M.SHORT_BEAM, M.LONG_BEAM, 1, exact, 1]
    return M.Scene({"lights": lights, "materials": materials, "media": media}, h)


def _path(sc, merge=None):
    v = [M.PathVertex("light", [0.02, 1.0, 0.01], normal=[0, -1, 0], ident=0),
         M.PathVertex("surface", [0.3, 0.0, -0.5], normal=[0, 0, 1], ident=0),
         M.PathVertex("medium", [0.1, 0.2, 0.1], ident=0),
         M.PathVertex("medium", [-0.1, 0.1, 0.6], ident=0),
         M.PathVertex("camera", [0.0, 0.0, 3.0])]
    # media: the medium fills the region between distance 0.3 of x_1's ray
    # and the camera side of x_3
    edges = []
    for i in range(4):
        d = float(np.linalg.norm(v[i + 1].pl - v[i].pl))
        if i == 0:
            edges.append([(0.0, d, 1)])
        elif i == 1:
            edges.append([(0.0, 0.3, 1), (0.3, d, 0)])
        elif i == 2:
            edges.append([(0.0, d, 0)])
        else:
            edges.append([(0.0, 0.4, 0), (0.4, d, 1)])
    return M.FullPath(sc, v, edges, merge)


def _all_weights(sc, reference):
    fp = _path(sc)
    k = fp.k
    ws = []
    for s in range(k + 1):
        tech = M.EMITTER_HIT if s == 0 else M.NEE if s == 1 else M.LIGHT_TRACE if s == k else M.BPT
        ws.append(fp.weight(tech, s, reference=reference))
    ws.append(fp.weight(M.SURF, 1, reference=reference))
    for i in (2, 3):
        for tech in (M.PP3D, M.PB2D, M.BP2D, M.BB1D):
            off = 0.3 if i == 2 else 0.0  # the beam into x_2 starts where its ray enters the medium
            ws.append(fp.weight(tech, i, reference=reference, beam_offset=off))
    return ws


def test_balance_heuristic_weights_sum_to_one():
    ws = _all_weights(_scene(1), reference=False)
    assert all(w > 0 for w in ws)
    assert abs(sum(ws) - 1.0) < 1e-12


def test_reference_form_departs_from_a_partition_of_unity():
    ws = _all_weights(_scene(0), reference=True)
    assert abs(sum(ws) - 1.0) > 1e-3


def test_free_flight_pdfs():
    sc = _scene()
    # survival through 0.5 of the medium, density at a medium vertex at the far end
    pr, pl = M._edge_pdfs(sc, [(0.0, 0.5, 0)], 0.5, a_medium=False, b_medium=True)
    assert math.isclose(pr, 0.9 * math.exp(-0.9 * 0.5), rel_tol=1e-12)
    assert math.isclose(pl, math.exp(-0.9 * 0.5), rel_tol=1e-12)
    # vacuum segments sample nothing
    assert M._edge_pdfs(sc, [(0.0, 2.0, 1)], 2.0, True, True) == (1.0, 1.0)
