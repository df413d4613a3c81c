"""FP64 full-path MIS weights of UPBP (test infrastructure, the checker of the
renderer's recursive FP32 weights; nothing in the product imports it).

The renderer computes each contribution's MIS weight with the constant-time
recursion of the reference (kernel/functs_shared.cuh:37-154 sample_scattering,
Eq 4.47-4.49; path_weight.cuh:35-51 get_pde_factor, Eq 4.23; the weights of
functs_camera.cuh:107-527, functs_light.cuh:251-388 and pde/functs_pp.cuh,
functs_pb2d.cuh, functs_bb1d.cuh, functs_bp2d.cuh).  This module evaluates the
same balance heuristic the long way, SmallUPBP style: it rebuilds the full
path x_0 (on the light) .. x_k (the camera) of a contribution from the
recorded subpath vertices, computes in float64 the pdf of every vertex in both
directions from the geometry, the materials and the media, forms the pdf of
every technique that can sample that path -- the BPT splits s = 0..k (s = 0
an emitter hit, s = 1 next-event estimation or a connection to the light
vertex, s = k light tracing), and the five photon density estimators at each
inner vertex -- and returns

    w = p_technique / sum over all techniques of p_t.

Conventions (those of the reference's recursion, written out):

* p_fwd[i]: pdf of sampling x_i from x_{i-1} in area (surface) or volume
  (medium) measure: the directional pdf at x_{i-1} (scattering function, or
  cos/pi emission of an area light at x_0) times the continuation probability
  at x_{i-1}, times |cos| at x_i (1 in a medium) / distance^2, times the
  free-flight pdf of the light-side trace along the edge (pr): a survival
  exp(-sigma d) per medium segment with the minimum positive attenuation
  coefficient, sigma exp(-sigma d) for the segment that ends at a medium
  vertex.  p_fwd[0] is the light pick probability over the light's area.
* p_rev[i]: the same for sampling x_i from x_{i+1} (camera direction; pl);
  p_rev[k-1] uses the camera's directional pdf (image-plane distance^2 / cos^3)
  and p_rev[k] = 1.
* BPT split s (light vertices x_0..x_{s-1}, camera vertices x_s..x_k):
  p = n_s * prod_{i<s} p_fwd[i] * prod_{i>=s} p_rev[i], with n_s = 1 (BPT
  subpath count) for s < k and the light-path count for light tracing;
  available when x_{s-1} and x_s are both non-specular (s = 0: an area light
  reached by the camera path; s = k: k >= 2).
* Merging at inner vertex i: p = prod_{j<=i} p_fwd[j] * prod_{j>=i} p_rev[j]
  * F_i, with F_i the sum of the estimators' factors at that vertex:
  SURF pi r^2 L at a non-specular surface vertex; at a medium vertex PP3D
  4/3 pi r^3 L, PB2D pi r^2 L R_i, BP2D pi r^2 L Fo_i, BB1D r/2 n_bb1d
  sin(theta_i) Fo_i R_i, where Fo_i = 1/pr_i (long photon beams) or
  1/sigma (short), R_i = 1/pl_i (long query beams) or 1/sigma (short), and
  theta_i the scattering angle at x_i.
* A merged vertex has two positions: the light side's (photon, or the point
  on the photon beam) for every pdf toward the light, the camera side's
  (camera vertex, or the point on the query ray) for every pdf toward the
  camera; its directional pdfs use the light side's incoming direction and the
  camera side's outgoing one, with the camera side's scattering function.

Supported scattering: diffuse surfaces and Henyey-Greenstein media, area
lights and the pinhole camera (the scenes of the MIS tests); contributions
through other materials or lights are reported as unsupported.
"""
from __future__ import annotations

import math

import numpy as np

VTX_VALID, VTX_MEDIUM, VTX_SPECULAR, VTX_DELTA, VTX_LIGHT, VTX_CAMERA, VTX_MISS = 1, 2, 4, 8, 16, 32, 64
TECH_NAMES = ["emitter_hit", "nee", "bpt", "light_trace", "surf", "pp3d", "pb2d", "bb1d", "bp2d"]
EMITTER_HIT, NEE, BPT, LIGHT_TRACE, SURF, PP3D, PB2D, BB1D, BP2D = range(9)
SHORT_BEAM, LONG_BEAM = 1, 2
INV_PI = 1.0 / math.pi


def _bits(f) -> int:
    return int(np.float32(f).view(np.uint32))


def _vec(a) -> np.ndarray:
    return np.asarray(a, np.float64)


def _norm(v):
    n = math.sqrt(float(np.dot(v, v)))
    return v / n, n


class Scene:
    """What the weights need of the scene: lights, media and materials as the
    library's scene loader gave them, and the recorded header (camera,
    MIS factors, counts)."""

    def __init__(self, scene: dict, header: np.ndarray):
        h = [float(x) for x in header]
        self.max_verts, self.light_paths, self.camera_paths = int(h[0]), int(h[1]), int(h[2])
        self.events_total, self.event_capacity = int(h[3]), int(h[4])
        self.vtx_words, self.ev_words, self.segs = int(h[5]), int(h[6]), int(h[7])
        self.cam_origin, self.cam_dir = _vec(h[8:11]), _vec(h[11:14])
        self.image_plane_dist = h[14]
        self.mis_surf, self.mis_pp3d, self.mis_pb2d, self.mis_bp2d, self.mis_bb1d = h[17:22]
        self.n_bpt, self.L = h[22], h[23]
        self.photon_beam, self.query_beam = int(h[24]), int(h[25])
        self.light_count = int(h[26])
        self.mis_exact = int(h[27])
        self.lt_from_surf = int(h[28])
        self.lights = scene["lights"]
        self.materials = scene["materials"]
        self.media = []
        for m in scene["media"]:
            att = np.abs(_vec(m["absorption"])) + np.abs(_vec(m["scattering"]))
            pos = [a for a in att if a > 0]
            sig = min(pos) if pos else 0.0
            self.media.append({"sigma": sig, "scatter": bool(np.any(np.abs(_vec(m["scattering"])) > 0)),
                               "g": float(m["mean_cosine"]), "cont": float(m["continuation_prob"])})

    # ------------------------------------------------------------ media
    def seg_pdf(self, med: int, length: float, ends_at_vertex: bool) -> float:
        """Free-flight pdf of one medium segment: the survival probability, or
        the density of stopping at its far end when a medium vertex lies
        there (homogeneous media sample with the minimum attenuation)."""
        m = self.media[med] if 0 <= med < len(self.media) else None
        if m is None or m["sigma"] == 0.0 or not m["scatter"]:
            return 1.0
        s = math.exp(-m["sigma"] * length)
        return m["sigma"] * s if ends_at_vertex else s

    # ------------------------------------------------------------ scattering
    def surface_pdf(self, mat: int, n: np.ndarray, w_in: np.ndarray, w_out: np.ndarray) -> float:
        """Directional pdf of a diffuse surface (reference bsdf.cuh:232-250,
        cosine-weighted hemisphere on the side of the incoming direction);
        w_in points away from the vertex toward where the path came from."""
        m = self.materials[mat]
        if any(abs(x) > 0 for x in list(m["phong"]) + list(m["mirror"])) or m["ior"] > 0:
            raise NotImplementedError("only diffuse materials")
        ci, co = float(np.dot(n, w_in)), float(np.dot(n, w_out))
        if ci * co <= 0.0:
            return 0.0
        return abs(co) * INV_PI

    def surface_cont(self, mat: int) -> float:
        """Continuation probability of a surface (reference
        bsdf.cuh:143-177): the largest reflectance component plus the
        transmitted Fresnel part; without a dielectric the Fresnel reflectance
        is 1, so it is the largest diffuse (+ phong + mirror) component."""
        m = self.materials[mat]
        r = [a + b + c for a, b, c in zip(m["diffuse"], m["phong"], m["mirror"])]
        return min(1.0, max(0.0, max(r)))

    def hg_pdf(self, med: int, travel_in: np.ndarray, w_out: np.ndarray) -> float:
        g = self.media[med]["g"]
        if abs(g) < 1e-3:
            return 0.25 * INV_PI
        c = float(np.dot(travel_in, w_out))
        d = 1.0 + g * g - 2.0 * g * c
        return 0.25 * INV_PI * (1.0 - g * g) / (d * math.sqrt(d)) if d > 0 else 0.0


class PathVertex:
    def __init__(self, kind: str, pos_l, pos_c=None, normal=None, ident: int = -1, specular: bool = False,
                 normal_l=None):
        self.kind = kind                 # light | surface | medium | camera
        self.pl = _vec(pos_l)            # position seen from the light side
        self.pc = _vec(pos_c if pos_c is not None else pos_l)  # ... from the camera side
        self.normal = None if normal is None else _norm(_vec(normal))[0]
        # the light side's normal at a merged surface vertex (the photon's)
        self.normal_l = self.normal if normal_l is None else _norm(_vec(normal_l))[0]
        self.id = ident                  # light, material or medium index
        self.specular = specular


def _edge_pdfs(scene: Scene, segs, length: float, a_medium: bool, b_medium: bool) -> tuple[float, float]:
    """(pr, pl) of an edge from a to b of the given length whose media
    segments (dmin, dmax, medium) are measured from a: pr samples b from a,
    pl samples a from b.  The recorded segment ends are float32 distances of
    the GPU's trace and the length is recomputed in float64, so the segments
    touching the end points are recognised within 1e-5 of the length."""
    pr = pl = 1.0
    tol = 1e-5 * (1.0 + length)
    segs = sorted((d0, min(d1, length), m) for d0, d1, m in segs if min(d1, length) > d0)
    for j, (d0, d1, med) in enumerate(segs):
        ln = d1 - d0
        at_b = j == len(segs) - 1 and d1 >= length - tol
        at_a = j == 0 and d0 <= tol
        pr *= scene.seg_pdf(med, ln, b_medium and at_b)
        pl *= scene.seg_pdf(med, ln, a_medium and at_a)
    return pr, pl


class FullPath:
    """A full path x_0..x_k with the media segments of each edge
    (edges[i] joins x_i and x_{i+1}, segments measured from x_i), the
    index of the merged vertex (None for BPT techniques), and per edge the
    traced ray's direction (from x_i toward x_{i+1}) and length where a
    subpath traced it (None for connections: those are taken from the
    positions, as the renderer takes them).  Traced rays keep their own
    direction and length because a float32 position is too coarse for a
    medium vertex sampled a few micrometres from the previous one."""

    def __init__(self, scene: Scene, verts: list, edges: list, merge: int | None, geo: list | None = None):
        self.s, self.v, self.e, self.merge = scene, verts, edges, merge
        self.k = len(verts) - 1
        self.geo = geo if geo is not None else [None] * self.k
        assert len(edges) == self.k and len(self.geo) == self.k

    def ends(self, i: int):
        """The two points edge i joins: x_i's camera-side point when x_i is
        the merged vertex (the camera subpath left from there), else its
        light-side one; x_{i+1}'s light-side point when it is the merged
        vertex, else its camera-side one (equal for unmerged vertices)."""
        a = self.v[i].pc if i == self.merge else self.v[i].pl
        b = self.v[i + 1].pl if i + 1 == self.merge else self.v[i + 1].pc
        return a, b

    def _toward(self, i: int, j: int):
        """Unit direction from x_i to its neighbour x_j along their edge."""
        e = min(i, j)
        if self.geo[e] is not None:
            d = self.geo[e][0]
            return d if j > i else -d
        a, b = self.ends(e)
        return _norm(b - a)[0] if j > i else _norm(a - b)[0]

    def _length(self, e: int) -> float:
        if self.geo[e] is not None:
            return self.geo[e][1]
        a, b = self.ends(e)
        return _norm(b - a)[1]

    def _dir_pdf(self, i: int, toward: int) -> float:
        """Directional pdf at x_i of the direction toward its neighbour
        x_toward, given the path arrived from the other neighbour, times the
        continuation probability at x_i."""
        sc, v = self.s, self.v[i]
        w_out = self._toward(i, toward)
        if v.kind == "light":
            if sc.lights[v.id]["type"] != 0:
                raise NotImplementedError("only area lights")
            return abs(float(np.dot(v.normal, w_out))) * INV_PI
        if v.kind == "camera":
            c = float(np.dot(sc.cam_dir, w_out))
            ipd = sc.image_plane_dist / c
            return ipd * ipd / c
        w_in = self._toward(i, i - 1 if toward == i + 1 else i + 1)
        if v.kind == "surface":
            return sc.surface_pdf(v.id, v.normal, w_in, w_out) * sc.surface_cont(v.id)
        return sc.hg_pdf(v.id, -w_in, w_out) * sc.media[v.id]["cont"]

    def _cos(self, i: int, other: int) -> float:
        """|cos| at x_i of the edge to its neighbour x_other (1 in a medium)."""
        v = self.v[i]
        if v.kind in ("medium", "camera"):
            return 1.0
        n = v.normal_l if other < i else v.normal
        return abs(float(np.dot(n, self._toward(i, other))))

    def pdfs(self):
        k, sc, v = self.k, self.s, self.v
        pr_e, pl_e, len_e = [], [], []
        for i in range(k):
            d = self._length(i)
            pr, pl = _edge_pdfs(sc, self.e[i], d, v[i].kind == "medium", v[i + 1].kind == "medium")
            pr_e.append(pr)
            pl_e.append(pl)
            len_e.append(d)
        lt = sc.lights[v[0].id]
        area = float(np.linalg.norm(np.cross(_vec(lt["p1"]) - _vec(lt["p0"]), _vec(lt["p2"]) - _vec(lt["p0"])))) * 0.5
        fwd = [0.0] * (k + 1)
        rev = [0.0] * (k + 1)
        fwd[0] = 1.0 / (sc.light_count * area)
        for i in range(1, k):
            fwd[i] = self._dir_pdf(i - 1, i) * self._cos(i, i - 1) / (len_e[i - 1] ** 2) * pr_e[i - 1]
        for i in range(k - 1, -1, -1):
            rev[i] = self._dir_pdf(i + 1, i) * self._cos(i, i + 1) / (len_e[i] ** 2) * pl_e[i]
        rev[k] = 1.0
        return fwd, rev, pr_e, pl_e

    def factor(self, i: int, pr_e, pl_e, which: str | None = None) -> float:
        """F_i (or one estimator's term of it) at inner vertex i."""
        sc, v = self.s, self.v[i]
        if v.kind == "surface":
            if v.specular:
                return 0.0
            return sc.mis_surf if which in (None, "surf") else 0.0
        if v.kind != "medium":
            return 0.0
        sigma = sc.media[v.id]["sigma"]
        fo = 1.0 / pr_e[i - 1] if sc.photon_beam == LONG_BEAM else 1.0 / sigma
        ro = 1.0 / pl_e[i] if sc.query_beam == LONG_BEAM else 1.0 / sigma
        c = float(np.clip(np.dot(-self._toward(i, i - 1), self._toward(i, i + 1)), -1.0, 1.0))
        sin_t = math.sqrt(max(0.0, 1.0 - c * c))
        terms = {"pp3d": sc.mis_pp3d, "pb2d": sc.mis_pb2d * ro, "bp2d": sc.mis_bp2d * fo,
                 "bb1d": sc.mis_bb1d * sin_t * fo * ro}
        return sum(terms.values()) if which is None else terms.get(which, 0.0)

    def weight(self, tech: int, split: int, reference: bool = False, beam_offset: float = 0.0) -> float:
        """Balance-heuristic weight of technique `tech` (BPT split s = `split`,
        or a merge at vertex `split`).

        reference=True gives instead the weight the reference's recursion
        computes, which departs from the balance heuristic in three places:
        * next-event estimation: its ratio for the emitter-hit technique
          leaves out the camera-side free-flight pdf of the light ray
          (functs_camera.cuh:296), i.e. it divides p(s=0) by pl of edge 0;
        * BP2D and BB1D: the light side's area-measure conversion at the
          merged point uses its distance from the photon beam's origin, not
          from the light vertex (functs_bp2d.cuh:137-140,
          functs_bb1d.cuh:189-193), which scales the connection technique
          that ends the light subpath at x_{m-1} by (t / (offset + t))^2
          (t the distance along the beam, offset from the vertex to the
          beam's origin);
        * BB1D beams leaving the light (m = 1) of a finite light skip the
          conversion altogether (functs_bb1d.cuh:191), a factor
          1 / (offset + t)^2 on that technique.
        The three change a path's weights so that they no longer sum to one."""
        k, v, sc = self.k, self.v, self.s
        fwd, rev, pr_e, pl_e = self.pdfs()

        def bpt_pdf(s: int) -> float:
            if s == 0:
                if sc.lights[v[0].id]["type"] != 0:
                    return 0.0
            elif s < k:
                if v[s - 1].specular or v[s].specular:
                    return 0.0
            else:
                if k < 2 or v[k - 1].specular:
                    return 0.0
                if not sc.lt_from_surf and v[k - 1].kind != "medium":
                    return 0.0
            n = sc.n_bpt * (sc.L if s == k else 1.0)
            return n * math.prod(fwd[:s]) * math.prod(rev[s:])

        def pde_pdf(i: int, which: str | None = None) -> float:
            return math.prod(fwd[:i + 1]) * math.prod(rev[i:]) * self.factor(i, pr_e, pl_e, which)

        terms = [bpt_pdf(s) for s in range(k + 1)]
        if reference:
            if tech == NEE:
                terms[0] /= pl_e[0]
            elif tech in (BP2D, BB1D):
                dl = self._length(split - 1)
                t = dl - beam_offset
                f = (t / dl) ** 2
                if tech == BB1D and split == 1:
                    f = 1.0 / (dl * dl)
                terms[split] *= f
        total = sum(terms) + sum(pde_pdf(i) for i in range(1, k))
        if tech in (EMITTER_HIT, NEE, BPT, LIGHT_TRACE):
            cur = bpt_pdf(split)
        else:
            cur = pde_pdf(split, {SURF: "surf", PP3D: "pp3d", PB2D: "pb2d", BB1D: "bb1d", BP2D: "bp2d"}[tech])
        return cur / total


class Records:
    """The recorded subpaths and contributions of one iteration
    (upbp_debug_mis_records)."""

    def __init__(self, rec: dict, scene: dict):
        self.sc = Scene(scene, rec["header"])
        sc = self.sc
        self.light = rec["light"].reshape(sc.light_paths, sc.max_verts, sc.vtx_words, 4)
        self.camera = rec["camera"].reshape(sc.camera_paths, sc.max_verts, sc.vtx_words, 4)
        self.events = rec["events"].reshape(-1, sc.ev_words, 4)

    def _vertex(self, table, path: int, k: int):
        """Vertex k of a subpath, the segments of the ray that reached it
        (measured from vertex k - 1), that ray's length to it and its unit
        direction."""
        r = table[path, k]
        flags = _bits(r[0, 3])
        if not flags & VTX_VALID:
            raise KeyError("vertex not recorded")
        ident = _bits(r[1, 3])
        if flags & VTX_LIGHT:
            kind = "light"
        elif flags & VTX_CAMERA:
            kind = "camera"
        elif flags & VTX_MEDIUM:
            kind = "medium"
        else:
            kind = "surface"
        pv = PathVertex(kind, r[0, :3], normal=r[1, :3] if kind in ("light", "surface", "camera") else None,
                        ident=ident, specular=bool(flags & (VTX_SPECULAR | VTX_DELTA)))
        d = r[4, :3].astype(np.float64)
        n = float(np.linalg.norm(d))
        return pv, self._ray_segments(table, path, k), float(r[3, 0]), (d / n if n > 0 else d)

    @staticmethod
    def _clip(segs, length):
        return [(d0, min(d1, length), m) for d0, d1, m in segs if d0 < length]

    @staticmethod
    def _flip(segs, length):
        return sorted([(max(0.0, length - d1), length - d0, m) for d0, d1, m in segs if d1 > d0])

    def full_path(self, ev: np.ndarray) -> tuple[FullPath, int, int]:
        """The full path of contribution record ev, its technique and the
        BPT split or merged-vertex index."""
        tech = _bits(ev[0, 0])
        cam_path, t = _bits(ev[0, 2]), _bits(ev[0, 3])
        light_path, s = _bits(ev[1, 0]), _bits(ev[1, 1])
        pl, pc = ev[2, :3].astype(np.float64), ev[3, :3].astype(np.float64)
        tl, tc = float(ev[2, 3]), float(ev[3, 3])
        nconn = _bits(ev[4, 0])
        conn = [(float(ev[5 + j, 0]), float(ev[5 + j, 1]), _bits(ev[5 + j, 2])) for j in range(nconn)]

        def camera_part(upto: int):
            """Camera vertices z_upto .. z_0 in light-to-camera order, the
            edges between them (segments measured from the light side) and
            their traced directions (light to camera) and lengths."""
            vs, es, gs = [], [], []
            for j in range(upto, -1, -1):
                pv, segs, dist, d = self._vertex(self.camera, cam_path, j)
                vs.append(pv)
                if j > 0:
                    es.append(self._flip(self._clip(segs, dist), dist))
                    gs.append((-d, dist))
            return vs, es, gs

        def light_part(upto: int):
            vs, es, gs = [], [], []
            for j in range(upto + 1):
                pv, segs, dist, d = self._vertex(self.light, light_path, j)
                vs.append(pv)
                if j > 0:
                    es.append(self._clip(segs, dist))
                    gs.append((d, dist))
            return vs, es, gs

        sc = self.sc
        if tech == EMITTER_HIT:
            vs, es, gs = camera_part(t)
            return FullPath(sc, vs, es, None, gs), tech, 0
        if tech == NEE:
            light_id = _bits(ev[1, 2])
            lt = sc.lights[light_id]
            n = np.cross(_vec(lt["p1"]) - _vec(lt["p0"]), _vec(lt["p2"]) - _vec(lt["p0"]))
            lv = PathVertex("light", pl, normal=n, ident=light_id)
            cvs, ces, cgs = camera_part(t)
            d = float(np.linalg.norm(cvs[0].pc - pl))
            return FullPath(sc, [lv] + cvs, [self._flip(self._clip(conn, d), d)] + ces, None, [None] + cgs), tech, 1
        if tech == BPT:
            lvs, les, lgs = light_part(s)
            cvs, ces, cgs = camera_part(t)
            d = float(np.linalg.norm(cvs[0].pc - lvs[-1].pl))
            return (FullPath(sc, lvs + cvs, les + [self._flip(self._clip(conn, d), d)] + ces, None, lgs + [None] + cgs),
                    tech, s + 1)
        if tech == LIGHT_TRACE:
            lvs, les, lgs = light_part(s)
            cam = PathVertex("camera", sc.cam_origin)
            d = float(np.linalg.norm(sc.cam_origin - lvs[-1].pl))
            return FullPath(sc, lvs + [cam], les + [self._clip(conn, d)], None, lgs + [None]), tech, s + 1
        # merges: the light side up to the merged vertex (the photon y_s, or
        # the point at tl on the photon beam of the ray y_{s-1} -> y_s), the
        # camera side from it (the camera vertex z_t, or the point at tc on the
        # query ray z_{t-1} -> z_t)
        if tech in (SURF, PP3D, PB2D):
            lvs, les, lgs = light_part(s)
            photon = lvs[-1]
        else:
            lvs, les, lgs = light_part(s - 1)
            _, segs, _, d = self._vertex_ray(self.light, light_path, s)
            les.append(self._clip(segs, tl))
            lgs.append((d, tl))
            photon = PathVertex("medium", pl, ident=self._medium_at(segs, tl))
            lvs.append(photon)
        if tech in (SURF, PP3D, BP2D):
            cvs, ces, cgs = camera_part(t)
            cam = cvs[0]
            cvs = cvs[1:]
        else:
            cvs, ces, cgs = camera_part(t - 1)
            _, segs, _, d = self._vertex_ray(self.camera, cam_path, t)
            ces = [self._flip(self._clip(segs, tc), tc)] + ces
            cgs = [(-d, tc)] + cgs
            cam = PathVertex("medium", pc, ident=self._medium_at(segs, tc))
        # the camera side's scattering function at the merged vertex
        mv = PathVertex(cam.kind, photon.pl, cam.pc, normal=cam.normal, ident=cam.id, normal_l=photon.normal)
        m = len(lvs) - 1
        return FullPath(sc, lvs[:-1] + [mv] + cvs, les + ces, m, lgs + cgs), tech, m

    def _vertex_ray(self, table, path, k):
        """The ray that reached slot k (recorded even when it hit nothing)."""
        r = table[path, k]
        d = r[4, :3].astype(np.float64)
        return None, self._ray_segments(table, path, k), float(r[3, 0]), d / np.linalg.norm(d)

    def _has(self, table, path, k) -> bool:
        return bool(_bits(table[path, k, 0, 3]) & VTX_VALID)

    def _ray_segments(self, table, path, k):
        r = table[path, k]
        nseg = _bits(r[2, 3])
        return [(float(r[5 + j, 0]), float(r[5 + j, 1]), _bits(r[5 + j, 2])) for j in range(nseg)]

    @staticmethod
    def _medium_at(segs, t):
        """Medium of the segment holding distance t of a ray."""
        for d0, d1, m in segs:
            if d0 <= t <= d1 * (1 + 1e-6) + 1e-7:
                return m
        return segs[-1][2]

    def check(self, limit: int | None = None, reference: bool | None = None):
        """(technique, GPU weight, FP64 weight, full path length) of every
        supported contribution, and the count of unsupported ones.  The FP64
        weight is the balance heuristic, or the reference's form of it
        (FullPath.weight) when the renderer ran without mis_exact (or
        `reference` says so)."""
        if reference is None:
            reference = not self.sc.mis_exact
        out, skipped = [], 0
        evs = self.events if limit is None else self.events[:limit]
        for ev in evs:
            try:
                fp, tech, split = self.full_path(ev)
                w = fp.weight(tech, split, reference=reference, beam_offset=float(ev[1, 3]))
            except (NotImplementedError, KeyError):
                skipped += 1
                continue
            out.append((tech, float(ev[0, 1]), w, fp.k))
        return out, skipped
