"""Seeded procedural scenes written in the reference's OBJ + MTL + AUX format.

The reference loads a scene from ``<name>.obj`` with its ``mtllib`` and an
auxiliary ``<name>.obj.aux`` file holding the camera, media, per-material
medium/priority/geometry-type settings and extra lights
(gpuupbp/misc/scene_loader_obj.cpp:335-612 for the AUX keys, 744-893 for OBJ).
Both renderers read the same generated files, so every parity test and the
benchmark run on identical inputs.

Workloads (sizes fixed by the benchmark spec):
  * ``box_medium``   -- 12-triangle unit box, diffuse walls (albedo U[0.2,0.8]
    per RGB channel), an icosphere of subdivision 3 (1280 triangles, radius
    0.3) bounding a homogeneous medium (sigma_s 0.5, sigma_a 0.1, HG g 0.3),
    one 2-triangle area light of radiance 10.
  * ``media_field``  -- ground plane, 20 seeded displaced icospheres of
    subdivision 6 (81 920 triangles each) bounding media with random
    coefficients nested by priority, one emissive sphere light and one quad
    area light.
  * ``dense_beams``  -- one thick medium (sigma_s 5, sigma_a 0.05, g 0.9)
    inside a displaced-box enclosure of about 500k triangles.
A ``tiny`` flag shrinks the meshes for quick tests without changing the
structure.
"""
from __future__ import annotations

import math
import contextlib
import os
from dataclasses import dataclass, field

import numpy as np


# --------------------------------------------------------------------------- meshes

def icosphere(subdiv: int):
    """Unit icosphere: (verts Nx3 float64, faces Mx3 int64), outward winding."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
                  [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(subdiv):
        nv = len(v)
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        v = np.concatenate([v, mid])
        m = inv.reshape(3, -1).T + nv  # midpoints of edges (01, 12, 20)
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([a, m01, m20], 1), np.stack([b, m12, m01], 1),
                            np.stack([c, m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return v, f


def displace(v: np.ndarray, rng: np.random.Generator, amplitude: float, waves: int = 6):
    """Radial displacement by a sum of random smooth waves (star-shaped result)."""
    d = np.zeros(len(v))
    for _ in range(waves):
        k = rng.normal(size=3)
        k /= np.linalg.norm(k)
        freq = rng.uniform(1.5, 4.0)
        phase = rng.uniform(0, 2 * math.pi)
        d += np.sin(freq * (v @ k) * math.pi + phase)
    d *= amplitude / waves
    return v * (1.0 + d)[:, None]


def grid_quad(n: int):
    """Unit square [0,1]^2 split into n x n cells of two triangles (z = 0)."""
    xs = np.linspace(0.0, 1.0, n + 1)
    gx, gy = np.meshgrid(xs, xs, indexing="xy")
    v = np.stack([gx.ravel(), gy.ravel(), np.zeros(gx.size)], 1)
    idx = np.arange((n + 1) * (n + 1)).reshape(n + 1, n + 1)
    a = idx[:-1, :-1].ravel()
    b = idx[:-1, 1:].ravel()
    c = idx[1:, 1:].ravel()
    d = idx[1:, :-1].ravel()
    f = np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d], 1)])
    return v, f


# --------------------------------------------------------------------------- writer

@dataclass
class Material:
    name: str
    kd: tuple = (0.0, 0.0, 0.0)
    ke: tuple | None = None
    ns: float = 0.0
    ks: tuple = (0.0, 0.0, 0.0)
    real: bool = True
    priority: int = -1
    medium: str | None = None
    mirror: tuple | None = None
    ior: float | None = None


@dataclass
class Medium:
    name: str
    absorption: tuple
    scattering: tuple
    g: float = 0.0
    emission: tuple = (0.0, 0.0, 0.0)
    continuation: float | None = None


@dataclass
class Camera:
    position: tuple
    target: tuple
    up: tuple
    hfov_deg: float


@contextlib.contextmanager
def _atomic_open(path: str):
    """A text file opened under a temporary name of this process and
    renamed to `path` when the block ends without an error."""
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        yield f
    os.replace(tmp, path)


@dataclass
class SceneBuilder:
    groups: list = field(default_factory=list)  # (material name, verts, faces, normals|None)
    materials: list = field(default_factory=list)
    media: list = field(default_factory=list)
    camera: Camera | None = None
    global_medium: str | None = None
    aux_lights: list = field(default_factory=list)  # AUX light lines (light_point, light_directional, ...)
    env_map: tuple | None = None  # (H x W x 3 image, scale, rotate): a light_background_em written beside the OBJ

    def add(self, material: str, verts, faces, normals=None):
        self.groups.append((material, np.asarray(verts, np.float64), np.asarray(faces, np.int64),
                            None if normals is None else np.asarray(normals, np.float64)))

    def triangle_count(self) -> int:
        return int(sum(len(g[2]) for g in self.groups))

    def write(self, obj_path: str):
        """Writes the .mtl, .obj and .aux files.  Each file is written under a
        name of this process and then renamed into place, so that processes
        writing the same scene at once (the ranks of a multi-process run)
        never read a partly written file."""
        base = os.path.basename(obj_path)
        mtl_name = base + ".mtl"
        d = os.path.dirname(obj_path) or "."
        with _atomic_open(os.path.join(d, mtl_name)) as fm:
            for m in self.materials:
                fm.write(f"newmtl {m.name}\n")
                fm.write("Kd %.6f %.6f %.6f\n" % m.kd)
                fm.write("Ks %.6f %.6f %.6f\n" % m.ks)
                fm.write("Ns %.6f\n" % m.ns)
                if m.ke is not None:
                    fm.write("Ke %.6f %.6f %.6f\n" % m.ke)
        with _atomic_open(obj_path) as fo:
            fo.write(f"mtllib {mtl_name}\n")
            voff, noff = 1, 1
            for mat, v, f, n in self.groups:
                np.savetxt(fo, v, fmt="v %.7f %.7f %.7f")
                if n is not None:
                    np.savetxt(fo, n, fmt="vn %.7f %.7f %.7f")
                fo.write(f"usemtl {mat}\n")
                fv = f + voff
                if n is not None:
                    fn = f + noff
                    inter = np.stack([fv[:, 0], fn[:, 0], fv[:, 1], fn[:, 1], fv[:, 2], fn[:, 2]], 1)
                    np.savetxt(fo, inter, fmt="f %d//%d %d//%d %d//%d")
                    noff += len(n)
                else:
                    np.savetxt(fo, fv, fmt="f %d %d %d")
                voff += len(v)
        with _atomic_open(obj_path + ".aux") as fa:
            c = self.camera
            pos = np.array(c.position, np.float64)
            fwd = np.array(c.target, np.float64) - pos
            fwd /= np.linalg.norm(fwd)
            up = np.array(c.up, np.float64)
            right = np.cross(fwd, up)
            right /= np.linalg.norm(right)
            up = np.cross(right, fwd)
            # rows: right, up, -forward, position (scene_loader_obj.cpp:215-243)
            for i, row in enumerate([right, up, -fwd, pos]):
                fa.write("TM_ROW%d %.7f %.7f %.7f\n" % (i, *row))
            fa.write("CAMERA_FOV %.7f\n" % math.radians(c.hfov_deg))
            fa.write("CAMERA_TDIST 1.0\n")
            for m in self.media:
                fa.write(f"medium {m.name}\n")
                fa.write("absorption %.6f %.6f %.6f\n" % m.absorption)
                fa.write("scattering %.6f %.6f %.6f\n" % m.scattering)
                fa.write("emission %.6f %.6f %.6f\n" % m.emission)
                fa.write("g %.6f\n" % m.g)
                if m.continuation is not None:
                    fa.write("continuation_probability %.6f\n" % m.continuation)
            for m in self.materials:
                fa.write(f"material {m.name}\n")
                fa.write("geometryType %s\n" % ("real" if m.real else "imaginary"))
                fa.write("priority %d\n" % m.priority)
                if m.medium is not None:
                    fa.write(f"mediumId {m.medium}\n")
                if m.mirror is not None:
                    fa.write("mirror %.6f %.6f %.6f\n" % m.mirror)
                if m.ior is not None:
                    fa.write("ior %.6f\n" % m.ior)
            if self.global_medium is not None:
                fa.write(f"globalMediumId {self.global_medium}\n")
            for line in self.aux_lights:
                fa.write(line + "\n")
            if self.env_map is not None:
                img, scale, rotate = self.env_map
                name = os.path.basename(obj_path) + ".env.exr"
                write_exr_float(os.path.join(os.path.dirname(obj_path), name), img)
                fa.write(f"light_background_em {scale} {rotate} {name}\n")


def _box_walls(sb: SceneBuilder, rng: np.random.Generator, lo=-0.5, hi=0.5):
    """Closed axis-aligned box, 6 walls x 2 triangles, normals facing inward."""
    # each wall: (corner, edge u, edge v, inward normal)
    L = hi - lo
    walls = [
        ((lo, lo, lo), (L, 0, 0), (0, 0, L), (0, 1, 0)),    # floor
        ((lo, hi, lo), (0, 0, L), (L, 0, 0), (0, -1, 0)),   # ceiling
        ((lo, lo, lo), (0, L, 0), (L, 0, 0), (0, 0, 1)),    # back
        ((lo, lo, hi), (L, 0, 0), (0, L, 0), (0, 0, -1)),   # front
        ((lo, lo, lo), (0, 0, L), (0, L, 0), (1, 0, 0)),    # left
        ((hi, lo, lo), (0, L, 0), (0, 0, L), (-1, 0, 0)),   # right
    ]
    for i, (c, u, v, n) in enumerate(walls):
        c, u, v, n = (np.array(x, np.float64) for x in (c, u, v, n))
        verts = np.stack([c, c + u, c + u + v, c + v])
        faces = np.array([[0, 1, 2], [0, 2, 3]])
        if np.dot(np.cross(u, v), n) < 0:
            faces = faces[:, ::-1]
        albedo = tuple(float(x) for x in rng.uniform(0.2, 0.8, size=3))
        sb.materials.append(Material(f"wall{i}", kd=albedo))
        sb.add(f"wall{i}", verts, faces, np.repeat(n[None], 4, 0))


def _quad_light(sb: SceneBuilder, name: str, center, size: float, normal_down=True, radiance=10.0):
    cx, cy, cz = center
    h = size / 2
    verts = np.array([[cx - h, cy, cz - h], [cx + h, cy, cz - h], [cx + h, cy, cz + h], [cx - h, cy, cz + h]])
    faces = np.array([[0, 1, 2], [0, 2, 3]])
    # winding gives the emitting side (area-light frame = e1 x e2)
    e = np.cross(verts[1] - verts[0], verts[2] - verts[0])
    if (e[1] > 0) == normal_down:
        faces = faces[:, ::-1]
    n = np.array([0, -1 if normal_down else 1, 0], np.float64)
    sb.materials.append(Material(name, kd=(0.0, 0.0, 0.0), ke=(radiance, radiance, radiance)))
    sb.add(name, verts, faces, np.repeat(n[None], 4, 0))


def box_medium(seed: int = 1, tiny: bool = False) -> SceneBuilder:
    """Unit box + icosphere medium + one quad light (the 256x256 plain workload)."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder()
    _box_walls(sb, rng)
    _quad_light(sb, "light", (0.0, 0.499, 0.0), 0.3)
    v, f = icosphere(1 if tiny else 3)
    sb.media.append(Medium("fog", absorption=(0.1, 0.1, 0.1), scattering=(0.5, 0.5, 0.5), g=0.3))
    sb.materials.append(Material("fog_boundary", real=False, priority=1, medium="fog"))
    sb.add("fog_boundary", v * 0.3, f, v)
    sb.camera = Camera(position=(0.0, 0.0, 0.45), target=(0.0, 0.0, -0.5), up=(0.0, 1.0, 0.0), hfov_deg=80.0)
    return sb


def media_field(seed: int = 2, tiny: bool = False) -> SceneBuilder:
    """Ground plane + 20 displaced icosphere media + sphere light + quad light."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder()
    gv, gf = grid_quad(1)
    gv = (gv - [0.5, 0.5, 0.0]) * 40.0
    ground = np.stack([gv[:, 0], np.zeros(len(gv)), gv[:, 1]], 1)
    gf = gf[:, ::-1]  # normal +y
    sb.materials.append(Material("ground", kd=tuple(float(x) for x in rng.uniform(0.3, 0.7, 3))))
    sb.add("ground", ground, gf, np.repeat(np.array([[0.0, 1.0, 0.0]]), len(ground), 0))
    sub = 2 if tiny else 6
    base_v, base_f = icosphere(sub)
    for i in range(20):
        gx, gz = i % 5, i // 5
        center = np.array([(gx - 2) * 2.2 + rng.uniform(-0.3, 0.3), 0.0, (gz - 1.5) * 2.2 + rng.uniform(-0.3, 0.3)])
        radius = rng.uniform(0.6, 1.0)
        center[1] = radius * 1.1
        v = displace(base_v, rng, amplitude=0.15) * radius + center
        mname = f"med{i}"
        ss = float(rng.uniform(0.1, 2.0))
        sa = float(rng.uniform(0.01, 0.3))
        sb.media.append(Medium(mname, absorption=(sa, sa, sa), scattering=(ss, ss, ss), g=float(rng.uniform(-0.5, 0.8))))
        sb.materials.append(Material(f"bound{i}", real=False, priority=i + 1, medium=mname))
        sb.add(f"bound{i}", v, base_f)
    # emissive sphere light (each triangle becomes an area light in the loader)
    lv, lf = icosphere(1)
    sb.materials.append(Material("sphere_light", kd=(0.0, 0.0, 0.0), ke=(20.0, 18.0, 15.0)))
    sb.add("sphere_light", lv * 0.5 + np.array([3.0, 6.0, 2.0]), lf)
    _quad_light(sb, "quad_light", (-3.0, 7.0, -2.0), 2.0, radiance=10.0)
    sb.camera = Camera(position=(0.0, 7.0, 12.0), target=(0.0, 0.5, 0.0), up=(0.0, 1.0, 0.0), hfov_deg=55.0)
    return sb


def dense_beams(seed: int = 5, tiny: bool = False) -> SceneBuilder:
    """Thick medium in a displaced-box enclosure of ~500k triangles."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder()
    n = 8 if tiny else 204  # 6 faces * 2 * 204^2 = 499 392 triangles
    faces_spec = [((0, 1, 0), 1), ((0, -1, 0), 1), ((1, 0, 0), 1), ((-1, 0, 0), 1), ((0, 0, 1), 1), ((0, 0, -1), 1)]
    sb.media.append(Medium("thick", absorption=(0.05, 0.05, 0.05), scattering=(5.0, 5.0, 5.0), g=0.9))
    sb.materials.append(Material("enclosure", kd=tuple(float(x) for x in rng.uniform(0.3, 0.7, 3)),
                                 real=True, priority=-1))
    sb.materials.append(Material("thick_boundary", real=False, priority=1, medium="thick"))
    qv, qf = grid_quad(n)
    for normal, _ in faces_spec:
        nrm = np.array(normal, np.float64)
        # inward normal = -nrm: wall at +nrm side of the cube [-1,1]^3
        a = np.array([1, 0, 0]) if abs(nrm[0]) < 0.5 else np.array([0, 1, 0])
        u = np.cross(nrm, a)
        w = np.cross(nrm, u)
        p = nrm[None] + (qv[:, 0:1] * 2 - 1) * u[None] + (qv[:, 1:2] * 2 - 1) * w[None]
        bump = 0.03 * np.sin(7.0 * p[:, 0] + rng.uniform(0, 6)) * np.sin(5.0 * p[:, 2] + rng.uniform(0, 6))
        p = p - nrm[None] * bump[:, None]
        f = qf.copy()
        e = np.cross(p[f[0, 1]] - p[f[0, 0]], p[f[0, 2]] - p[f[0, 0]])
        if np.dot(e, -nrm) < 0:
            f = f[:, ::-1]
        sb.add("enclosure", p, f, np.repeat(-nrm[None], len(p), 0))
    v, f = icosphere(3 if tiny else 4)
    sb.add("thick_boundary", v * 0.6, f, v)
    _quad_light(sb, "light", (0.0, 0.9, 0.0), 0.5, radiance=10.0)
    sb.camera = Camera(position=(0.0, 0.0, 0.95), target=(0.0, 0.0, -1.0), up=(0.0, 1.0, 0.0), hfov_deg=75.0)
    return sb


def glass_box(seed: int = 3, tiny: bool = False) -> SceneBuilder:
    """The unit box with specular and glossy materials: a real glass sphere
    (mirror 1, ior 1.5) holding a medium, a Phong back wall, beside the
    imaginary fog sphere."""
    rng = np.random.default_rng(seed)
    sb = box_medium(seed, tiny)
    sb.groups = [g for g in sb.groups if g[0] != "fog_boundary"]
    v, f = icosphere(1 if tiny else 3)
    sb.add("fog_boundary", v * 0.18 + np.array([-0.2, -0.25, -0.15]), f, v)
    sb.media.append(Medium("smoke", absorption=(0.3, 0.2, 0.1), scattering=(1.5, 1.5, 1.5), g=-0.2))
    sb.materials.append(Material("glass", real=True, priority=2, medium="smoke", mirror=(1.0, 1.0, 1.0), ior=1.5))
    sb.add("glass", v * 0.16 + np.array([0.18, -0.2, -0.2]), f, v)
    gloss = Material("gloss", kd=tuple(float(x) for x in rng.uniform(0.2, 0.4, 3)), ks=(0.4, 0.4, 0.4), ns=40.0)
    sb.materials.append(gloss)
    qv, qf = grid_quad(1)
    p = np.stack([qv[:, 0] * 0.98 - 0.49, qv[:, 1] * 0.98 - 0.49, np.full(len(qv), -0.49)], 1)
    sb.add("gloss", p, qf, np.repeat(np.array([[0.0, 0.0, 1.0]]), len(p), 0))
    return sb


def fog_box(seed: int = 4, tiny: bool = False) -> SceneBuilder:
    """The unit box filled with a thin global medium (globalMediumId; the
    camera starts in it) around the fog sphere, whose medium continues paths
    with probability 0.7 (continuation_probability)."""
    sb = box_medium(seed, tiny)
    sb.media[0].continuation = 0.7
    sb.media.append(Medium("air", absorption=(0.05, 0.08, 0.1), scattering=(0.3, 0.3, 0.3), g=0.5))
    sb.global_medium = "air"
    return sb


def media_field_lights(seed: int = 2, tiny: bool = False) -> SceneBuilder:
    """The media field with the AUX light types beside its area lights: a
    point light, a directional light and a constant background."""
    sb = media_field(seed, tiny)
    sb.aux_lights += ["light_point 1.5 4.0 3.0 30.0 25.0 20.0",
                      "light_directional -0.3 -1.0 -0.4 0.8 0.9 1.0",
                      "light_background_constant 0.15 0.2 0.3"]
    return sb


def write_exr_float(path: str, img: np.ndarray):
    """Writes an (H, W, 3) image as an uncompressed OpenEXR scanline file with
    FLOAT channels B, G, R (OpenEXR file layout: magic, version, attributes,
    offset table, one (y, size, B row, G row, R row) block per scanline)."""
    import struct
    img = np.ascontiguousarray(img, np.float32)
    h, w = img.shape[:2]

    def attr(name, typ, data):
        return name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<i", len(data)) + data

    chl = b"".join(c.encode() + b"\0" + struct.pack("<iB3xii", 2, 0, 1, 1) for c in "BGR") + b"\0"
    box = struct.pack("<iiii", 0, 0, w - 1, h - 1)
    hdr = (struct.pack("<ii", 20000630, 2) + attr("channels", "chlist", chl) + attr("compression", "compression", b"\0")
           + attr("dataWindow", "box2i", box) + attr("displayWindow", "box2i", box)
           + attr("lineOrder", "lineOrder", b"\0") + attr("pixelAspectRatio", "float", struct.pack("<f", 1.0))
           + attr("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0))
           + attr("screenWindowWidth", "float", struct.pack("<f", 1.0)) + b"\0")
    line = 12 * w
    start = len(hdr) + 8 * h
    offsets = struct.pack(f"<{h}Q", *[start + y * (8 + line) for y in range(h)])
    blocks = b"".join(struct.pack("<ii", y, line) + img[y, :, 2].tobytes() + img[y, :, 1].tobytes()
                      + img[y, :, 0].tobytes() for y in range(h))
    with open(path, "wb") as f:
        f.write(hdr + offsets + blocks)


def sky_image(seed: int, width: int = 64) -> np.ndarray:
    """A seeded lat-long sky (width x width/2): a blue gradient, noise and a
    bright sun lobe, so importance sampling has a peak to find."""
    rng = np.random.default_rng(seed)
    h = width // 2
    v = (np.arange(h) + 0.5) / h
    u = (np.arange(width) + 0.5) / width
    sky = np.zeros((h, width, 3), np.float32)
    sky[...] = (0.3 + 0.5 * (1 - v))[:, None, None] * np.array([0.5, 0.7, 1.0], np.float32)
    sky *= (1 + 0.2 * rng.random((h, width, 1))).astype(np.float32)
    su, sv = rng.uniform(0.2, 0.8), rng.uniform(0.15, 0.35)
    d2 = ((u[None, :] - su) * 2) ** 2 + (v[:, None] - sv) ** 2
    sky += (40.0 * np.exp(-d2 / 0.002))[..., None].astype(np.float32) * np.array([1.0, 0.9, 0.7], np.float32)
    return sky.astype(np.float32)


def media_field_env(seed: int = 2, tiny: bool = False) -> SceneBuilder:
    """The media field under an environment-map sky (light_background_em,
    scale 0.8, rotated by a quarter turn) beside its area lights."""
    sb = media_field(seed, tiny)
    sb.env_map = (sky_image(seed + 100), 0.8, 0.25)
    return sb


def media_row(seed: int = 7, tiny: bool = False) -> SceneBuilder:
    """Overflow of the imaginary boundaries a ray may meet between two real
    hits: 12 small fog spheres in a row along the camera's view axis, 24
    crossings for a camera ray along the row, more than the 8 the reference
    keeps (MAX_IMAGINARY_INTERSECTIONS), so those rays end with the
    intersection-stack failure."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder()
    _box_walls(sb, rng)
    _quad_light(sb, "light", (0.0, 0.499, 0.0), 0.3)
    v, f = icosphere(1 if tiny else 2)
    sb.media.append(Medium("fog", absorption=(0.05, 0.05, 0.05), scattering=(0.2, 0.2, 0.2), g=0.2))
    sb.materials.append(Material("fog_boundary", real=False, priority=1, medium="fog"))
    for i in range(12):
        sb.add("fog_boundary", v * 0.028 + np.array([0.0, 0.0, 0.33 - 0.068 * i]), f, v)
    sb.camera = Camera(position=(0.0, 0.0, 0.45), target=(0.0, 0.0, -0.5), up=(0.0, 1.0, 0.0), hfov_deg=30.0)
    return sb


def batch_job(seed: int, tiny: bool = False) -> SceneBuilder:
    """One job of the batched workload, drawn from its seed: a closed box with
    a quad light and 1-3 randomly displaced icospheres bounding homogeneous
    media (sigma_s in [0.1, 2], sigma_a in [0.01, 0.3], g in [-0.5, 0.8],
    nested by priority), about log-uniform in [1k, 200k] triangles (each
    sphere's subdivision the one nearest its share of the draw)."""
    rng = np.random.default_rng(10_000 + seed)
    sb = SceneBuilder()
    _box_walls(sb, rng)
    _quad_light(sb, "light", (0.0, 0.499, 0.0), 0.3)
    media = int(rng.integers(1, 4))
    target = math.exp(rng.uniform(math.log(1000.0), math.log(200000.0)))
    for i in range(media):
        share = max(target / media, 80.0)
        sub = int(min(7, max(1, round(math.log(share / 20.0, 4)))))
        if tiny:
            sub = min(sub, 2)
        v, f = icosphere(sub)
        radius = rng.uniform(0.12, 0.28)
        centre = rng.uniform(-0.45 + radius, 0.45 - radius, size=3)
        v = displace(v, rng, amplitude=0.12) * radius + centre
        name = f"m{i}"
        ss, sa = float(rng.uniform(0.1, 2.0)), float(rng.uniform(0.01, 0.3))
        sb.media.append(Medium(name, absorption=(sa, sa, sa), scattering=(ss, ss, ss), g=float(rng.uniform(-0.5, 0.8))))
        sb.materials.append(Material(f"b{i}", real=False, priority=i + 1, medium=name))
        sb.add(f"b{i}", v, f)
    sb.camera = Camera(position=(0.0, 0.0, 0.45), target=(0.0, 0.0, -0.5), up=(0.0, 1.0, 0.0), hfov_deg=80.0)
    return sb


def batch_job_config(seed: int) -> dict:
    """The view and path settings of batched job `seed`: resolution
    uniform in {64^2, 128^2, 256^2, 512^2}, path length uniform in [4, 16]."""
    rng = np.random.default_rng(20_000 + seed)
    side = int(rng.choice([64, 128, 256, 512]))
    return {"res": (side, side), "length": int(rng.integers(4, 17))}


WORKLOADS = {"media_field_env": media_field_env, "box_medium": box_medium, "media_field": media_field, "dense_beams": dense_beams,
             "media_field_lights": media_field_lights, "glass_box": glass_box, "fog_box": fog_box,
             "batch_job": batch_job, "media_row": media_row}


# Version of the generators' output: a change to any generator that changes
# the files it writes must bump it, so that no directory serves files an
# older generator left there.
GENERATOR_VERSION = 2


def write_workload(name: str, out_dir: str, seed: int | None = None, tiny: bool = False) -> str:
    """Writes the named workload into out_dir and returns the .obj path.

    The file name carries the workload, its size, the seed (`d` for the
    workload's default) and the generator version, so files written for
    other arguments or by another generator version are never reused."""
    os.makedirs(out_dir, exist_ok=True)
    fn = WORKLOADS[name]
    stem = f"{name}{'_tiny' if tiny else ''}_s{'d' if seed is None else int(seed)}_g{GENERATOR_VERSION}"
    path = os.path.join(out_dir, stem + ".obj")
    if not os.path.exists(path) or not os.path.exists(path + ".aux"):
        sb = fn(tiny=tiny) if seed is None else fn(seed=seed, tiny=tiny)
        sb.write(path)  # the .aux file, written last, marks a complete set
    return path
