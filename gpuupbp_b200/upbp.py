"""Python mirror of the renderer interface over the C ABI (include/upbp.h).

`Renderer` follows the reference's flow (gpuupbp/gpuupbp.cpp:57-148):
parse_commandline -> SceneLoader::load_scene -> Renderer::init ->
run_iteration per iteration -> scale and save.  All work runs in
libupbp_b200.so on the GPU; there is no CPU path here, and the module raises
if the library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libupbp_b200.so")
# the same ABI built with UPBP_MIS_DEBUG: records subpath vertices and MIS
# weights for the FP64 full-path check (upbp_debug_mis_records)
MISDBG_LIB_PATH = os.path.join(HERE, "libupbp_b200_misdbg.so")

UPBP_OK, UPBP_HELP = 0, 1
ERRORS = {-1: "invalid arguments", -2: "I/O error", -3: "CUDA error", -4: "no CUDA device", -5: "invalid scene",
          -6: "host error"}
STATUS_BITS = {1: "boundary stack", 2: "intersection array", 4: "volume segment array", 8: "intersection stack",
               16: "beam capacity", 32: "traversal stack"}


class UpbpError(RuntimeError):
    pass


class Config(ctypes.Structure):
    _fields_ = [
        ("scene_id", ctypes.c_int), ("scene_path", ctypes.c_char * 1024), ("algorithm_flags", ctypes.c_uint32),
        ("iteration_count", ctypes.c_int), ("max_time", ctypes.c_float), ("output_name", ctypes.c_char * 1024),
        ("res_x", ctypes.c_uint32), ("res_y", ctypes.c_uint32), ("max_path_length", ctypes.c_uint32),
        ("min_path_length", ctypes.c_uint32), ("path_count_per_iter", ctypes.c_float),
        ("query_beam_type", ctypes.c_int), ("photon_beam_type", ctypes.c_int),
        ("bb1d_radius_initial", ctypes.c_float), ("bb1d_radius_alpha", ctypes.c_float),
        ("bb1d_used_light_subpath_count", ctypes.c_float),
        ("bp2d_radius_initial", ctypes.c_float), ("bp2d_radius_alpha", ctypes.c_float),
        ("pb2d_radius_initial", ctypes.c_float), ("pb2d_radius_alpha", ctypes.c_float),
        ("pp3d_radius_initial", ctypes.c_float), ("pp3d_radius_alpha", ctypes.c_float),
        ("surf_radius_initial", ctypes.c_float), ("surf_radius_alpha", ctypes.c_float),
        ("continuous_output", ctypes.c_int), ("ignore_fully_spec_paths", ctypes.c_int), ("gpu_assert", ctypes.c_int),
        ("iteration_offset", ctypes.c_uint64), ("do_log", ctypes.c_int), ("use_shading_normal", ctypes.c_int),
        ("mis_exact", ctypes.c_int), ("guide_train_iterations", ctypes.c_int),
        ("checkpoint_path", ctypes.c_char * 1024), ("resume_path", ctypes.c_char * 1024),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("light_vertices", ctypes.c_uint32), ("surface_vertices", ctypes.c_uint32),
        ("medium_vertices", ctypes.c_uint32), ("light_beams", ctypes.c_uint32),
        ("light_paths", ctypes.c_uint32), ("camera_paths", ctypes.c_uint32), ("status", ctypes.c_uint32),
        ("iterations_done", ctypes.c_uint32), ("ms_light", ctypes.c_double), ("ms_build", ctypes.c_double),
        ("ms_camera", ctypes.c_double), ("triangle_count", ctypes.c_uint64), ("scene_radius", ctypes.c_double),
        ("work_light", ctypes.c_uint64 * 8), ("work_camera", ctypes.c_uint64 * 8), ("beam_chunks", ctypes.c_uint32),
        ("kernel_launches", ctypes.c_uint32), ("h2d_bytes", ctypes.c_uint32), ("d2h_bytes", ctypes.c_uint32),
        ("ms_light_sum", ctypes.c_double), ("ms_build_sum", ctypes.c_double), ("ms_camera_sum", ctypes.c_double),
        ("timed_iterations", ctypes.c_uint32), ("radius", ctypes.c_float * 6),
        ("work", (ctypes.c_uint64 * 8) * 9), ("ms_kernel_sum", ctypes.c_double * 9),
        ("segment_queries", ctypes.c_uint32), ("point_queries", ctypes.c_uint32),
        ("nee_samples", ctypes.c_uint32), ("bpt_pairs", ctypes.c_uint32),
        ("ms_guide", ctypes.c_double), ("ms_guide_sum", ctypes.c_double), ("ms_scene_bvh", ctypes.c_double),
        ("beam_map_passes", ctypes.c_uint32),
    ]


F3 = ctypes.c_float * 3


class MaterialDesc(ctypes.Structure):
    _fields_ = [("diffuse", F3), ("phong", F3), ("phong_exponent", ctypes.c_float), ("mirror", F3),
                ("ior", ctypes.c_float), ("priority", ctypes.c_int), ("real", ctypes.c_int), ("medium", ctypes.c_int)]


class MediumDesc(ctypes.Structure):
    _fields_ = [("absorption", F3), ("emission", F3), ("scattering", F3), ("continuation_prob", ctypes.c_float),
                ("mean_cosine", ctypes.c_float)]


class LightDesc(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("mat_id", ctypes.c_int), ("med_id", ctypes.c_int), ("p0", F3), ("p1", F3),
                ("p2", F3), ("intensity", F3), ("position", F3), ("scale", ctypes.c_float)]


class CameraDesc(ctypes.Structure):
    _fields_ = [("origin", F3), ("target", F3), ("roll", F3), ("horizontal_fov_deg", ctypes.c_float),
                ("focal_dist", ctypes.c_float), ("mat_id", ctypes.c_int), ("med_id", ctypes.c_int)]


class SceneDesc(ctypes.Structure):
    """upbp_scene_desc (include/upbp.h)."""
    _fields_ = [
        ("triangle_count", ctypes.c_uint32), ("verts", ctypes.POINTER(ctypes.c_float)),
        ("normals", ctypes.POINTER(ctypes.c_float)), ("tri_material", ctypes.POINTER(ctypes.c_int32)),
        ("tri_light", ctypes.POINTER(ctypes.c_int32)), ("material_count", ctypes.c_uint32),
        ("materials", ctypes.POINTER(MaterialDesc)), ("medium_count", ctypes.c_uint32),
        ("media", ctypes.POINTER(MediumDesc)), ("global_medium", ctypes.c_int32), ("light_count", ctypes.c_uint32),
        ("lights", ctypes.POINTER(LightDesc)), ("background_light", ctypes.c_int32), ("camera", CameraDesc),
        ("res_x", ctypes.c_uint32), ("res_y", ctypes.c_uint32), ("bbox_min", F3), ("bbox_max", F3),
        ("sphere_count", ctypes.c_uint32), ("spheres", ctypes.POINTER(ctypes.c_float)),
        ("sph_material", ctypes.POINTER(ctypes.c_int32)),
        ("env_width", ctypes.c_uint32), ("env_height", ctypes.c_uint32), ("env_rgb", ctypes.POINTER(ctypes.c_float)),
    ]


KERNELS = ["light_pass", "camera_extend", "pb2d_query", "bb1d_query", "surf_query", "pp3d_query", "bp2d_query",
           "nee_connect", "bpt_connect"]


WORK_NAMES = ["nodes", "tris", "rays", "point_cand", "point_hit", "beam_cand", "beam_hit", "vertex_loads"]


# symbols declared in include/upbp.h
EXPORTS = ["upbp_parse_command_line", "upbp_scene_load_obj", "upbp_scene_load_predefined", "upbp_scene_get_desc",
           "upbp_scene_free", "upbp_create", "upbp_run_iteration", "upbp_accumulate_to_host", "upbp_read_iteration",
           "upbp_get_stats", "upbp_destroy", "upbp_write_exr", "upbp_write_bmp", "upbp_write_hdr",
           "upbp_write_image", "upbp_get_stream", "upbp_last_error",
           "upbp_debug_photons", "upbp_debug_query", "upbp_debug_query_static", "upbp_get_device",
           "upbp_debug_mis_records", "upbp_guide_info", "upbp_guide_gradients", "upbp_run_batch",
           "upbp_set_grid_limit", "upbp_debug_scene_bvh", "upbp_save_checkpoint", "upbp_load_checkpoint"]

_libs = {}


def load_library(path: str = LIB_PATH):
    """Loads libupbp_b200.so, or another build of the same ABI (raises if it
    was not built)."""
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise UpbpError(f"{path} is missing: run gpuupbp_b200/build.py")
    L = ctypes.CDLL(path)
    P, VP = ctypes.POINTER, ctypes.c_void_p
    L.upbp_parse_command_line.argtypes = [ctypes.c_int, P(ctypes.c_char_p), P(Config)]
    L.upbp_scene_load_obj.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, P(VP)]
    L.upbp_scene_load_predefined.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, P(VP)]
    L.upbp_scene_get_desc.argtypes = [VP]
    L.upbp_scene_get_desc.restype = P(SceneDesc)
    L.upbp_scene_free.argtypes = [VP]
    L.upbp_create.argtypes = [VP, P(Config), P(VP)]
    L.upbp_run_iteration.argtypes = [VP, ctypes.c_int]
    L.upbp_accumulate_to_host.argtypes = [VP, VP, ctypes.c_double]
    L.upbp_read_iteration.argtypes = [VP, VP]
    L.upbp_get_stats.argtypes = [VP, P(Stats)]
    L.upbp_destroy.argtypes = [VP]
    L.upbp_write_exr.argtypes = [ctypes.c_char_p, VP, ctypes.c_uint32, ctypes.c_uint32]
    L.upbp_write_bmp.argtypes = [ctypes.c_char_p, VP, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float]
    L.upbp_write_hdr.argtypes = [ctypes.c_char_p, VP, ctypes.c_uint32, ctypes.c_uint32]
    L.upbp_write_image.argtypes = [ctypes.c_char_p, VP, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float]
    L.upbp_get_stream.argtypes = [VP]
    L.upbp_get_stream.restype = VP
    L.upbp_get_device.argtypes = [VP]
    L.upbp_run_batch.argtypes = [VP, ctypes.c_uint32, ctypes.c_int, ctypes.c_int]
    L.upbp_set_grid_limit.argtypes = [VP, ctypes.c_uint32]
    L.upbp_guide_info.argtypes = [VP, VP, ctypes.c_uint32]
    L.upbp_guide_gradients.argtypes = [VP, ctypes.c_uint32, VP, VP, ctypes.c_uint32, VP, VP, VP]
    L.upbp_debug_mis_records.argtypes = [VP, ctypes.c_int, VP, ctypes.c_uint64, P(ctypes.c_uint64)]
    L.upbp_last_error.restype = ctypes.c_char_p
    L.upbp_debug_photons.argtypes = [VP, ctypes.c_int, VP, ctypes.c_uint32, P(ctypes.c_uint32)]
    L.upbp_debug_query.argtypes = [VP, ctypes.c_int, VP, ctypes.c_uint32, VP, VP, ctypes.c_uint32]
    L.upbp_debug_query_static.argtypes = [VP, ctypes.c_int, VP, ctypes.c_uint32, VP, VP, ctypes.c_uint32]
    L.upbp_debug_scene_bvh.argtypes = [VP, ctypes.c_int, VP, ctypes.c_uint64, VP, ctypes.c_uint64,
                                       P(ctypes.c_uint32)]
    L.upbp_save_checkpoint.argtypes = [VP, ctypes.c_char_p]
    L.upbp_load_checkpoint.argtypes = [VP, ctypes.c_char_p]
    _libs[path] = L
    return L


def _check(rc: int, what: str, L=None):
    if rc != UPBP_OK:
        msg = (L or load_library()).upbp_last_error().decode(errors="replace")
        raise UpbpError(f"{what}: {ERRORS.get(rc, rc)}: {msg}")


def parse_command_line(args: list[str]) -> Config:
    """The reference's parse_commandline (same flags, defaults and errors)."""
    L = load_library()
    argv = ["upbp"] + list(args)
    arr = (ctypes.c_char_p * len(argv))(*[a.encode() for a in argv])
    cfg = Config()
    rc = L.upbp_parse_command_line(len(argv), arr, ctypes.byref(cfg))
    if rc == UPBP_HELP:
        raise UpbpError("help requested")
    _check(rc, "command line")
    return cfg


def load_scene(args: list[str]) -> dict:
    """The scene a command line names (-s <id> or -s -1 <file.obj>), loaded
    by the library on the host, as numpy arrays and record lists."""
    L = load_library()
    c = parse_command_line(args)
    sc = ctypes.c_void_p()
    if c.scene_id < 0:
        rc = L.upbp_scene_load_obj(c.scene_path, c.res_x, c.res_y, ctypes.byref(sc))
    else:
        rc = L.upbp_scene_load_predefined(c.scene_id, c.res_x, c.res_y, ctypes.byref(sc))
    _check(rc, "scene")
    try:
        d = L.upbp_scene_get_desc(sc).contents
        nt, ns = d.triangle_count, d.sphere_count

        def arr(ptr, n, dt):
            return np.ctypeslib.as_array(ptr, (n,)).astype(dt).copy() if n else np.zeros(0, dt)

        def recs(ptr, n):
            return [{k: (list(getattr(ptr[i], k)) if isinstance(getattr(ptr[i], k), ctypes.Array)
                         else getattr(ptr[i], k)) for k, _ in ptr[i]._fields_} for i in range(n)]

        return {
            "verts": arr(d.verts, 9 * nt, np.float32).reshape(nt, 3, 3),
            "normals": arr(d.normals, 12 * nt, np.float32).reshape(nt, 4, 3),
            "tri_material": arr(d.tri_material, nt, np.int32), "tri_light": arr(d.tri_light, nt, np.int32),
            "spheres": arr(d.spheres, 4 * ns, np.float32).reshape(ns, 4),
            "sph_material": arr(d.sph_material, ns, np.int32),
            "materials": recs(d.materials, d.material_count), "media": recs(d.media, d.medium_count),
            "lights": recs(d.lights, d.light_count), "global_medium": d.global_medium,
            "background_light": d.background_light,
            "bbox_min": np.array(list(d.bbox_min), np.float32), "bbox_max": np.array(list(d.bbox_max), np.float32),
            "env": (arr(d.env_rgb, 3 * d.env_width * d.env_height, np.float32).reshape(d.env_height, d.env_width, 3)
                    if d.env_rgb else None),
        }
    finally:
        L.upbp_scene_free(sc)


class Renderer:
    """Drop-in for the reference's Renderer on a scene file + command line."""

    def __init__(self, args: list[str], library: str = LIB_PATH):
        L = self._L = load_library(library)
        self.config = parse_command_line(args)
        c = self.config
        self._scene = ctypes.c_void_p()
        if c.scene_id < 0:
            rc = L.upbp_scene_load_obj(c.scene_path, c.res_x, c.res_y, ctypes.byref(self._scene))
        else:
            rc = L.upbp_scene_load_predefined(c.scene_id, c.res_x, c.res_y, ctypes.byref(self._scene))
        _check(rc, "scene")
        self._ctx = ctypes.c_void_p()
        _check(L.upbp_create(L.upbp_scene_get_desc(self._scene), ctypes.byref(c), ctypes.byref(self._ctx)), "init", L)
        self.width, self.height = c.res_x, c.res_y
        self.iterations = 0

    def run_iteration(self, iteration: int) -> int:
        """Renders one iteration; returns its device status bits (0, or
        UPBP_STATUS_* bits for paths ended early or beams dropped, as the
        reference ends or drops them; the image is complete either way)."""
        rc = self._L.upbp_run_iteration(self._ctx, iteration)
        if rc < 0:
            _check(rc, f"iteration {iteration}", self._L)
        self.iterations += 1
        self.last_status = rc
        return rc

    def iteration_image(self, out: np.ndarray | None = None) -> np.ndarray:
        """The last iteration's image, (H, W, 3) float32: a new array, or
        `out` (C-contiguous float32 of that shape, e.g. page-locked memory
        the caller reuses every iteration) filled and returned."""
        if out is None:
            out = np.empty((self.height, self.width, 3), np.float32)
        elif out.dtype != np.float32 or out.shape != (self.height, self.width, 3) or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float32 array of shape (H, W, 3)")
        _check(self._L.upbp_read_iteration(self._ctx, out.ctypes.data), "read")
        return out

    def accumulated(self, scale: float | None = None) -> np.ndarray:
        out = np.zeros((self.height, self.width, 3), np.float32)
        s = (1.0 / max(1, self.iterations)) if scale is None else scale
        _check(self._L.upbp_accumulate_to_host(self._ctx, out.ctypes.data, s), "accumulate")
        return out

    def render(self, iterations: int, start: int = 0) -> np.ndarray:
        for it in range(start, start + iterations):
            self.run_iteration(it)
        return self.accumulated()

    def stats(self) -> dict:
        st = Stats()
        _check(self._L.upbp_get_stats(self._ctx, ctypes.byref(st)), "stats")
        out = {k: getattr(st, k) for k, _ in Stats._fields_}
        out["work_light"] = dict(zip(WORK_NAMES, list(st.work_light)))
        out["work_camera"] = dict(zip(WORK_NAMES, list(st.work_camera)))
        out["radius"] = list(st.radius)
        out["work"] = {k: dict(zip(WORK_NAMES, list(st.work[i]))) for i, k in enumerate(KERNELS)}
        out["ms_kernel_sum"] = dict(zip(KERNELS, list(st.ms_kernel_sum)))
        return out

    def save_checkpoint(self, path: str):
        """Writes the render's state (upbp_save_checkpoint)."""
        _check(self._L.upbp_save_checkpoint(self._ctx, path.encode()), "save_checkpoint")

    def load_checkpoint(self, path: str) -> int:
        """Restores a render's state written by save_checkpoint for the same
        scene and configuration; returns the iterations it had rendered (the
        index to continue with)."""
        _check(self._L.upbp_load_checkpoint(self._ctx, path.encode()), "load_checkpoint")
        self.iterations = self.stats()["iterations_done"]
        return self.iterations

    def scene_bvh(self, real: bool):
        """The device-built scene BVH of one class of triangles
        (upbp_debug_scene_bvh): (nodes n-1 x 16 float32, leaf-order
        triangles n x 12 float32)."""
        L = self._L
        n = ctypes.c_uint32()
        _check(L.upbp_debug_scene_bvh(self._ctx, int(real), None, 0, None, 0, ctypes.byref(n)), "scene_bvh")
        nodes = np.zeros((max(n.value - 1, 0), 16), np.float32)
        tris = np.zeros((n.value, 12), np.float32)
        _check(L.upbp_debug_scene_bvh(self._ctx, int(real), nodes.ctypes.data if nodes.size else None, nodes.size,
                                      tris.ctypes.data if tris.size else None, tris.size, ctypes.byref(n)),
               "scene_bvh")
        return nodes, tris

    def photons(self, kind: int) -> np.ndarray:
        """Photon map contents of the last iteration (see upbp_debug_photons)."""
        L = self._L
        n = ctypes.c_uint32()
        _check(L.upbp_debug_photons(self._ctx, kind, None, 0, ctypes.byref(n)), "photons")
        width = 4 if kind < 2 else 8
        out = np.zeros((n.value, width), np.float32)
        if n.value:
            _check(L.upbp_debug_photons(self._ctx, kind, out.ctypes.data, n.value, ctypes.byref(n)), "photons")
        return out

    def query(self, kind: int, queries: np.ndarray, cap: int = 4096):
        """Neighbour sets of the estimators' range queries (upbp_debug_query)."""
        q = np.ascontiguousarray(queries, np.float32).reshape(-1, 8)
        counts = np.zeros(len(q), np.uint32)
        ids = np.zeros((len(q), cap), np.uint32)
        _check(self._L.upbp_debug_query(self._ctx, kind, q.ctypes.data, len(q), counts.ctypes.data,
                                               ids.ctypes.data, cap), "query")
        return [ids[i, :min(int(c), cap)].copy() for i, c in enumerate(counts)], counts

    def mis_records(self) -> dict:
        """MIS records of the last iteration (recording build only):
        header, light and camera subpath vertices, contributions, as float32
        arrays (upbp_debug_mis_records)."""
        out = {}
        for which, name in ((3, "header"), (0, "light"), (1, "camera"), (2, "events")):
            n = ctypes.c_uint64()
            _check(self._L.upbp_debug_mis_records(self._ctx, which, None, 0, ctypes.byref(n)), "mis records", self._L)
            a = np.zeros(n.value, np.float32)
            if n.value:
                _check(self._L.upbp_debug_mis_records(self._ctx, which, a.ctypes.data, n.value, ctypes.byref(n)),
                       "mis records", self._L)
            out[name] = a
        return out

    def stream_handle(self) -> int:
        return self._L.upbp_get_stream(self._ctx) or 0

    def close(self):
        L = self._L
        if getattr(self, "_ctx", None):
            L.upbp_destroy(self._ctx)
            self._ctx = None
        if getattr(self, "_scene", None):
            L.upbp_scene_free(self._scene)
            self._scene = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_exr(path: str, rgb: np.ndarray):
    a = np.ascontiguousarray(rgb, np.float32)
    _check(load_library().upbp_write_exr(path.encode(), a.ctypes.data, a.shape[1], a.shape[0]), "exr")


def write_image(path: str, rgb: np.ndarray, gamma: float = 2.2):
    """Writes an (H, W, 3) image as .exr, .bmp or .hdr by the name's extension."""
    a = np.ascontiguousarray(rgb, np.float32)
    _check(load_library().upbp_write_image(path.encode(), a.ctypes.data, a.shape[1], a.shape[0], gamma), "image")
