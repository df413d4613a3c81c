"""ctypes binding of oracle/_ref/libupbp_ref_cpu.so: the reference renderer's own
device programs and host loaders compiled for the CPU (see oracle/Makefile).

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use it, as the checker and the timed reference arm.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libupbp_ref_cpu.so")
REFERENCE_ROOT = "/root/reference"

_lib = None


SAH_LIB_PATH = os.path.join(HERE, "_ref", "libsah_ref.so")


def build(reference_root: str = REFERENCE_ROOT) -> bool:
    """Compiles the scene-BVH checker, and the oracle from the reference
    sources when they are present."""
    subprocess.run(["make", "-C", HERE, "sah", "-s"], check=True)
    if not os.path.isdir(os.path.join(reference_root, "gpuupbp")):
        return os.path.exists(LIB_PATH)
    subprocess.run(["make", "-C", HERE, f"REF={reference_root}", "-s"], check=True)
    return True


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle)")
        L = ctypes.CDLL(LIB_PATH)
        L.upbp_ref_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_void_p)]
        L.upbp_ref_create.restype = ctypes.c_int
        L.upbp_ref_run_iteration.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.upbp_ref_run_iteration.restype = ctypes.c_int
        L.upbp_ref_get_stats.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.upbp_ref_exception_counts.argtypes = [ctypes.c_void_p]
        L.upbp_ref_destroy.argtypes = [ctypes.c_void_p]
        L.upbp_ref_output_name.argtypes = [ctypes.c_void_p]
        L.upbp_ref_output_name.restype = ctypes.c_char_p
        L.upbp_ref_iteration_count.argtypes = [ctypes.c_void_p]
        L.upbp_ref_iteration_count.restype = ctypes.c_int
        L.upbp_ref_describe.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
        L.upbp_ref_describe.restype = ctypes.c_int
        L.upbp_ref_scene_json.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
        L.upbp_ref_scene_json.restype = ctypes.c_int
        L.upbp_ref_save_exr.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int]
        L.upbp_ref_save_exr.restype = ctypes.c_int
        _lib = L
    return _lib


_current = None


def save_exr(path: str, rgb, half: bool, compression: int) -> None:
    """Writes an (H, W, 3) float image with tinyexr's encoder (compression
    0 none, 1 RLE, 2 ZIPS, 3 ZIP), for tests of the library's EXR reader."""
    import numpy as np
    a = np.ascontiguousarray(rgb, np.float32)
    rc = lib().upbp_ref_save_exr(path.encode(), a.ctypes.data, a.shape[1], a.shape[0], int(half), compression)
    if rc != 0:
        raise RuntimeError(f"tinyexr could not write {path} (rc={rc})")


class RefRenderer:
    """The reference renderer on host cores, driven by its own command line.

    The reference keeps its launch parameters in one global, so only one
    instance can be alive; creating a new one closes the previous one.
    """

    def __init__(self, args: list[str], threads: int = 0):
        global _current
        L = lib()
        if _current is not None:
            _current.close()
        _current = self
        argv = ["gpuupbp"] + list(args)
        arr = (ctypes.c_char_p * len(argv))(*[a.encode() for a in argv])
        self._h = None
        h = ctypes.c_void_p()
        rc = L.upbp_ref_create(len(argv), arr, threads, ctypes.byref(h))
        if rc != 0:
            raise RuntimeError(f"reference command line rejected (rc={rc}): {args}")
        self._h = h
        st = self.stats()
        self.width, self.height = st["width"], st["height"]

    def run_iteration(self, iteration: int) -> np.ndarray:
        """This iteration's image (H, W, 3) float32, not accumulated."""
        out = np.zeros((self.height, self.width, 3), np.float32)
        lib().upbp_ref_run_iteration(self._h, iteration, out.ctypes.data)
        return out

    def render(self, iterations: int, start: int = 0) -> np.ndarray:
        acc = np.zeros((self.height, self.width, 3), np.float64)
        for it in range(start, start + iterations):
            acc += self.run_iteration(it)
        return (acc / iterations).astype(np.float32)

    def stats(self) -> dict:
        u = (ctypes.c_uint * 8)()
        t = (ctypes.c_double * 3)()
        lib().upbp_ref_get_stats(self._h, u, t)
        return {"vertices": u[0], "surface": u[1], "medium": u[2], "beams": u[3], "light_paths": u[4],
                "pixels": u[5], "width": u[6], "height": u[7],
                "t_light": t[0], "t_build": t[1], "t_camera": t[2]}

    def describe(self) -> dict:
        """The reference's parsed Config and loaded Scene, summarised."""
        import json
        buf = ctypes.create_string_buffer(8192)
        lib().upbp_ref_describe(self._h, buf, len(buf))
        return json.loads(buf.value.decode())

    def scene(self) -> dict:
        """Every record of the scene the reference's loader built: triangles
        (3 vertices, face normal, (material, light)), sphere boxes (lo, hi,
        (material, light)), materials, media, lights."""
        import json
        n = lib().upbp_ref_scene_json(self._h, None, 0)
        buf = ctypes.create_string_buffer(n)
        lib().upbp_ref_scene_json(self._h, buf, n)
        return json.loads(buf.value.decode())

    @staticmethod
    def exception_counts() -> list[int]:
        a = (ctypes.c_ulonglong * 8)()
        lib().upbp_ref_exception_counts(a)
        return list(a)

    def close(self):
        global _current
        if getattr(self, "_h", None):
            lib().upbp_ref_destroy(self._h)
            self._h = None
        if _current is self:
            _current = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sah_build(tri):
    """The sequential statement of the device's scene BVH build
    (oracle/sah_ref.cpp) on triangle records (n x 12 float32: v0, e1, e2 as
    float4s): (nodes n-1 x 16 float32 words, leaf order, widened boxes)."""
    import numpy as np
    tri = np.ascontiguousarray(tri, np.float32).reshape(-1, 12)
    n = len(tri)
    L = ctypes.CDLL(SAH_LIB_PATH)
    L.upbp_sah_ref_build.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p]
    nodes = np.zeros((max(n - 1, 1), 16), np.float32)
    order = np.zeros(n, np.uint32)
    boxes = np.zeros((n, 6), np.float32)
    L.upbp_sah_ref_build(tri.ctypes.data, n, nodes.ctypes.data, order.ctypes.data, boxes.ctypes.data)
    return nodes[:max(n - 1, 0)], order, boxes
