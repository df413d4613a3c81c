"""Builds the in-tree CUDA library and executable for sm_100a.

  gpuupbp_b200/libupbp_b200.so         -- the C ABI declared in include/upbp.h
  gpuupbp_b200/libupbp_b200_misdbg.so  -- the same ABI built with UPBP_MIS_DEBUG: it also records
                                          every subpath vertex and contribution weight for the FP64
                                          full-path MIS check (upbp_debug_mis_records)
  gpuupbp_b200/upbp                    -- the command-line renderer on that ABI

nvcc cross-compiles without a GPU, so this runs on any machine with CUDA 12.8+.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libupbp_b200.so")
LIB_MISDBG = os.path.join(HERE, "libupbp_b200_misdbg.so")
EXE = os.path.join(HERE, "upbp")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_CXX = "/usr/bin/g++"   # system toolchain (dynamic libstdc++)
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-ccbin", HOST_CXX, "-Xcompiler", "-fPIC", "-diag-suppress", "549,550"]

DEVICE_SOURCES = ["upbp_capi.cu", "upbp_slot0.cu"]
HOST_SOURCES = ["host/upbp_cli.cpp", "host/upbp_scene.cpp", "host/upbp_predef.cpp", "host/upbp_exr.cpp",
                "host/upbp_exr_read.cpp"]


def _sources():
    out = []
    for root, _, files in os.walk(CSRC):
        for f in files:
            if f.endswith((".cu", ".cuh", ".cpp", ".h")):
                out.append(os.path.join(root, f))
    return out


def _stale(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    deps = _sources() + [os.path.join(HERE, "..", "include", "upbp.h"), os.path.abspath(__file__)]
    return any(os.path.getmtime(s) > t for s in deps)


def _run(cmd):
    r = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd))
    return r


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles libupbp_b200.so, libupbp_b200_misdbg.so and the upbp
    executable if sources changed."""
    if force or _stale(LIB) or _stale(LIB_MISDBG):
        host_objs = []
        for src in HOST_SOURCES:
            obj = os.path.join(CSRC, "_build", os.path.basename(src) + ".o")
            os.makedirs(os.path.dirname(obj), exist_ok=True)
            _run([NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj])
            host_objs.append(obj)
        for lib, defs, tag in ((LIB, [], ""), (LIB_MISDBG, ["-DUPBP_MIS_DEBUG"], ".misdbg")):
            objs = []
            for src in DEVICE_SOURCES:
                obj = os.path.join(CSRC, "_build", os.path.basename(src) + tag + ".o")
                cmd = [NVCC] + ARCH + FLAGS + defs + ["-c", src, "-o", obj]
                if verbose and not defs:
                    cmd += ["-Xptxas", "-v"]
                r = _run(cmd)
                if verbose:
                    sys.stderr.write(r.stderr)
                objs.append(obj)
            _run([NVCC] + ARCH + ["-ccbin", HOST_CXX, "-shared", "-o", lib] + objs + host_objs + ["-lcudart", "-lz"])
        _run([NVCC] + ARCH + FLAGS + ["-o", EXE, "upbp_main.cpp", "-L" + HERE, "-lupbp_b200",
                                      "-Xlinker", "-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
