"""Benchmark of the UPBP render iteration on B200.

Workload (the plain large configuration): `media_field` -- 1280x720 pixels,
ground plane + 20 displaced icosphere media of 81 920 triangles each (about
1.64M triangles), one emissive sphere light and one quad light, path length
12, all five estimators plus BPT (`-a upbp_bpt+surf+pp3d+pb2d+bb1d+bp2d`),
one light path per pixel.  A step is one render iteration (light pass,
photon-map builds, camera pass).

Metric: paths/s = (camera + light subpaths per iteration) x iterations / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload media_field|dense_beams|batch|guided]

`--workload dense_beams` times the dense-beam stress case instead (1920x1080,
one thick medium in a 500k-triangle enclosure, path length 16, BB1D over the
beams of the first 600 000 light paths, about 2M, BP2D over all, about 7M,
and 4-5M photon points per iteration); `--workload batch` times 64 seeded
scene/view jobs rendered together (run_batch_workload); `--workload guided`
compares the learned proposal with plain UPBP at equal device time
(run_guided_workload).  The headline line is the default workload.

`value` is timed with CUDA events on the library's stream, inputs resident;
`e2e` renders the same iterations through the C ABI and reads every
iteration's image back into page-locked host memory.  Each is the median of
three windows of the same K iterations (all windows are in `repeats`).
nvidia-smi samples the clocks through all six windows.

N > 1 runs under torchrun, one rank per GPU; rank r renders iterations
r, r+N, ... (iterations are independent given the seed), so the scaling is
weak; value = all ranks' paths / max over ranks of the timed region.  The
reference arm times the reference's own render loop compiled for the host
cores (oracle/_ref/libupbp_ref_cpu.so) on a bounded sample of the workload:
1/64 of the camera paths with all of the light paths (media field), timed
from the same iteration index as the B200 arm.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

SCENE_DIR = os.environ.get("UPBP_SCENE_DIR", "/tmp/upbp_scenes")
# timed windows of K steps each; value and e2e are their medians
REPEATS = 3
RES = (1280, 720)
TECH = "upbp_bpt+surf+pp3d+pb2d+bb1d+bp2d"
METRIC = "paths/s (camera + light subpaths per second), plain UPBP render iterations"

# name: (resolution, path length, further flags, scene description)
WORKLOADS = {
    "media_field": (RES, 12, [], "20 displaced icosphere media (1.64M tris)"),
    "dense_beams": ((1920, 1080), 16, ["-r_initial_bb1d", "-0.004", "-r_initial_bp2d", "-0.004", "-pbc", "600000"],
                    "one thick medium (sigma_s 5, g 0.9) in a displaced-box enclosure (0.5M tris), "
                    "beam radius 0.004 x scene radius, beams from the first 600000 light paths"),
}


def workload_args(scene_path: str, res=RES, workload: str = "media_field") -> list[str]:
    _, length, extra, _ = WORKLOADS[workload]
    return ["-s", "-1", scene_path, "-a", TECH, "-l", str(length), "-r", f"{res[0]}x{res[1]}"] + extra


def measured_peaks() -> dict:
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples, started before the warm-up
    once its first sample is in (nvidia-smi's start-up stalls the host's CUDA
    calls for a while: started at the warm-up alone, it stalled the first
    timed window by about a third of a second) and summarised over the
    samples taken inside the timed region."""

    QUERY = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        """Starts nvidia-smi and waits (up to 10 s) for its first sample:
        its start-up (NVML initialisation) stalls the host's CUDA calls, so
        it must be over before anything is timed."""
        import atexit
        import threading
        atexit.register(self.stop)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        first = threading.Event()

        def pump(stream):
            for ln in stream:
                if ln.strip():
                    self.lines.append(ln.rstrip("\n"))
                    first.set()
            first.set()

        self._reader = threading.Thread(target=pump, args=(self.proc.stdout,), daemon=True)
        self._reader.start()
        first.wait(timeout=10.0)
        return self

    def stop(self):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.proc.wait()
            self._reader.join(timeout=5)
            self.proc = None

    def summary(self, t0: float | None = None, t1: float | None = None) -> dict:
        """Median SM clock and active throttle reasons of the samples taken
        between wall-clock times t0 and t1 (all samples when not given)."""
        import datetime
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                ts = None
            if t0 is not None and ts is not None and not (t0 - 0.25 <= ts <= t1 + 0.25):
                continue
            parts = parts[1:]
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# Algorithmic bytes of the camera-pass kernel per unit of counted work
# (record sizes of this build's layouts): BVH node 64 B (two child boxes +
# links), triangle 48 B (v0, e1, e2), per ray the hit's normals + record 72 B,
# photon point 16 B, accepted photon's vertex record 128 B, beam chunk 48 B,
# accepted beam record 128 B, BPT light-vertex record 128 B; plus 24 B of
# framebuffer read-modify-write per pixel.
BYTES_PER_WORK = {"nodes": 64, "tris": 48, "rays": 72, "point_cand": 16, "point_hit": 128, "beam_cand": 48,
                  "beam_hit": 128, "vertex_loads": 128}
# The PB2D, BB1D and BP2D searches walk the maps' 32-byte compressed nodes.
COMPRESSED_NODE_KERNELS = ("pb2d_query", "bb1d_query", "bp2d_query")


def algorithmic_bytes(work: dict, extra: float = 0.0, node_bytes: int = 64) -> float:
    per = dict(BYTES_PER_WORK, nodes=node_bytes)
    return float(sum(per[k] * v for k, v in work.items())) + extra


# Bytes of the query records each camera-side kernel writes or reads.
SEG_RECORD, POINT_RECORD = 128, 144
# PB2D / BB1D hit-list entry (query record, neighbour), written by the
# search kernel and read by the evaluation kernel.
HIT_RECORD = 8
# Deferred connections: an NEE sample reads its 80 B record and 64 B of its
# camera vertex and writes a 16 B contribution; a BPT pair reads its 8 B
# pair and 144 B of its camera vertex and writes 16 B (the light vertex is
# counted by vertex_loads, the occlusion ray by the traversal counters).
NEE_BYTES, PAIR_BYTES = 160.0, 168.0


def kernel_rooflines(st: dict, pixels: int) -> dict:
    """Algorithmic bytes and time per launch of each kernel of an iteration."""
    n = max(1, st["timed_iterations"])
    ms = st["ms_kernel_sum"]
    nseg, npt = st["segment_queries"], st["point_queries"]
    nnee, npairs = st["nee_samples"], st["bpt_pairs"]
    hits = st["work"]["bb1d_query"]["beam_hit"]
    pb2d_hits = st["work"]["pb2d_query"]["point_hit"]
    extra = {"light_pass": 0.0,
             "camera_extend": 12.0 * pixels + SEG_RECORD * nseg + POINT_RECORD * npt,
             "pb2d_query": SEG_RECORD * nseg + HIT_RECORD * 2 * pb2d_hits, "bb1d_query": SEG_RECORD * nseg + HIT_RECORD * 2 * hits,
             "surf_query": POINT_RECORD * npt, "pp3d_query": POINT_RECORD * npt,
             "bp2d_query": POINT_RECORD * npt + HIT_RECORD * 2 * st["work"]["bp2d_query"]["beam_hit"],
             "nee_connect": NEE_BYTES * nnee, "bpt_connect": PAIR_BYTES * npairs}
    out = {}
    for k, w in st["work"].items():
        t = ms[k] / n
        b = algorithmic_bytes(w, extra[k], 32 if k in COMPRESSED_NODE_KERNELS else 64)
        out[k] = {"ms": t, "bytes": b, "gbs": (b / (t * 1e-3) / 1e9) if t > 0 else 0.0}
    return out


def iteration_bytes(st: dict, pixels: int) -> float:
    """Algorithmic bytes of one whole iteration with implementation-independent
    record sizes: rays (node visits x 32 B + triangle tests x 40 B), stored
    light vertices 80 B and beams 128 B (written and read), query candidates x
    their record (photon 80 B, beam 128 B), BPT connections 80 B, photon-map
    builds (8-byte key/value + one 32-byte node per primitive), pixels 12 B
    (written and read)."""
    w = st["work"]
    rays = sum(w[k]["nodes"] * 32 + w[k]["tris"] * 40
               for k in ("light_pass", "camera_extend", "nee_connect", "bpt_connect"))
    cand = sum(w[k]["point_cand"] * 80 + w[k]["beam_cand"] * 128
               for k in ("surf_query", "pp3d_query", "pb2d_query", "bb1d_query", "bp2d_query"))
    build = (st["surface_vertices"] + st["medium_vertices"] + st["beam_chunks"]) * (8 + 32)
    return float(rays + st["light_vertices"] * 80 * 2 + st["light_beams"] * 128 * 2 + cand + st["bpt_pairs"] * 80
                 + build + pixels * 12 * 2)


def profiled_traffic() -> float | None:
    """DRAM bytes per iteration of the BB1D kernels from the committed ncu summary."""
    p = os.path.join(HERE, "profiles", "bb1d_query_media_field.md")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for ln in f:
            if ln.startswith("traffic_bytes_per_launch:"):
                try:
                    return float(ln.split(":", 1)[1].strip())
                except ValueError:
                    return None
    return None


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_b200(args) -> dict | None:
    import torch
    from gpuupbp_b200 import scenes, upbp

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        pg = dist
    scene = scenes.write_workload(args.workload, SCENE_DIR) if rank == 0 else None
    if pg is not None:
        pg.barrier()
        scene = scenes.write_workload(args.workload, SCENE_DIR)
    r = upbp.Renderer(workload_args(scene, args.res, args.workload))
    paths_per_iter = r.config.res_x * r.config.res_y + int(r.config.path_count_per_iter)
    stream = torch.cuda.ExternalStream(r.stream_handle())
    # rank r renders iterations r, r+N, ...; the device-timed and the
    # end-to-end runs render the same iterations (the radius schedule shrinks
    # with the iteration index, so later iterations are cheaper)
    clk = ClockSampler(local).start()
    for k in range(args.warmup):
        r.run_iteration(rank + world * k)
    timed_iterations = [rank + world * (args.warmup + k) for k in range(args.steps)]
    r.stats()  # drain the event ring

    # the step's result is read into page-locked host memory the caller owns
    result = torch.empty((r.height, r.width, 3), dtype=torch.float32, pin_memory=True).numpy()

    window = []

    def timed(iterations: list, readback: bool):
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        window.append(time.time())
        t0.record(stream)
        wall = time.perf_counter()
        for it in iterations:
            r.run_iteration(it)
            if readback:
                r.iteration_image(out=result)  # device->host of this step's result
        t1.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall
        window.append(time.time())
        ms = t0.elapsed_time(t1)
        if pg is not None:
            t = torch.tensor([ms], device="cuda")
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ms = float(t.item())
        return ms, wall

    # three windows of the same K iterations each, device-timed then end to
    # end; the clock sampler runs through all of them
    runs = [timed(timed_iterations, False) for _ in range(REPEATS)]
    st = r.stats()
    runs_e2e = [timed(timed_iterations, True) for _ in range(REPEATS)]
    st_e2e = r.stats()
    clk.stop()
    ms = statistics.median(m for m, _ in runs)
    ms_e2e = statistics.median(m for m, _ in runs_e2e)
    wall = statistics.median(w for _, w in runs)
    wall_e2e = statistics.median(w for _, w in runs_e2e)

    # final reduction of the accumulated images over ranks (output time, untimed)
    if pg is not None:
        acc = torch.from_numpy(r.accumulated(scale=1.0)).cuda()
        pg.all_reduce(acc)
        pg.barrier()
        pg.destroy_process_group()
    if rank != 0:
        r.close()
        return None

    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    pixels = r.config.res_x * r.config.res_y
    cam_ms = st["ms_camera_sum"] / max(1, st["timed_iterations"])
    kernels = kernel_rooflines(st, pixels)
    top = max(kernels, key=lambda k: kernels[k]["ms"])
    b_top, top_ms = kernels[top]["bytes"], kernels[top]["ms"]
    achieved = kernels[top]["gbs"]
    # the committed capture is scaled to the default resolution only
    traffic = (profiled_traffic() if top == "bb1d_query" and args.workload == "media_field" and tuple(args.res) == RES
               else None)
    b_iter = iteration_bytes(st, pixels)
    iteration_roofline = {"bound": "hbm", "achieved": b_iter / (ms / args.steps * 1e-3) / 1e9, "peak": hbm,
                          "unit": "GB/s", "frac": b_iter / (ms / args.steps * 1e-3) / 1e9 / hbm,
                          "algorithmic_bytes_per_step": b_iter, "peak_source": peak_src}
    total_paths = paths_per_iter * args.steps * world
    value = total_paths / (ms * 1e-3)
    e2e = total_paths / (ms_e2e * 1e-3)
    out = {
        "metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene, OBJ/MTL/AUX)",
        "config": {"workload": f"{args.workload}: {args.res[0]}x{args.res[1]}, {WORKLOADS[args.workload][3]}, "
                               f"{TECH}, path length {WORKLOADS[args.workload][1]}, 1 light path per pixel",
                   "triangles": int(st["triangle_count"]), "light_paths_per_iter": int(r.config.path_count_per_iter),
                   "camera_paths_per_iter": pixels, "parallelism": f"iterations sharded over {world} rank(s)",
                   "l2": "inputs larger than L2 (scene BVH + triangle data, photon records per iteration)"},
        "e2e": {"value": e2e, "unit": "paths/s", "h2d_bytes_per_step": int(st_e2e["h2d_bytes"]),
                "d2h_bytes_per_step": int(st_e2e["d2h_bytes"]) + pixels * 12,
                "wall_s": wall_e2e},
        "gpu_launches": int(st["kernel_launches"]) * args.steps,
        "roofline": {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm, "peak_source": peak_src,
                     "traffic": traffic, "algorithmic_bytes_per_launch": b_top, "launch_ms": top_ms},
        "iteration_roofline": iteration_roofline,
        "kernels": kernels,
        "clocks": clk.summary(window[0], window[-1]),
        "repeats": {"windows": REPEATS, "ms_per_step": [m / args.steps for m, _ in runs],
                    "e2e_ms_per_step": [m / args.steps for m, _ in runs_e2e],
                    "statistic": "median of the windows"},
        "passes_ms": {"light": st["ms_light_sum"] / max(1, st["timed_iterations"]),
                      "build": st["ms_build_sum"] / max(1, st["timed_iterations"]), "camera": cam_ms},
        "work": st["work"], "queries": {"segment": st["segment_queries"], "point": st["point_queries"],
                    "nee_samples": st["nee_samples"], "bpt_pairs": st["bpt_pairs"]},
        "status": int(st["status"]), "wall_s": wall,
    }
    r.close()
    return out


def reference_sample_args(workload: str) -> tuple[list[str], tuple[int, int], int]:
    """Command line of the reference's CPU sample of a workload: 1/8 of the
    width and height (1/64 of the camera paths).  On the media field it keeps
    every light path of the full-size workload (-pcpi = its pixel count),
    so photon, beam and query densities are the benchmark's own.  The dense
    beams keep 1/64 of the light paths (and of -pbc): at full density one
    iteration of its CPU build takes minutes (86 s at 48x27 on 8 threads)."""
    from gpuupbp_b200 import scenes

    scene = scenes.write_workload(workload, SCENE_DIR)
    full = WORKLOADS[workload][0]
    res = (full[0] // 8, full[1] // 8)
    args = workload_args(scene, res, workload)
    if workload == "media_field":
        light_paths = full[0] * full[1]
        args += ["-pcpi", str(light_paths)]
    else:
        light_paths = res[0] * res[1]
        if "-pbc" in args:  # the same fraction of beam-storing light paths
            i = args.index("-pbc") + 1
            args[i] = str(max(1, int(float(args[i]) / 64)))
    return args, res, light_paths


def run_reference_sample(seconds: float, threads: int, warmup: int = 1, max_iters: int | None = None,
                         workload: str = "media_field") -> dict:
    """Times the reference's render loop on host cores on a bounded sample of
    the workload (reference_sample_args).  Iterations 0 .. warmup-1 run
    untimed; the timed ones start at iteration `warmup`, as the B200 arm's
    do, and run until `seconds` have been timed or `max_iters` iterations."""
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import ref_cpu

    args, res, light_paths = reference_sample_args(workload)
    r = ref_cpu.RefRenderer(args, threads=threads)
    for w in range(warmup):
        r.run_iteration(w)
    it, n, t = warmup, 0, 0.0
    while (n == 0 or t < seconds) and (max_iters is None or n < max_iters):
        t0 = time.perf_counter()
        r.run_iteration(it)
        t += time.perf_counter() - t0
        it += 1
        n += 1
    st = r.stats()
    paths = (res[0] * res[1] + st["light_paths"]) * n
    r.close()
    return {"value": paths / t, "unit": "paths/s", "cores": threads, "kind": "reference",
            "sample": f"{workload} scene at {res[0]}x{res[1]} (1/64 of the camera paths) with "
                      f"{st['light_paths']} light paths per iteration, iterations {warmup}..{it - 1} timed "
                      f"({t:.1f} s on {threads} host threads)"}


def run_batch_workload(args) -> dict:
    """Config 3: 64 seeded jobs (resolution 64^2..512^2, path length 4..16,
    1k..200k triangles of displaced icospheres bounding 1-3 media in a box),
    rendered a batch iteration at a time through upbp_run_batch after the
    batch autotuner chose workers and the per-job launch cap.  A step is one
    iteration of every job; value = all jobs' camera + light subpaths per
    second; the same jobs run one after another (one worker, no cap) give the
    sequential figure beside it."""
    import torch

    from gpuupbp_b200 import batch
    jobs = [batch.job_args(j, SCENE_DIR) for j in range(64)]
    b = batch.Batch(jobs)
    paths = b.paths_per_iteration()
    free0, total = torch.cuda.mem_get_info()
    tune = batch.autotune(b, 0, workers=(8, 16, 32), limits=(0, 148 * 2))
    free1, _ = torch.cuda.mem_get_info()
    it = tune["next_iteration"]
    for _ in range(args.warmup):
        b.run_iteration(it)
        it += 1
    windows = []
    for _ in range(REPEATS):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            b.run_iteration(it)
            it += 1
        torch.cuda.synchronize()
        windows.append(time.perf_counter() - t0)
    t = statistics.median(windows)
    b.set_grid_limit(0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.run_iteration(it, workers=1)
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    res = sorted({a[a.index("-r") + 1] for a in jobs})
    lengths = [int(a[a.index("-l") + 1]) for a in jobs]
    b.close()
    return {"metric": "paths/s of a batch of 64 independent scene/view jobs", "value": paths * args.steps / t,
            "unit": "paths/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded procedural jobs)",
            "config": {"workload": "batch: 64 jobs, resolutions " + ",".join(res) +
                                   f", path lengths {min(lengths)}..{max(lengths)}, upbp_all",
                       "paths_per_step": paths, "timing": "wall clock around whole batch iterations, median of "
                                                          f"{REPEATS} windows"},
            "device_memory_gb": {"total": total / 1e9, "used_after_create": (total - free0) / 1e9,
                                 "used_after_autotune": (total - free1) / 1e9},
            "autotune": tune, "sequential": {"value": paths / t_seq, "unit": "paths/s",
                                             "note": "the same jobs one after another, one worker, no launch cap"},
            "repeats": {"s_per_window": windows}}


# FLOPs of the proposal's network per row: forward 2 x (96x64 + 64x64 + 64x64
# + 64x48) multiply-adds; a training row adds the weight gradients (as many)
# and the hidden gradients 2 x (48x64 + 64x64 + 64x64)
GUIDE_FWD_FLOP = 2 * (96 * 64 + 64 * 64 + 64 * 64 + 64 * 48)
GUIDE_TRAIN_FLOP = 2 * GUIDE_FWD_FLOP + 2 * (48 * 64 + 64 * 64 + 64 * 64)
GUIDE_BATCH, GUIDE_STEPS_PER_ITERATION = 1 << 18, 4
CONFIG1_ARGS = ["-a", "upbp_all", "-l", "8", "-r", "256x256", "-r_initial", "-0.02", "-r_alpha", "0.75"]


def run_guided_workload(args) -> dict:
    """Config 4: the learned proposal (-guide 8: trained online on the light
    subpaths' medium records during the first 8 of 60 iterations) on config
    1's scene -- the 256x256 box with the icosphere medium, BPT + SURF + PP3D
    + PB2D + BB1D, path length 8, radius 0.01 x scene diameter shrinking with
    alpha 0.75 -- against plain UPBP at equal device time.  Both are compared
    by relMSE with a converged plain render of --ref-iterations iterations on
    independent random streams.  value = relMSE(plain) / relMSE(guided) at
    equal time (above 1: the proposal pays).  The training phase (4 fused
    tcgen05 training steps of 2^18 rows and the table bake per training
    iteration) is reported against the tensor peak."""
    import numpy as np
    import torch

    from gpuupbp_b200 import quality, scenes, upbp
    path = scenes.write_workload("box_medium", SCENE_DIR)
    plain = ["-s", "-1", path] + CONFIG1_ARGS
    guided = plain + ["-guide", "8"]
    res = quality.equal_time(plain, guided, args.ref_iterations, 60)
    # the training phase alone, from the library's own events
    r = upbp.Renderer(guided)
    r.stats()
    for it in range(8):
        r.run_iteration(it)
    st = r.stats()
    info = np.zeros(9, np.float32)
    r._L.upbp_guide_info(r._ctx, info.ctypes.data, 9)
    r.close()
    torch.cuda.synchronize()
    table_rows = int(info[4])
    flop = GUIDE_STEPS_PER_ITERATION * GUIDE_BATCH * GUIDE_TRAIN_FLOP + table_rows * GUIDE_FWD_FLOP
    ms = st["ms_guide_sum"] / max(1, st["timed_iterations"])
    peaks = measured_peaks()
    peak = peaks.get("bf16_tflops") or 1590.0
    achieved = flop / (ms * 1e-3) / 1e12
    return {"metric": "equal-time relMSE ratio, plain / guided UPBP (config 4)",
            "value": res["relmse_ratio_plain_over_other"], "unit": "x", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32 render, f16 network with f32 accumulation", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": "guided: box_medium 256x256, upbp_all, path length 8, -guide 8, 60 iterations; "
                                   f"reference {args.ref_iterations} plain iterations"},
            "equal_time": res,
            "guided_ms_per_iteration": res["other_ms"] / res["other_iterations"],
            "plain_ms_per_iteration": res["plain_ms"] / res["plain_iterations"],
            "training": {"ms_per_training_iteration": ms, "steps_per_iteration": GUIDE_STEPS_PER_ITERATION,
                         "batch_rows": GUIDE_BATCH, "table_rows": table_rows, "final_loss": float(info[2]),
                         "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                                      "frac": achieved / peak, "peak_source": "measured" if peaks else "fallback",
                                      "flop_per_iteration": flop}}}


def run_dense_quality_workload(args) -> dict:
    """Config 5's guided form: the dense-beam enclosure (one thick medium,
    sigma_s 5, g 0.9, 0.5M triangles, path length 16, beam radius 0.004 x
    scene radius, BB1D over the beams of the first 600 000 light paths) with
    all 2 073 600 light paths of the 1920x1080 workload on a 480x270 camera
    (a bounded sample: 1/16 of the camera paths, the photon, beam and query
    densities of the full case), the learned proposal (-guide 8) against the
    plain method at equal device time, by relMSE against a converged plain
    render of --ref-iterations iterations.  Also the plain method's query
    throughput (segment + point queries per second) and the BB1D kernels'
    algorithmic GB/s."""
    import torch

    from gpuupbp_b200 import quality, scenes, upbp
    path = scenes.write_workload("dense_beams", SCENE_DIR)
    plain = workload_args(path, (480, 270), "dense_beams") + ["-pcpi", str(1920 * 1080)]
    guided = plain + ["-guide", "8"]
    res = quality.equal_time(plain, guided, args.ref_iterations, args.method_iterations)
    r = upbp.Renderer(plain)
    stream = torch.cuda.ExternalStream(r.stream_handle())
    for it in range(2):
        r.run_iteration(it)
    r.stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for it in range(2, 6):
        r.run_iteration(it)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 4
    st = r.stats()
    r.close()
    kernels = kernel_rooflines(st, 480 * 270)
    queries = st["segment_queries"] + st["point_queries"]
    return {"metric": "equal-time relMSE ratio, plain / guided UPBP (config 5 sample)",
            "value": res["relmse_ratio_plain_over_other"], "unit": "x", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": "dense_quality: dense_beams enclosure, 480x270 camera with the 1920x1080 "
                                   f"light paths, path length 16, -guide 8, {args.method_iterations} guided "
                                   f"iterations; reference {args.ref_iterations} plain iterations"},
            "equal_time": res, "plain_ms_per_iteration": ms,
            "queries_per_s": queries / (ms * 1e-3),
            "bb1d_query": kernels["bb1d_query"], "bp2d_query": kernels["bp2d_query"]}


def run_batch_quality_workload(args) -> dict:
    """Config 3's quality target: the guided, batched renderer against the
    plain single-scene renderer at equal wall time, by relMSE per job
    against each job's converged plain render (quality.batch_equal_time).
    Jobs 0..--jobs-1 of the seeded 64 (a bounded sample of config 3, so that
    the converged references -- --ref-iterations iterations of every job --
    stay within minutes); the guided jobs train their proposal during the
    first 8 of --method-iterations iterations.  value = mean relMSE of the
    plain renderer / mean relMSE of the guided batch (above 1: the batched,
    guided form wins)."""
    from gpuupbp_b200 import batch, quality
    jobs = [batch.job_args(j, SCENE_DIR) for j in range(args.jobs)]
    res = quality.batch_equal_time(jobs, ["-guide", "8"], args.ref_iterations, args.method_iterations)
    return {"metric": "equal-time relMSE ratio, plain single-scene / guided batched UPBP (config 3 sample)",
            "value": res["relmse_ratio_plain_over_method"], "unit": "x", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (seeded procedural jobs)",
            "config": {"workload": f"batch_quality: jobs 0..{args.jobs - 1} of the 64 seeded config-3 jobs, "
                                   f"upbp_all, guided (-guide 8) and batched vs plain one job at a time, "
                                   f"{args.method_iterations} guided iterations, reference "
                                   f"{args.ref_iterations} plain iterations per job",
                       "timing": "wall clock of whole batch iterations"},
            "equal_time": res}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="media_field", choices=sorted(WORKLOADS) + ["batch", "batch_quality", "dense_quality", "guided"])
    ap.add_argument("--ref-iterations", type=int, default=None,
                    help="iterations of the converged plain render the guided (default 4096) and batch_quality "
                         "(default 192) workloads compare with")
    ap.add_argument("--jobs", type=int, default=16, help="batch_quality: jobs of the seeded 64")
    ap.add_argument("--method-iterations", type=int, default=None,
                    help="guided iterations of batch_quality (default 24) and dense_quality (default 16)")
    ap.add_argument("--res", default=None,
                    help="image size WxH (default: the workload's); smaller sizes are for profiling captures, "
                         "not bench lines")
    args = ap.parse_args()
    if args.workload == "batch":
        print(json.dumps(run_batch_workload(args)))
        return
    if args.workload == "guided":
        args.ref_iterations = args.ref_iterations or 4096
        print(json.dumps(run_guided_workload(args)))
        return
    if args.workload == "dense_quality":
        args.ref_iterations = args.ref_iterations or 64
        args.method_iterations = args.method_iterations or 16
        print(json.dumps(run_dense_quality_workload(args)))
        return
    if args.workload == "batch_quality":
        args.ref_iterations = args.ref_iterations or 192
        args.method_iterations = args.method_iterations or 24
        print(json.dumps(run_batch_quality_workload(args)))
        return
    args.res = (tuple(int(v) for v in args.res.lower().split("x")) if args.res
                else tuple(WORKLOADS[args.workload][0]))
    threads = os.cpu_count() or 1
    world, rank, _ = dist_env()
    if args.impl == "reference":
        if rank != 0:
            return
        # each step is one bounded iteration of the reference loop
        s2 = run_reference_sample(seconds=1e9, threads=threads, warmup=args.warmup, max_iters=args.steps,
                                  workload=args.workload)
        v = s2["value"]
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "paths/s", "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                          "config": {"workload": f"{args.workload} (reference CPU build; per step one iteration "
                                                 "of the sample in cpu_baseline.sample)"},
                          "cpu_baseline": s2, "e2e": {"value": v, "unit": "paths/s", "h2d_bytes_per_step": 0,
                                                      "d2h_bytes_per_step": 0}}))
        return
    out = run_b200(args)
    if out is None:
        return
    if not args.no_cpu_baseline and world == 1:
        try:
            out["cpu_baseline"] = run_reference_sample(args.cpu_seconds, threads, warmup=args.warmup,
                                                       workload=args.workload)
        except Exception as e:  # the oracle build is absent
            out["cpu_baseline"] = {"value": None, "unit": "paths/s", "cores": threads, "kind": "reference",
                                   "sample": f"unavailable: {e}"}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
