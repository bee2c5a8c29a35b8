"""Benchmark of the B200 SortedAlpha renderer: 1080p frames/s of the plain
one-frame path on the 279,199-splat SH-degree-3 synthetic scene.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

Under torchrun each rank renders its own replica of the workload on its GPU
(the per-frame path does not shard; no collective is used) and the reported
value is the whole-job frames/s from the max-over-ranks device time.

value: frames/s with the scene resident in HBM, device time of K frames
  measured with CUDA events on the renderer's stream; L2 is flushed (a
  256 MiB write) between frames, outside the timed spans.
e2e: the same frames through the public C ABI from host memory: camera upload,
  gsplat_context_render_frame_async and an asynchronous RGBA8 readback into
  pinned host memory every step (the copy of one frame overlaps the render
  of the next), host wall clock until the last image is on the host.
--impl reference: the reference's SortedAlpha frame restated on the host CPU
  (depth preprocess and 8-bit LSD radix sort on one thread, vertex stage and
  UNORM8 blending on every host thread), on the same workload.
"""

import argparse
import gc
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time
import types

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gsplat-rs_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

import gsplat_scenes  # noqa: E402

METRIC = "1080p frames/s @279k SH3"
WORKLOAD = "plain SortedAlpha frame: 279,199 synthetic splats, SH degree 3, 1920x1080, 16x16 tiles"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")


def bench_config(world):
    """The `config` both arms print, identical so that the two lines compare
    as one workload; per-arm details go in top-level keys."""
    return {"workload": WORKLOAD,
            "l2": "CUDA arm: flushed between frames (256 MiB write); CPU arm: not flushed",
            "parallelism": f"CUDA arm: one replica per GPU (x{world}), no collective on the "
                           "data path; CPU arm: host threads on rank 0"}
FALLBACK_HBM_GBS = 6650.0
# Per-launch counters of the 1080p raster (raster_fp32_kernel<16, 256>) from
# one ncu capture of this workload (profiles/frame_279k_sh3_1080p.md gives
# the command): DRAM bytes read + written, warp instructions issued, and
# executed FP32 thread operations (2 x FFMA + FADD + FMUL). None until
# captured for the current kernel.
# thread_flop: FP32 operations of one launch from the scalar build of the
# same arithmetic (-D GSR_RASTER_F32X2=0; ncu's per-op counters do not count
# the paired f32x2 instructions of the default build, which performs exactly
# the same operations).
NCU_RASTER = {"dram_bytes": 18_311_168, "warp_inst": 95_671_016,
              "thread_flop": 2 * 1_223_868_317 + 202_085_090 + 375_960_460,
              "source": "profiles/frame_279k_sh3_1080p.md (ncu --set full, one launch)"}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Replicas:
    """The replicas of a multi-GPU run (one process per GPU under torchrun,
    no data-path collective): a barrier around each timed region and the max
    of the ranks' times, over `backend` (nccl for the GPUs; gloo in the CPU
    tests). A single process needs no process group."""

    def __init__(self, world, rank, backend="nccl", device=None, timeout_s=120.0):
        self.world, self.rank = world, rank
        self.dist = None
        if world > 1:
            import datetime

            import torch.distributed as dist

            kw = {"device_id": device} if device is not None else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.dist = dist
            self.device = device

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, value):
        """The max over ranks of a per-rank time."""
        if not self.dist:
            return value
        import torch

        t = torch.tensor([value], dtype=torch.float64,
                         device=self.device if self.device is not None else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None


def whole_job_rate(world, units_per_rank, max_seconds):
    """Units all ranks processed per second of the slowest rank."""
    return world * units_per_rank / max_seconds


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 100 ms from before
    the warm-up until after the timed region; stop() keeps the samples whose
    timestamps fall inside the timed window (widened by one sampling period),
    or the nearest ones when the window is shorter than a period."""

    QUERY = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.window = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.out,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def mark(self, t0, t1):
        self.window = (t0, t1)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        self.proc.wait()
        self.out.flush()
        with open(self.out.name) as f:
            lines = [r for r in f.read().strip().splitlines() if r.strip()]
        os.unlink(self.out.name)
        import datetime

        samples = []
        for line in lines:
            r = [x.strip() for x in line.split(",")]
            try:
                ts = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                samples.append((ts, float(r[2]), float(r[3]), r[6:10]))
            except (ValueError, IndexError):
                continue
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sel, how = samples, "whole run"
        if self.window:
            t0, t1 = self.window
            sel = [x for x in samples if t0 - 0.1 <= x[0] <= t1 + 0.1]
            how = "timed window"
            if not sel:
                mid = 0.5 * (t0 + t1)
                sel = sorted(samples, key=lambda x: abs(x[0] - mid))[:3]
                how = "nearest to the timed window"
        reasons = set()
        for x in sel:
            for k, name in enumerate(self.REASONS):
                if k < len(x[3]) and x[3][k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median([x[1] for x in sel])), "sm_max_mhz": sel[0][2],
                "reasons": sorted(reasons), "samples": len(sel), "selection": how}


def algorithmic_bytes(phase, counts, n, planes, width, height, tile_passes):
    """Bytes each phase must move at minimum (reads + writes), per frame."""
    v, d, k = counts.visible, counts.drawn, counts.tile_keys
    if phase == "preprocess":
        return n * 16 + v * 32 + d * 16 * planes + v * 16 + d * 48
    if phase == "depth_sort":
        return v * 4 + 3 * v * 16  # histogram read + three non-trivial passes
    if phase == "emit":
        return v * 4 + v * 8 + k * 8
    if phase == "tile_sort":
        return k * 4 + tile_passes * k * 16
    if phase == "ranges":
        return k * 4
    if phase == "raster":
        return k * 52 + width * height * 4
    return 0


def batched_preprocess_bytes(specs, stats, scenes, planes, set_views=16):
    """Preprocess bytes of a batch at minimum: a view set (up to `set_views`
    consecutive views of one scene in a launch group, in render order: views
    sorted by scene, stable) reads its scene once: the 16-byte position of
    every splat, and the 32-byte shape and the SH planes of each splat some
    view of the set sees or draws (the per-view sums, capped at the scene);
    every view writes its own keys, ids, rects and records."""
    order = sorted(range(len(specs)), key=lambda v: specs[v][0])
    total = 0
    run = []

    def close(run):
        if not run:
            return 0
        n = scenes[specs[run[0]][0]]["positions"].shape[0]
        shape = sum(stats[v].visible_count * 32 + stats[v].drawn_count * 16 * planes for v in run)
        return n * 16 + min(shape, n * (32 + 16 * planes))

    for v in order:
        if run and (specs[v][0] != specs[run[0]][0] or stats[v].group != stats[run[0]].group
                    or len(run) == set_views):
            total += close(run)
            run = []
        run.append(v)
        total += stats[v].visible_count * 16 + stats[v].drawn_count * 48
    return total + close(run)


def image_errors(img, ref):
    """Per-pixel error of an RGBA8 image against a reference image, in UNORM8
    steps: max over channels, mean over RGB, fraction of pixels with any RGB
    channel more than 1/255 (and 3/255) off, and the reference's own image
    gate (mean |dRGB| <= 1/255 and <= 0.1% of pixels above 3/255,
    crates/gsplat-render-wgpu/src/lib.rs:3520-3537)."""
    d = np.abs(img.astype(np.int32) - ref.astype(np.int32))
    rgb = d[..., :3]
    over1 = float((rgb > 1).any(axis=-1).mean())
    over3 = float((rgb > 3).any(axis=-1).mean())
    mean_rgb = float(rgb.mean()) / 255.0
    return {"max_abs_steps": int(d.max(initial=0)), "max_abs_rgb": int(rgb.max(initial=0)),
            "mean_abs_rgb": mean_rgb, "frac_px_over_1_255": over1, "frac_px_over_3_255": over3,
            "reference_gate": bool(mean_rgb <= 1.0 / 255.0 and over3 <= 0.001)}


def nearest_rank(values, q):
    """Nearest-rank percentile (the reference bench-runner's definition,
    tools/bench-runner/src/main.rs:1051-1072)."""
    v = sorted(values)
    return float(v[max(0, int(math.ceil(q * len(v))) - 1)])


def _dist(values):
    return {"median": nearest_rank(values, 0.5), "p95": nearest_rank(values, 0.95),
            "mean": float(np.mean(values))}


def host_cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def lcg_keys(seed, n):
    """The reference sort tests' key generator (x = x * 1664525 + 1013904223,
    crates/gsplat-sort/src/lib.rs:597-612)."""
    out = np.empty(n, np.uint32)
    x = seed & 0xFFFFFFFF
    for i in range(n):
        x = (x * 1664525 + 1013904223) & 0xFFFFFFFF
        out[i] = x
    return out


def cpu_baseline(scene, cam, w, h, warmup=5, iters=30, gpu_images=None, gpu_projected=None):
    """The reference frame restated on the host (the oracle's C++ port of the
    CPU depth preprocess and radix sort on one thread, the vertex stage and
    UNORM8 blend on every host thread), per phase as median and p95 over
    `iters` frames after `warmup`, at the 16,384-splat SH0 256x256 workload
    and at the headline 279,199-splat SH3 1080p one; and the CPU radix sort
    on its own, on the reference's 200k-key microbenchmark input
    (crates/gsplat-sort/src/lib.rs:649-676) and on the 1080p frame's depth
    keys. gpu_images: {mode: RGBA8 image} rendered on the GPU for the headline
    camera; each is compared with the CPU frame's image (the reference image
    model) and with the FP64 evaluation of the same frame. gpu_projected: the
    GPU's per-splat vertex outputs for that camera (the debug tap), compared
    with a float64 evaluation of the reference's vertex stage."""
    import oracle_py

    threads = os.cpu_count() or 1
    per_config = {}
    ref_img = None
    sv2 = None
    c1 = gsplat_scenes.config1(seed=0)
    for name, (sc, cm, ww, hh) in (("config1_16k_sh0_256", c1),
                                   ("config2_279k_sh3_1080p", (scene, cam, w, h))):
        sv = oracle_py.SceneView(sc)
        for _ in range(warmup):
            img, _ = oracle_py.render_reference_frame(sv, cm, ww, hh, threads)
        rows = {k: [] for k in ("preprocess", "sort", "vertex", "raster", "total")}
        t0 = time.perf_counter()
        for _ in range(iters):
            img, t = oracle_py.render_reference_frame(sv, cm, ww, hh, threads)
            rows["preprocess"].append(t.preprocess_ms)
            rows["sort"].append(t.sort_ms)
            rows["vertex"].append(t.project_ms)
            rows["raster"].append(t.raster_ms)
            rows["total"].append(t.total_ms)
        el = time.perf_counter() - t0
        per_config[name] = {"frames_per_s": iters / el, "visible": int(t.visible),
                            "phases_ms": {k: _dist(v) for k, v in rows.items()}}
        if sc is scene:
            ref_img, sv2 = img, sv
    # the CPU radix sort alone (one thread)
    sort_alone = {}
    keys2, ids2 = oracle_py.preprocess_visible(sv2.pos.reshape(-1, 3), cam)
    for name, keys in (("reference_microbench_200k_lcg99", lcg_keys(99, 200_000)),
                       ("config2_depth_keys", keys2)):
        vals0 = np.arange(len(keys), dtype=np.uint32)
        for _ in range(warmup):
            oracle_py.sort_values_by_keys(keys, vals0)
        ms = []
        for _ in range(iters):
            t0 = time.perf_counter()
            oracle_py.sort_values_by_keys(keys, vals0)
            ms.append((time.perf_counter() - t0) * 1e3)
        sort_alone[name] = {"n": int(len(keys)), "ms": _dist(ms)}
    head = per_config["config2_279k_sh3_1080p"]
    out = {"value": head["frames_per_s"], "unit": "frames/s", "cores": threads, "kind": "port",
           "host_cpu": host_cpu_model(),
           "sample": f"{iters} full frames of each workload after {warmup} warm-up frames; depth "
                     f"preprocess and radix sort on 1 thread, vertex stage and UNORM8 blend on "
                     f"{threads} threads; value = frames/s of the 279,199-splat SH3 1080p frame",
           "per_config": per_config, "sort_alone": sort_alone}
    if gpu_images:
        fr = oracle_py.Frame(sv2, cam, w, h)
        f64, _ = fr.raster_f64(threads)
        out["gpu_image_errors"] = {
            mode: {"vs_reference_model": image_errors(img, ref_img),
                   "vs_fp64": image_errors(img, f64)} for mode, img in gpu_images.items()}
        out["gpu_image_errors"]["reference_model_vs_fp64"] = image_errors(ref_img, f64)
    if gpu_projected is not None:
        import oracle_f64

        out["gpu_vertex_errors_vs_fp64"] = oracle_f64.output_errors(
            gpu_projected, oracle_f64.project(scene, cam, w, h))
    return out


def run_reference(args, world, rank, budget_s=150.0):
    """Reference arm on rank 0: the CPU restatement of the reference frame.
    Each step is one frame; when K full frames would exceed the time budget,
    each step rasterises a band of rows and the frame time is scaled from it."""
    if rank != 0:
        return
    scene, cam, w, h = gsplat_scenes.config2()
    import oracle_py

    sv = oracle_py.SceneView(scene)
    threads = os.cpu_count() or 1
    _, t = oracle_py.render_reference_frame(sv, cam, w, h, threads)
    frac = min(1.0, budget_s / max(1e-9, (args.steps + args.warmup) * t.total_ms / 1000.0))
    rows = max(1, int(h * frac))
    for _ in range(args.warmup):
        oracle_py.render_reference_frame(sv, cam, w, h, threads, rows=rows)
    frame_ms = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _, t = oracle_py.render_reference_frame(sv, cam, w, h, threads, rows=rows)
        frame_ms.append(t.preprocess_ms + t.sort_ms + t.project_ms + t.raster_ms * h / rows)
    el = time.perf_counter() - t0
    value = 1000.0 * len(frame_ms) / sum(frame_ms)
    sample = ("one frame per step: the reference SortedAlpha path restated in C++ (oracle/): "
              f"depth preprocess and radix sort on 1 thread, vertex stage and UNORM8 blend on "
              f"{threads} threads")
    if rows < h:
        sample += f"; raster of rows 0-{rows} per step, frame time scaled by {h}/{rows}"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "frames/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(args.gpus),
            "cpu_baseline": {"value": value, "unit": "frames/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def measure_batched(ffi, torch, steps, warmup, cameras_per_scene=64):
    """Batched form on the multi-scene workload: 4 resident SH3 scenes
    (50k / 279,199 / 1M / 3M splats) x 64 seeded orbit cameras, resolutions
    mixed from {512^2, 720p, 1080p}; all 256 views per gsplat_batch_render
    call. Compared with the plain drop-in call, one gsplat_context_render_frame
    per view (one context per scene, views grouped by size so no context
    resizes between calls), on the same views and device."""
    scenes, views = gsplat_scenes.config4(cameras_per_scene=cameras_per_scene)
    specs = [(v["scene"], v["camera"], v["width"], v["height"]) for v in views]
    b = ffi.Batch()
    for s in scenes:
        b.add_scene(s)
    arr = ffi.Batch.make_views(specs)
    # launch shape from the autotuner, searched on every 8th view
    tune_views = ffi.Batch.make_views(specs[::8])
    tuned = b.autotune(tune_views, os.path.join(tempfile.gettempdir(), "gsplat_bench_tune.txt"),
                       reps=2)
    for _ in range(max(warmup, 2)):
        b.render(arr)
    dev, wall = [], []
    torch.cuda.nvtx.range_push("batched_timed")  # ncu --nvtx-include batched_timed/
    for _ in range(steps):
        t = b.render(arr)
        dev.append(t.device_ms)
        wall.append(t.wall_ms)
    torch.cuda.nvtx.range_pop()
    t = b.times()
    pixels = sum(w * h for _, _, w, h in specs)
    # e2e: cameras in, all images read back into pinned host memory
    pinned = torch.empty(pixels * 4, dtype=torch.uint8, pin_memory=True)
    out = pinned.numpy()
    offs = np.cumsum([0] + [w * h * 4 for _, _, w, h in specs])
    e2e = []
    for _ in range(steps):
        t0 = time.perf_counter()
        b.render(arr)
        for k in range(len(specs)):
            b.readback_rgba8(k, out[offs[k]:offs[k + 1]])
        e2e.append(time.perf_counter() - t0)
    # Per-phase device times of the same batch, group by group (a measurement
    # mode: each group waits for the one before, so no whole-batch graph),
    # against each phase's algorithmic bytes summed over the views.
    b.set_phase_timing(True)
    b.render(arr)
    b.render(arr)
    phase_ms = b.phase_times()
    b.set_phase_timing(False)
    stats = [b.view_stats(k) for k in range(len(specs))]
    group_tiles = {}
    for k, (sid, _, w, h) in enumerate(specs):
        g = stats[k].group
        group_tiles[g] = group_tiles.get(g, 0) + ((w + 15) // 16) * ((h + 15) // 16)
    group_passes = {}
    for g, tiles in group_tiles.items():
        p = 1
        while (1 << (8 * p)) < tiles:
            p += 1
        group_passes[g] = p
    hbm = hbm_peak_gbs()
    phases = {}
    for k, ms in phase_ms.items():
        if k == "preprocess":
            nbytes = batched_preprocess_bytes(specs, stats, scenes, 12)
        else:
            nbytes = 0
            for v, (sid, _, w, h) in enumerate(specs):
                st = stats[v]
                c = types.SimpleNamespace(visible=st.visible_count, drawn=st.drawn_count,
                                          tile_keys=st.tile_pairs)
                nbytes += algorithmic_bytes(k, c, scenes[sid]["positions"].shape[0], 12, w, h,
                                            group_passes[st.group])
        gbs = nbytes / (ms * 1e-3) / 1e9 if ms > 0 else None
        phases[k] = {"ms": ms, "bytes": nbytes, "gbs": gbs,
                     "frac_measured": gbs / hbm[0] if gbs else None}
    per_scene = []
    for sid in range(len(scenes)):
        sub = ffi.Batch.make_views([v for v in specs if v[0] == sid])
        # a batch per scene, on the same resident scenes
        b.render(sub)
        ms = [b.render(sub).device_ms for _ in range(2)]
        per_scene.append({"splats": int(scenes[sid]["positions"].shape[0]), "views": len(sub),
                          "batched_ms": float(np.median(ms))})
    b.close()

    # plain drop-in calls
    plain_dev = {sid: 0.0 for sid in range(len(scenes))}
    plain_wall = 0.0
    ctxs = []
    for sid, scene in enumerate(scenes):
        ctx = ffi.Context(512, 512)
        ctx.load_scene(scene)
        ctxs.append(ctx)
    order = sorted(range(len(specs)), key=lambda k: (specs[k][0], specs[k][2], specs[k][3]))
    for rep in range(2):  # first pass warms graphs and pair buffers
        plain_wall = 0.0
        plain_dev = {sid: 0.0 for sid in range(len(scenes))}
        for k in order:
            sid, cam, w, h = specs[k]
            ctx = ctxs[sid]
            if (ctx.width, ctx.height) != (w, h):
                ctx.set_size(w, h)
            ctx.set_camera(cam)
            t0 = time.perf_counter()
            ctx.render_frame()
            plain_wall += time.perf_counter() - t0
            plain_dev[sid] += sum(ctx.phase_times().values())
    for c in ctxs:
        c.close()
    for ps in per_scene:
        sid = per_scene.index(ps)
        ps["plain_ms"] = plain_dev[sid]
        ps["speedup"] = ps["plain_ms"] / ps["batched_ms"] if ps["batched_ms"] > 0 else None
    n = len(specs)
    batched_vps = n / (float(np.median(dev)) / 1000.0)
    plain_dev_total = sum(plain_dev.values())
    return {"workload": f"4 resident SH3 scenes (50k/279,199/1M/3M splats) x {cameras_per_scene} "
                        "orbit cameras, "
                        "resolutions mixed from 512^2/720p/1080p, 16x16 tiles",
            "views": n, "views_per_s": batched_vps,
            "ms_per_batch": float(np.median(dev)), "wall_ms_per_batch": float(np.median(wall)),
            "groups": t.groups, "kernel_launches": t.kernel_launches, "tile_pairs": int(t.tile_pairs),
            "autotune": {"tile": tuned.tile_size, "chunk": tuned.chunk,
                         "blocks_per_sm": tuned.blocks_per_sm, "candidates": tuned.candidates,
                         "from_cache": bool(tuned.from_cache),
                         "subset_best_ms": tuned.best_ms, "subset_default_ms": tuned.default_ms},
            "e2e_views_per_s": n / float(np.median(e2e)),
            "e2e_d2h_bytes": int(pixels * 4),
            "plain_views_per_s": n / (plain_dev_total / 1000.0),
            "plain_wall_views_per_s": n / plain_wall,
            "speedup_vs_plain": (n / (float(np.median(dev)) / 1000.0)) / (n / (plain_dev_total / 1000.0)),
            "per_scene": per_scene,
            "phases": phases, "phases_hbm_peak_gbs": hbm[0], "phases_hbm_peak_source": hbm[1],
            "phases_timing": "a separate phase-timed render of the same batch "
                             "(gsplat_batch_set_phase_timing): per-phase CUDA events of each "
                             "launch group, summed; groups run one by one",
            "timing": "device ms from CUDA events around all launch groups (batched) and the "
                      "per-phase CUDA events of each plain frame; scenes exceed L2"}


def _spin_until(t):
    while True:
        d = t - time.perf_counter()
        if d <= 0:
            return
        if d > 0.002:
            time.sleep(d - 0.001)


# Pipeline workspace the served section's lanes may admit per batch (over all
# lanes): batches stay a few dozen views, and the warm-up's extreme bursts take
# every lane to its largest workspace before any rate is timed.
SERVE_WORK_BUDGET = 16 << 30


def measure_served(ffi, rates, seconds, max_requests, lanes=2):
    """Served stream: 8 resident scenes (sizes log-uniform in [50k, 3M], SH
    degree 0-3 mixed), Poisson arrivals at each offered rate, each request a
    random scene, orbit camera and resolution from {512^2, 720p, 1080p}.
    Latency is submit -> RGBA8 image in host memory. The plain drop-in call
    serves the same arrival sequence one gsplat_context_render_frame +
    readback at a time, in arrival order (one context per scene and size,
    pinned readback buffers). Both paths are warmed up first."""
    import torch

    scenes = gsplat_scenes.config5_scenes()
    # 4 GiB of pinned result memory reserved up front: pinning on demand under
    # load stalls the request loop for tens of milliseconds per 64 MiB slab
    # (a host that cannot pin that much serves without the reserve)
    reserve_mib = 4096
    # requests still queued 50 ms after their submit are shed, so under
    # overload the requests that run keep a bounded queueing delay
    max_queue_ms = 50
    try:
        srv = ffi.Server(lanes=lanes, max_views=256, work_budget=SERVE_WORK_BUDGET,
                         result_pool_mib=reserve_mib, max_queue_ms=max_queue_ms)
    except ffi.GsplatError:
        reserve_mib = 0
        srv = ffi.Server(lanes=lanes, max_views=256, work_budget=SERVE_WORK_BUDGET,
                         max_queue_ms=max_queue_ms)
    for sc in scenes:
        srv.add_scene(sc)
    # The plain call gets its best case: one context per (scene, size), so no
    # context ever resizes, and pinned readback buffers.
    ctxs = {}
    for sid, sc in enumerate(scenes):
        for w, h in gsplat_scenes.RESOLUTIONS:
            ctx = ffi.Context(w, h)
            ctx.load_scene(sc)
            ctxs[(sid, w, h)] = ctx
    pinned = {(w, h): torch.empty(w * h * 4, dtype=torch.uint8, pin_memory=True).numpy()
              for w, h in gsplat_scenes.RESOLUTIONS}
    cam0 = gsplat_scenes.camera((0.0, 0.5, -5.0), (0, 0, 0), 50.0)
    for (sid, w, h), ctx in ctxs.items():
        ctx.set_camera(cam0)
        ctx.render_frame()
        ctx.readback_rgba8(pinned[(w, h)])
    # Server warm-up: two bursts of random requests grow the lanes'
    # workspaces, pair predictions and pinned result pools to steady state.
    for burst in range(2):
        warm = [srv.submit(r["scene"], r["camera"], r["width"], r["height"])
                for r in gsplat_scenes.config5_requests(900 + burst, 1e6, 256, len(scenes))]
        for rid in warm:
            srv.wait(rid)
            srv.release(rid)
    # Then the extremes an overloaded queue can hand a lane, twice each (the
    # lanes take batches in turn): full batches of the largest scene at
    # 1080p (splats, pairs), of the smallest at 1080p (tiles) and of the
    # largest at 512^2 (splats per pixel), so no workspace has to grow while
    # a rate is timed (growing maps gigabytes of device memory in the middle
    # of the request stream).
    sizes = [int(s["positions"].shape[0]) for s in scenes]
    big, small = sizes.index(max(sizes)), sizes.index(min(sizes))
    rng = np.random.default_rng(905)
    for sid, (w, h) in ((big, (1920, 1080)), (small, (1920, 1080)), (big, (512, 512))):
        for _ in range(2):
            warm = [srv.submit(sid, gsplat_scenes.orbit_camera(rng), w, h)
                    for _ in range(256)]
            for rid in warm:
                srv.wait(rid)
                srv.release(rid)
    # ... and single requests, one at a time, four times for every (scene,
    # size): a light load runs one-view batches, whose launch graphs a lane
    # captures on a layout's second run on that lane (a capture takes about
    # 3 ms of the scheduler's time), as a server in steady state has.
    for _ in range(4):
        for sid in range(len(scenes)):
            for w, h in gsplat_scenes.RESOLUTIONS:
                rid = srv.submit(sid, cam0, w, h)
                srv.wait(rid)
                srv.release(rid)
    out = []
    for rate in rates:
        count = int(min(max_requests, max(50, rate * seconds)))
        reqs = gsplat_scenes.config5_requests(int(rate), rate, count, len(scenes))
        srv.reset_stats()
        done = threading.Event()
        ids = []

        def consumer():
            k = 0
            while k < count:
                if k >= len(ids):
                    time.sleep(0.0002)
                    continue
                srv.wait(ids[k])
                srv.release(ids[k])
                k += 1
            done.set()

        # no garbage-collector pause inside the timed arrival streams (the
        # process holds the earlier sections' objects)
        gc.collect()
        gc.disable()
        th = threading.Thread(target=consumer)
        th.start()
        t0 = time.perf_counter()
        for r in reqs:
            _spin_until(t0 + r["arrival_s"])
            ids.append(srv.submit(r["scene"], r["camera"], r["width"], r["height"]))
        done.wait()
        th.join()
        st = srv.stats()
        # plain: one request at a time, in arrival order
        lat = []
        busy = 0.0
        t0 = time.perf_counter()
        for r in reqs:
            _spin_until(t0 + r["arrival_s"])
            ctx = ctxs[(r["scene"], r["width"], r["height"])]
            ts = time.perf_counter()
            ctx.set_camera(r["camera"])
            ctx.render_frame()
            ctx.readback_rgba8(pinned[(r["width"], r["height"])])
            te = time.perf_counter()
            busy += te - ts
            lat.append((te - (t0 + r["arrival_s"])) * 1000.0)
        plain_span = time.perf_counter() - t0
        gc.enable()
        lat = np.sort(np.array(lat))
        out.append({"offered_req_per_s": rate, "requests": count,
                    "views_per_s": st.views_per_s, "p50_ms": st.p50_ms, "p99_ms": st.p99_ms,
                    "shed": int(st.shed),
                    "mean_batch_views": st.mean_batch_views, "batches": int(st.batches),
                    "reruns": int(st.reruns), "peak_admitted_gb": st.peak_admitted_bytes / 1e9,
                    "device_ms": st.device_ms, "host_launch_ms": st.launch_ms,
                    "graph_captures": int(st.graph_captures), "capture_ms": st.capture_ms,
                    "pinned_slabs": int(st.pinned_slabs), "pinned_alloc_ms": st.pinned_alloc_ms,
                    "workspace_regrowths": int(st.workspace_regrowths),
                    "regrowth_ms": st.regrowth_ms,
                    "plain_views_per_s": count / plain_span,
                    "plain_capacity_views_per_s": count / busy,
                    "plain_p50_ms": float(lat[int(math.ceil(0.5 * len(lat))) - 1]),
                    "plain_p99_ms": float(lat[int(math.ceil(0.99 * len(lat))) - 1])})
    srv.close()
    for c in ctxs.values():
        c.close()
    return {"workload": "8 resident scenes, sizes log-uniform in [50k, 3M] splats, SH degree 0-3 "
                        "mixed; Poisson arrivals; each request a random scene, orbit camera and "
                        f"resolution from 512^2/720p/1080p; {lanes} lanes, <=256 views per batch, "
                        "16 GiB work budget",
            "result_pool_mib": reserve_mib, "max_queue_ms": max_queue_ms,
            "latency": "submit -> RGBA8 image in pinned host memory (host clock)",
            "rates": out}


def write_plain_artifact(args, ffi, ctx, scene, cams, out, w, h):
    """The plain frames as a benchmark artifact in the reference's v1 contract
    (manifest.json, frames.jsonl, summary.json under args.artifact): one frame
    per camera through the C ABI, per-frame host and device times."""
    import platform
    import uuid

    import bench_artifact

    run_id = "b200-plain-" + uuid.uuid4().hex[:12]
    started = bench_artifact.utc_now()
    for c in cams[:3]:
        ctx.set_camera(c)
        ctx.render_frame()
    m_start = bench_artifact.utc_now()
    frames = bench_artifact.record_frames(ctx, cams, out, run_id)
    m_end = bench_artifact.utc_now()
    commit, dirty = None, None
    try:
        commit = subprocess.run(["git", "-C", ROOT, "rev-parse", "HEAD"], capture_output=True,
                                text=True, check=True).stdout.strip() or None
        dirty = bool(subprocess.run(["git", "-C", ROOT, "status", "--porcelain"],
                                    capture_output=True, text=True, check=True).stdout.strip())
    except (OSError, subprocess.CalledProcessError):
        commit, dirty = None, None
    dev = ffi.device_info()
    driver = None
    try:
        driver = subprocess.run(["nvidia-smi", "--query-gpu=driver_version", "--format=csv,noheader"],
                                capture_output=True, text=True, check=True).stdout.strip().splitlines()[0]
    except (OSError, subprocess.CalledProcessError, IndexError):
        driver = None
    arrays = [np.ascontiguousarray(scene[k], np.float32) for k in
              ("positions", "opacity", "scale_xyz", "rotation_xyzw", "color_dc")]
    if scene.get("sh_rest") is not None:
        arrays.append(np.ascontiguousarray(scene["sh_rest"], np.float32))
    trace = np.array([[*c.position, *c.rotation_xyzw, c.vertical_fov_radians] for c in cams],
                     np.float32)
    unavailable = ["environment.browser"]
    if commit is None:
        unavailable.append("build.repository_commit")
    if dirty is None:
        unavailable.append("build.dirty")
    if driver is None:
        unavailable.append("environment.driver")
    manifest = {
        "run_id": run_id,
        "identity": {"series_id": "b200-plain-279k-sh3-1080p", "started_at_utc": started,
                     "ended_at_utc": bench_artifact.utc_now(),
                     "measurement_started_at_utc": m_start, "measurement_ended_at_utc": m_end},
        "build": {"repository_commit": commit, "dirty": dirty, "profile": "release",
                  "package_version": "0.1.0"},
        "dataset": {"id": "synthetic-279199-sh3-gmm-seed1",
                    "sha256": bench_artifact.sha256_of_arrays(arrays),
                    "bytes": int(sum(a.nbytes for a in arrays)),
                    "splat_count": int(scene["positions"].shape[0]),
                    "sh_degree": int(scene["sh_degree"])},
        "trace": {"id": "orbit-r4-yaw0.7-step0.002", "sha256": bench_artifact.sha256_of_arrays([trace])},
        "renderer": {"implementation": "gsplat-rs-b200-cuda", "path": "sorted_alpha_cuda_tiles",
                     "backend": "cuda-sm_100a", "sort_policy": "gpu_every_frame"},
        "display": {"width": w, "height": h, "dpr": 1.0, "refresh_hz": 60.0,
                    "frame_budget_ms": 1000.0 / 60.0, "refresh_hz_source": "configured",
                    "frame_budget_source": "configured"},
        "environment": {"platform": platform.machine(), "os": platform.platform(),
                        "device": dev["name"], "browser": None, "adapter": dev["name"],
                        "driver": driver},
        "timing": {"frame_wall_source": "host time of set_camera + gsplat_context_render_frame + "
                                        "RGBA8 readback into pinned memory (no presentation surface)",
                   "device_timings": "CUDA events on the renderer's stream"},
        "unavailable_fields": unavailable,
    }
    bench_artifact.write_artifact(args.artifact, manifest, frames, warmup_count=3,
                                  frame_budget_ms=1000.0 / 60.0)
    bench_artifact.validate(args.artifact)


def measure_ingest(ffi, splats=279_199, repeats=3):
    """PLY ingestion: a synthetic SH3 scene written as a binary PLY and loaded
    through gsplat_context_load_scene_path (body decoded on the device) and
    through the host path (gsplat_ply_load, host precompute, upload). The
    file is read once before timing (page cache warm); best of `repeats`."""
    rng = np.random.default_rng(11)
    scene = gsplat_scenes.make_scene(rng, gsplat_scenes.gmm_means(rng, splats), -4.5, 0.7, 0.5,
                                     1.5, 3)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "scene.ply")
        gsplat_scenes.write_ply(path, scene)
        size = os.path.getsize(path)
        with open(path, "rb") as f:
            while f.read(64 << 20):
                pass
        dev, host = [], []
        with ffi.Context(64, 64) as ctx:
            for _ in range(repeats):
                t0 = time.perf_counter()
                ctx.load_scene_path(path)
                dev.append(time.perf_counter() - t0)
            for _ in range(repeats):
                t0 = time.perf_counter()
                ctx.load_scene(ffi.ply_load(path))
                host.append(time.perf_counter() - t0)
    return {"workload": f"binary PLY, {splats} splats, SH degree 3, page cache warm",
            "file_bytes": size, "splats": splats,
            "device_ms": min(dev) * 1e3, "host_ms": min(host) * 1e3,
            "device_gbs": size / min(dev) / 1e9, "host_gbs": size / min(host) / 1e9,
            "speedup": min(host) / min(dev)}


def measure_packed(ffi, torch, frames=60):
    """The 1080p workload with its scene in the packed resident format (20-byte
    hot record + 48-byte SH sidecar, decoded by the preprocess kernel) against
    the plane format: per-phase device times (median over `frames`, L2 flushed
    between frames), bytes per splat, and the image difference."""
    scene, cam, w, h = gsplat_scenes.config2()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")
    out = {"workload": "1080p frame, 279,199 SH3 splats, scene in the plane vs the packed format",
           "bytes_per_splat": {"planes": 240, "packed": 68}}
    images = {}
    for fmt in ("planes", "packed"):
        with ffi.Context(w, h) as ctx:
            (ctx.load_scene if fmt == "planes" else ctx.load_scene_packed)(scene)
            ctx.set_camera(cam)
            for _ in range(5):
                ctx.render_frame()
            stream = torch.cuda.ExternalStream(ctx.stream())
            acc = {}
            for i in range(frames):
                with torch.cuda.stream(stream):
                    flush.fill_(i)
                ctx.render_frame()
                for k, v in ctx.phase_times().items():
                    acc.setdefault(k, []).append(v)
            images[fmt] = ctx.readback_rgba8().astype(np.int32)
            ph = {k: float(np.median(v)) for k, v in acc.items()}
            out[fmt] = {"phases_ms": ph, "frame_ms": sum(ph.values())}
    d = np.abs(images["planes"] - images["packed"])[..., :3] / 255.0
    out["image_mean_abs_diff"] = float(d.mean())
    out["image_frac_over_3"] = float((d > 3.0 / 255.0).any(axis=-1).mean())
    out["preprocess_speedup"] = (out["planes"]["phases_ms"]["preprocess"] /
                                 out["packed"]["phases_ms"]["preprocess"])
    return out


NOMINAL_HBM_GBS = 8000.0  # B200 HBM3e data-sheet bandwidth, for context beside the measured peak


def hbm_peak_gbs():
    """(HBM copy peak in GB/s, "measured" | "fallback")."""
    if os.path.exists(PEAKS_FILE):
        with open(PEAKS_FILE) as f:
            hbm = json.load(f).get("hbm_gbs")
        if hbm:
            return float(hbm), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def measure_config3(ffi, torch, frames=20):
    """The sort/raster stress frame: 3,000,000 SH3 splats (uniform 10^3 box
    plus a dense core), camera inside the volume, 3840x2160, 16x16 tiles.
    Per-phase device time (median over `frames`, L2 flushed between frames),
    achieved GB/s of each phase's algorithmic bytes against the measured HBM
    copy peak and the nominal 8 TB/s, in both blend modes."""
    scene, cam, w, h = gsplat_scenes.config3()
    peaks = {}
    if os.path.exists(PEAKS_FILE):
        with open(PEAKS_FILE) as f:
            peaks = json.load(f)
    hbm = peaks.get("hbm_gbs") or FALLBACK_HBM_GBS
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")
    n = scene["positions"].shape[0]
    tiles = ((w + 15) // 16) * ((h + 15) // 16)
    tile_passes = 1
    while (1 << (8 * tile_passes)) < tiles:
        tile_passes += 1
    out = {"workload": "3,000,000 synthetic splats, SH degree 3, uniform 10^3 box + dense core, "
                       "camera inside the volume, 3840x2160, 16x16 tiles",
           "hbm_peak_gbs": hbm, "hbm_peak_source": "measured" if peaks.get("hbm_gbs") else "fallback",
           "nominal_hbm_gbs": NOMINAL_HBM_GBS}
    with ffi.Context(w, h) as ctx:
        ctx.load_scene(scene)
        ctx.set_camera(cam)
        for blend, name in ((0, "fp32"), (1, "unorm8")):
            ctx.set_blend_mode(blend)
            for _ in range(3):
                ctx.render_frame()
            counts = ctx.frame_counts()
            stream = torch.cuda.ExternalStream(ctx.stream())
            acc = {}
            for i in range(frames):
                with torch.cuda.stream(stream):
                    flush.fill_(i)
                ctx.render_frame()
                for k, v in ctx.phase_times().items():
                    acc.setdefault(k, []).append(v)
            ph = {k: float(np.median(v)) for k, v in acc.items()}
            phases = {}
            for k, ms in ph.items():
                b = algorithmic_bytes(k, counts, n, 12, w, h, tile_passes)
                gbs = b / (ms * 1e-3) / 1e9 if ms > 0 else None
                phases[k] = {"ms": ms, "bytes": b, "gbs": gbs,
                             "frac_measured": gbs / hbm if gbs else None,
                             "frac_nominal": gbs / NOMINAL_HBM_GBS if gbs else None}
            ps = ["preprocess", "depth_sort", "emit", "tile_sort"]
            ps_bytes = sum(phases[k]["bytes"] for k in ps)
            ps_ms = sum(phases[k]["ms"] for k in ps)
            out[name] = {"frame_ms": sum(ph.values()), "frames_per_s": 1000.0 / sum(ph.values()),
                         "visible": int(counts.visible), "drawn": int(counts.drawn),
                         "tile_pairs": int(counts.tile_keys), "phases": phases,
                         "preprocess_emit_sort_gbs": ps_bytes / (ps_ms * 1e-3) / 1e9,
                         "preprocess_emit_sort_frac_measured":
                             ps_bytes / (ps_ms * 1e-3) / 1e9 / hbm}
    return out


def run_sections_only(args, ffi, torch):
    """The batched and/or served sections alone (no plain-frame line), for
    profiling those workloads by themselves."""
    out = {"metric": METRIC, "sections": args.only}
    if "batched" in args.only:
        out["batched"] = measure_batched(ffi, torch, args.batch_steps, args.warmup,
                                         args.cameras_per_scene)
    if "served" in args.only:
        out["served"] = measure_served(ffi, [float(x) for x in args.serve_rates.split(",")],
                                       args.serve_seconds, 4000, args.serve_lanes)
    if "ingest" in args.only:
        out["ingest"] = measure_ingest(ffi, args.ingest_splats)
    if "packed" in args.only:
        out["packed"] = measure_packed(ffi, torch)
    if "config3" in args.only:
        out["config3"] = measure_config3(ffi, torch)
    print(json.dumps(out), flush=True)


def run_cuda(args, world, rank, local):
    import torch

    import gsplat_ffi as ffi

    torch.cuda.set_device(local)
    if args.only:
        run_sections_only(args, ffi, torch)
        return
    replicas = Replicas(world, rank, "nccl", torch.device("cuda", local))
    scene, cam, w, h = gsplat_scenes.config2()
    clocks = ClockSampler(local)
    clocks.start()
    ctx = ffi.Context(w, h)
    ctx.load_scene(scene)
    ctx.set_camera(cam)
    for _ in range(max(args.warmup, 3)):
        ctx.render_frame()
    counts = ctx.frame_counts()
    stream = torch.cuda.ExternalStream(ctx.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")

    # Per-phase device times (separate untimed loop, L2 flushed before each frame).
    phase_acc = {}
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(i)
        ctx.render_frame()
        for k, v in ctx.phase_times().items():
            phase_acc[k] = phase_acc.get(k, 0.0) + v
    phases = {k: v / args.steps for k, v in phase_acc.items()}

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    replicas.barrier()
    torch.cuda.synchronize()
    t_begin = time.time()
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(i + 1)
            starts[i].record(stream)
        ctx.render_frame_async()
        with torch.cuda.stream(stream):
            ends[i].record(stream)
    ctx.sync()
    torch.cuda.synchronize()
    clocks.mark(t_begin, time.time())
    device_ms = replicas.max(sum(s.elapsed_time(e) for s, e in zip(starts, ends)))
    replicas.barrier()
    ms_per_frame = device_ms / args.steps
    value = whole_job_rate(world, args.steps, device_ms / 1000.0)
    img_fp32 = ctx.readback_rgba8().copy()

    # The UNORM8 parity mode (the reference's per-splat UNORM8 rounding,
    # bit-exact with the oracle's reference image model) on the same frames.
    ctx.set_blend_mode(1)
    for _ in range(max(args.warmup, 3)):
        ctx.render_frame()
    parity_phase = {}
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(i)
        ctx.render_frame()
        for k, v in ctx.phase_times().items():
            parity_phase[k] = parity_phase.get(k, 0.0) + v
    replicas.barrier()
    torch.cuda.synchronize()
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(i + 1)
            starts[i].record(stream)
        ctx.render_frame_async()
        with torch.cuda.stream(stream):
            ends[i].record(stream)
    ctx.sync()
    torch.cuda.synchronize()
    parity_ms = replicas.max(sum(s.elapsed_time(e) for s, e in zip(starts, ends)))
    img_unorm8 = ctx.readback_rgba8().copy()
    ctx.set_blend_mode(0)
    ctx.render_frame()
    parity = {"value": whole_job_rate(world, args.steps, parity_ms / 1000.0), "unit": "frames/s",
              "ms_per_step": parity_ms / args.steps,
              "phases_ms": {k: v / args.steps for k, v in parity_phase.items()},
              "blend": "UNORM8 after every splat, back to front (the reference image model)"}

    # End to end through the C ABI: camera in, frame, RGBA8 readback to pinned
    # memory every step. Frames are enqueued back to back and each image is
    # read back asynchronously while later frames render. With frame lanes
    # (gsplat_context_set_frame_lanes) consecutive frames also overlap on the
    # device, each on its own stream and workspace; one lane is measured too.
    cams = []
    for i in range(args.steps):
        yaw = 0.7 + 0.002 * i
        cams.append(ffi.GsplatCamera.from_dict(gsplat_scenes.camera(
            (4.0 * math.sin(yaw), 0.5, -4.0 * math.cos(yaw)), (0, 0, 0), 45.0)))

    def e2e_run(lanes):
        ctx.set_frame_lanes(lanes)
        pinned = [torch.empty(w * h * 4, dtype=torch.uint8, pin_memory=True)
                  for _ in range(max(2, lanes))]
        outs = [p.numpy() for p in pinned]
        for i in range(max(args.warmup, 3) * lanes):  # every lane captures its graph
            ctx.set_camera(cams[i % len(cams)])
            ctx.render_frame_async()
            ctx.readback_rgba8_async(outs[i % len(outs)])
        ctx.sync()
        replicas.barrier()
        t0 = time.perf_counter()
        for i in range(args.steps):
            ctx.set_camera(cams[i])
            ctx.render_frame_async()
            ctx.readback_rgba8_async(outs[i % len(outs)])
        ctx.sync()
        el = replicas.max(time.perf_counter() - t0)
        return el, outs[(args.steps - 1) % len(outs)]

    e2e_single_s, _ = e2e_run(1)
    e2e_s, out = e2e_run(args.frame_lanes)
    ctx.set_frame_lanes(1)
    if args.artifact and rank == 0:
        write_plain_artifact(args, ffi, ctx, scene, cams, out, w, h)
    clk = clocks.stop()
    e2e = {"value": whole_job_rate(world, args.steps, e2e_s), "unit": "frames/s",
           "h2d_bytes_per_step": 40, "d2h_bytes_per_step": w * h * 4 + 64,
           "frame_lanes": args.frame_lanes,
           "single_lane_value": whole_job_rate(world, args.steps, e2e_single_s)}

    tiles = ((w + 15) // 16) * ((h + 15) // 16)
    tile_passes = 2 if tiles > 256 else 1
    planes = 12
    dominant = max(phases, key=phases.get)
    peaks = {}
    if os.path.exists(PEAKS_FILE):
        with open(PEAKS_FILE) as f:
            peaks = json.load(f)
    hbm = peaks.get("hbm_gbs")
    bytes_dom = algorithmic_bytes(dominant, counts, scene["positions"].shape[0], planes, w, h,
                                  tile_passes)
    achieved = bytes_dom / (phases[dominant] * 1e-3) / 1e9
    peak = hbm if hbm else FALLBACK_HBM_GBS
    roofline = {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                "peak_source": "measured" if hbm else "fallback",
                "algorithmic_bytes": bytes_dom}
    if dominant == "raster":
        # The raster's limiter is FP32 issue, not HBM: its records and ids
        # stay in L2. Issue rate = warp instructions per launch (ncu) over the
        # live launch time, against 4 schedulers x SMs x the live SM clock;
        # FP32 rate = executed FP32 operations (ncu) over the live launch
        # time, against this device's measured FMA throughput.
        raster_s = phases["raster"] * 1e-3
        sms = ffi.device_info()["sm_count"]
        fp32_peak, _ = ffi.measure_fp32_peak()
        roofline["limiter"] = "fp32_issue"
        roofline["fp32_peak_tflops"] = fp32_peak
        roofline["fp32_peak_source"] = "measured (FMA-only kernel, gsplat_cuda_measure_fp32_peak)"
        if NCU_RASTER:
            roofline["traffic"] = NCU_RASTER["dram_bytes"]
            roofline["issue_inst_per_launch"] = NCU_RASTER["warp_inst"]
            roofline["fp32_flop_per_launch"] = NCU_RASTER["thread_flop"]
            roofline["fp32_tflops"] = NCU_RASTER["thread_flop"] / raster_s / 1e12
            roofline["fp32_frac"] = roofline["fp32_tflops"] / fp32_peak
            roofline["counters_source"] = NCU_RASTER["source"]
    phase_rooflines = {}
    for k, ms in phases.items():
        b = algorithmic_bytes(k, counts, scene["positions"].shape[0], planes, w, h, tile_passes)
        phase_rooflines[k] = {"ms": ms, "bytes": b, "gbs": b / (ms * 1e-3) / 1e9 if ms > 0 else None}

    # scratch zeroing; preprocess; depth sort: plan + 4 passes (histograms
    # from K1); emit; tile sort: plan + passes (histograms from K2); ranges;
    # raster
    launches_per_frame = 1 + 1 + (1 + 4) + 1 + (1 + tile_passes) + 1 + 1
    line = {"metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_frame,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": bench_config(world),
            "frame_counts": {"visible": int(counts.visible), "drawn": int(counts.drawn),
                             "tile_pairs": int(counts.tile_keys)},
            "e2e": e2e, "gpu_launches": launches_per_frame * args.steps, "clocks": clk,
            "roofline": roofline, "phases": phase_rooflines, "parity_mode": parity}
    if roofline.get("issue_inst_per_launch") and clk.get("sm_mhz"):
        issue_peak = ffi.device_info()["sm_count"] * 4 * clk["sm_mhz"] * 1e6
        roofline["issue_frac"] = (roofline["issue_inst_per_launch"] /
                                  (phases["raster"] * 1e-3) / issue_peak)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the GPU's per-splat outputs of the same frame, from a context with
        # the debug tap on (outside every timed region)
        with ffi.Context(w, h) as dbg:
            dbg.set_debug_taps(True)
            dbg.load_scene(scene)
            dbg.set_camera(cam)
            dbg.render_frame()
            projected = dbg.debug_projected()
        line["cpu_baseline"] = cpu_baseline(scene, cam, w, h, iters=args.cpu_iters,
                                            gpu_images={"fp32": img_fp32, "unorm8": img_unorm8},
                                            gpu_projected=projected)
    ctx.close()
    if not args.no_batched and world == 1:
        line["batched"] = measure_batched(ffi, torch, args.batch_steps, 2)
    if not args.no_served and world == 1:
        line["served"] = measure_served(ffi, [float(x) for x in args.serve_rates.split(",")],
                                        args.serve_seconds, 4000, args.serve_lanes)
    if not args.no_ingest and world == 1:
        line["ingest"] = measure_ingest(ffi, args.ingest_splats)
    if not args.no_packed and world == 1:
        line["packed"] = measure_packed(ffi, torch)
    if not args.no_config3 and world == 1:
        line["config3"] = measure_config3(ffi, torch)
    replicas.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["cuda", "reference"], default="cuda")
    ap.add_argument("--cpu-iters", type=int, default=30,
                    help="timed CPU-baseline frames per workload (after 5 warm-up frames)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-steps", type=int, default=3)
    ap.add_argument("--cameras-per-scene", type=int, default=64,
                    help="batched workload cameras per scene (64 is the headline workload)")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--serve-rates", default="500,2000,8000,20000")
    ap.add_argument("--serve-seconds", type=float, default=1.0)
    ap.add_argument("--serve-lanes", type=int, default=2,
                    help="server lanes (gsplat_server_create's lanes)")
    ap.add_argument("--artifact", default="",
                    help="also write the plain frames as a v1 benchmark artifact into this folder")
    ap.add_argument("--no-ingest", action="store_true")
    ap.add_argument("--no-packed", action="store_true")
    ap.add_argument("--no-config3", action="store_true")
    ap.add_argument("--frame-lanes", type=int, default=8,
                    help="frame lanes of the e2e loop (gsplat_context_set_frame_lanes)")
    ap.add_argument("--ingest-splats", type=int, default=279_199,
                    help="splats of the PLY ingestion workload")
    ap.add_argument("--only", default="",
                    help="comma list of batched,served,ingest,packed,config3: run just those "
                         "sections")
    args = ap.parse_args()
    args.only = [x for x in args.only.split(",") if x]
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_cuda(args, world, rank, local)


if __name__ == "__main__":
    main()
