"""Benchmark artifacts in the reference's v1 contract (schema
`gsplat-benchmark/v1`, tests/perf/benchmark-artifact-v1.md): a run directory
with manifest.json, frames.jsonl and summary.json, so frame series measured
on a B200 can be read by the same tooling as the reference's own runs.

Producer side: `frame_record` builds one frame line, `write_artifact` writes
the three files (summary distributions by nearest-rank percentiles and a
left-to-right f64 mean, missed frames against the frame budget). `validate`
checks a directory against the contract's rules; it is this project's own
statement of those rules (tools/bench-runner/src/artifact.rs and
tests/perf/validate-benchmark-artifacts.py in the reference enforce the same
contract).

Mapping of this renderer's frame onto the contract's fields:
  call_ms             host time of gsplat_context_render_frame
  frame_wall_ms       host time of set_camera + render_frame + RGBA8 readback
                      into pinned memory (there is no presentation surface;
                      manifest timing.frame_wall_source says so)
  preprocess_ms       device time of the preprocess kernel (CUDA events)
  sort_ms             device time of depth sort + pair emission + tile sort +
                      tile ranges
  gpu_complete_ms     device time of the whole frame (all phases)
  geometry_submit_ms  null: the scene is resident, no geometry is submitted
  gpu_wait_ms         null: the call waits inside the library
  sort_refreshed      whether the frame sorted its depth order (always, unless
                      a sort interval is set on the context)
"""

import hashlib
import json
import math
import os
import time

SCHEMA = "gsplat-benchmark/v1"
METRICS = ("call_ms", "frame_wall_ms", "preprocess_ms", "sort_ms", "geometry_submit_ms",
           "gpu_wait_ms", "gpu_complete_ms")
REQUIRED_TIMINGS = ("call_ms", "frame_wall_ms")


class ArtifactError(ValueError):
    pass


def frame_record(run_id, index, elapsed_ns, call_ms, frame_wall_ms, visible, drawn,
                 preprocess_ms=None, sort_ms=None, gpu_complete_ms=None, geometry_submit_ms=None,
                 gpu_wait_ms=None, sort_refreshed=True):
    return {"schema": SCHEMA, "record_type": "frame", "run_id": run_id, "frame_index": int(index),
            "elapsed_ns": int(elapsed_ns), "call_ms": float(call_ms),
            "frame_wall_ms": float(frame_wall_ms),
            "preprocess_ms": None if preprocess_ms is None else float(preprocess_ms),
            "sort_ms": None if sort_ms is None else float(sort_ms),
            "geometry_submit_ms": None if geometry_submit_ms is None else float(geometry_submit_ms),
            "gpu_wait_ms": None if gpu_wait_ms is None else float(gpu_wait_ms),
            "gpu_complete_ms": None if gpu_complete_ms is None else float(gpu_complete_ms),
            "visible": int(visible), "drawn": int(drawn), "sort_refreshed": sort_refreshed}


def percentile(values, fraction):
    """Nearest rank: sorted ascending, index max(ceil(p * n) - 1, 0)."""
    ordered = sorted(values)
    return ordered[max(math.ceil(fraction * len(ordered)) - 1, 0)]


def distribution(values):
    """None when no value is available; else count, mean (left-to-right f64
    sum in frame order, then one division) and nearest-rank percentiles."""
    vals = [v for v in values if v is not None]
    if not vals:
        return None
    total = 0.0
    for v in vals:
        total += v
    return {"count": len(vals), "mean": total / len(vals), "p50": percentile(vals, 0.50),
            "p90": percentile(vals, 0.90), "p95": percentile(vals, 0.95),
            "p99": percentile(vals, 0.99), "max": max(vals)}


def unavailable_frame_fields(frames):
    """frames[*].<metric> paths of the timings some frame could not observe."""
    out = []
    for m in METRICS:
        if any(f[m] is None for f in frames):
            out.append(f"frames[*].{m}")
    if any(f.get("sort_refreshed") is None for f in frames):
        out.append("frames[*].sort_refreshed")
    return out


def write_artifact(directory, manifest, frames, warmup_count, frame_budget_ms):
    """Writes manifest.json, frames.jsonl and summary.json. `manifest` holds
    the identity/build/dataset/trace/renderer/display/environment objects and
    may list unavailable fields; frame-level unavailable fields are added."""
    if not frames:
        raise ArtifactError("an artifact needs at least one frame")
    run_id = manifest["run_id"]
    man = dict(manifest)
    man["schema"] = SCHEMA
    man["record_type"] = "manifest"
    unavailable = list(man.get("unavailable_fields", []))
    for path in unavailable_frame_fields(frames):
        if path not in unavailable:
            unavailable.append(path)
    man["unavailable_fields"] = unavailable
    summary = {"schema": SCHEMA, "record_type": "summary", "run_id": run_id,
               "sample_count": len(frames), "warmup_count": int(warmup_count),
               "frame_budget_ms": float(frame_budget_ms),
               "missed_frame_count": sum(1 for f in frames if f["frame_wall_ms"] > frame_budget_ms),
               "distributions": {m: distribution([f[m] for f in frames]) for m in METRICS}}
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "manifest.json"), "w") as fh:
        json.dump(man, fh, indent=2, allow_nan=False)
        fh.write("\n")
    with open(os.path.join(directory, "frames.jsonl"), "w") as fh:
        for f in frames:
            fh.write(json.dumps(f, allow_nan=False) + "\n")
    with open(os.path.join(directory, "summary.json"), "w") as fh:
        json.dump(summary, fh, indent=2, allow_nan=False)
        fh.write("\n")


def _need(cond, message):
    if not cond:
        raise ArtifactError(message)


def _is_num(v):
    return isinstance(v, (int, float)) and not isinstance(v, bool) and math.isfinite(v)


def validate(directory):
    """Checks a v1 run directory: headers and run ids, the manifest's required
    objects and nullability rules, contiguous frames with monotonic time,
    unavailable timings listed, and summary counts and distributions (1e-9)."""
    def load(name):
        with open(os.path.join(directory, name)) as fh:
            return json.load(fh)

    man = load("manifest.json")
    _need(man.get("schema") == SCHEMA and man.get("record_type") == "manifest", "manifest header")
    run_id = man.get("run_id")
    _need(isinstance(run_id, str) and run_id, "run_id must be a non-empty string")
    for key in ("identity", "build", "dataset", "trace", "renderer", "display", "environment"):
        _need(isinstance(man.get(key), dict), f"manifest.{key} must be an object")
    unavailable = man.get("unavailable_fields")
    _need(isinstance(unavailable, list) and all(isinstance(u, str) and u for u in unavailable),
          "unavailable_fields must list non-empty strings")
    for key in ("series_id", "started_at_utc", "ended_at_utc", "measurement_started_at_utc",
                "measurement_ended_at_utc"):
        _need(isinstance(man["identity"].get(key), str) and man["identity"][key], f"identity.{key}")
    b = man["build"]
    for key in ("repository_commit", "dirty"):
        if b.get(key) is None:
            _need(f"build.{key}" in unavailable, f"null build.{key} must be listed as unavailable")
    for key in ("profile", "package_version"):
        _need(isinstance(b.get(key), str) and b[key], f"build.{key}")
    ds = man["dataset"]
    for key in ("bytes", "splat_count", "sh_degree"):
        _need(isinstance(ds.get(key), int) and ds[key] >= 0, f"dataset.{key}")
    for obj, name in ((ds, "dataset"), (man["trace"], "trace")):
        sha = obj.get("sha256")
        _need(isinstance(sha, str) and len(sha) == 64 and all(c in "0123456789abcdef" for c in sha),
              f"{name}.sha256 must be lowercase SHA-256")
    for key in ("implementation", "path", "backend", "sort_policy"):
        _need(isinstance(man["renderer"].get(key), str) and man["renderer"][key], f"renderer.{key}")
    d = man["display"]
    for key in ("width", "height"):
        _need(isinstance(d.get(key), int) and d[key] > 0, f"display.{key}")
    for key in ("dpr", "refresh_hz", "frame_budget_ms"):
        _need(_is_num(d.get(key)) and d[key] > 0, f"display.{key}")
    env = man["environment"]
    for key in ("device", "browser", "adapter", "driver"):
        _need(key in env and (env[key] is None or isinstance(env[key], str)), f"environment.{key}")

    frames = []
    with open(os.path.join(directory, "frames.jsonl")) as fh:
        for line in fh:
            if not line.strip():
                continue
            f = json.loads(line)
            _need(f.get("schema") == SCHEMA and f.get("record_type") == "frame" and
                  f.get("run_id") == run_id, "frame header")
            _need(f.get("frame_index") == len(frames), "frame_index must be contiguous from zero")
            for m in METRICS:
                v = f.get(m)
                if v is None:
                    _need(m not in REQUIRED_TIMINGS, f"{m} is required")
                    _need(f"frames[*].{m}" in unavailable, f"null {m} must be listed as unavailable")
                else:
                    _need(_is_num(v) and v >= 0, f"{m} must be a finite non-negative number")
            for key in ("visible", "drawn", "elapsed_ns"):
                _need(isinstance(f.get(key), int) and f[key] >= 0, f"{key}")
            _need(f.get("sort_refreshed") is None or isinstance(f["sort_refreshed"], bool),
                  "sort_refreshed must be boolean or null")
            _need(not frames or f["elapsed_ns"] >= frames[-1]["elapsed_ns"], "elapsed_ns monotonic")
            frames.append(f)
    _need(frames, "at least one frame")

    s = load("summary.json")
    _need(s.get("schema") == SCHEMA and s.get("record_type") == "summary" and
          s.get("run_id") == run_id, "summary header")
    _need(s.get("sample_count") == len(frames), "sample_count")
    _need(isinstance(s.get("warmup_count"), int), "warmup_count")
    budget = s.get("frame_budget_ms")
    _need(_is_num(budget) and budget > 0, "frame_budget_ms")
    _need(s.get("missed_frame_count") == sum(1 for f in frames if f["frame_wall_ms"] > budget),
          "missed_frame_count")
    dist = s.get("distributions")
    _need(isinstance(dist, dict), "distributions")
    for m in METRICS:
        want = distribution([f[m] for f in frames])
        got = dist.get(m)
        if want is None:
            _need(got is None, f"distributions.{m} must be null")
            continue
        _need(isinstance(got, dict) and got.get("count") == want["count"], f"distributions.{m}.count")
        for key in ("mean", "p50", "p90", "p95", "p99", "max"):
            _need(_is_num(got.get(key)) and abs(got[key] - want[key]) <= 1e-9,
                  f"distributions.{m}.{key}")
    return {"frames": len(frames), "run_id": run_id}


def record_frames(ctx, cameras, out, run_id, t_origin_ns=None):
    """Renders one frame per camera through the C ABI (gsplat_ffi.Context)
    and returns the v1 frame records; `out` receives each RGBA8 readback
    (pinned memory keeps the copy asynchronous-capable and fast)."""
    frames = []
    t0 = time.perf_counter_ns() if t_origin_ns is None else t_origin_ns
    for k, cam in enumerate(cameras):
        ts = time.perf_counter_ns()
        ctx.set_camera(cam)
        tc = time.perf_counter_ns()
        ctx.render_frame()
        tr = time.perf_counter_ns()
        ctx.readback_rgba8(out)
        te = time.perf_counter_ns()
        st = ctx.stats()
        ph = ctx.phase_times()
        frames.append(frame_record(
            run_id, k, te - t0, (tr - tc) / 1e6, (te - ts) / 1e6, st.visible_count,
            st.drawn_count, preprocess_ms=ph["preprocess"],
            sort_ms=ph["depth_sort"] + ph["emit"] + ph["tile_sort"] + ph["ranges"],
            gpu_complete_ms=sum(ph.values()),
            sort_refreshed=bool(ctx.frame_counts().sort_refreshed)))
    return frames


def sha256_of_arrays(arrays):
    h = hashlib.sha256()
    for a in arrays:
        if a is not None:
            h.update(memoryview(a).cast("B"))
    return h.hexdigest()


def utc_now():
    return time.strftime("%Y-%m-%dT%H:%M:%S", time.gmtime()) + "Z"
