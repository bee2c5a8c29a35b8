"""Deterministic benchmark-artifact fixture: a fixed manifest and ten
synthetic frames (two with unobservable timings) written by the product's
producer (gsplat-rs_b200/bench_artifact.py). make_golden.py writes it to
tests/golden/artifact_v1/ and checks it with the reference's own v1
validator; tests/test_bench_artifact.py regenerates it and compares byte for
byte."""

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "gsplat-rs_b200"))

import bench_artifact  # noqa: E402

RUN_ID = "fixture-b200-plain-0001"


def manifest():
    return {
        "run_id": RUN_ID,
        "identity": {"series_id": "fixture-series",
                     "started_at_utc": "2026-12-01T00:00:00Z",
                     "ended_at_utc": "2026-12-01T00:00:02Z",
                     "measurement_started_at_utc": "2026-12-01T00:00:00.500Z",
                     "measurement_ended_at_utc": "2026-12-01T00:00:01.500Z"},
        "build": {"repository_commit": None, "dirty": None, "profile": "release",
                  "package_version": "0.1.0"},
        "dataset": {"id": "synthetic-fixture", "sha256": "0" * 64, "bytes": 1024,
                    "splat_count": 4, "sh_degree": 0},
        "trace": {"id": "static", "sha256": "1" * 64},
        "renderer": {"implementation": "gsplat-rs-b200-cuda", "path": "sorted_alpha_cuda_tiles",
                     "backend": "cuda-sm_100a", "sort_policy": "gpu_every_frame"},
        "display": {"width": 256, "height": 256, "dpr": 1.0, "refresh_hz": 60.0,
                    "frame_budget_ms": 1.0, "refresh_hz_source": "configured",
                    "frame_budget_source": "configured"},
        "environment": {"platform": "fixture", "os": "fixture-os", "device": "fixture-gpu",
                        "browser": None, "adapter": "fixture-gpu", "driver": None},
        "timing": {"frame_wall_source": "fixture: synthetic values"},
        "unavailable_fields": ["build.repository_commit", "build.dirty", "environment.browser",
                               "environment.driver"],
    }


def frames():
    out = []
    for k in range(10):
        call = 0.40 + 0.037 * ((k * 7) % 10)
        wall = call + 0.25 + (0.9 if k == 6 else 0.0)
        unobserved = k in (3, 8)
        out.append(bench_artifact.frame_record(
            RUN_ID, k, 1_000_000 * (k + 1), call, wall, visible=4, drawn=4,
            preprocess_ms=None if unobserved else 0.03 + 0.001 * k,
            sort_ms=None if unobserved else 0.11 + 0.002 * k,
            gpu_complete_ms=None if unobserved else 0.38 + 0.003 * k))
    return out


def write(directory):
    bench_artifact.write_artifact(directory, manifest(), frames(), warmup_count=3,
                                  frame_budget_ms=1.0)
