"""Benchmark artifacts in the reference's v1 contract (tests/perf/
benchmark-artifact-v1.md in the reference): the producer regenerates the
golden fixture byte for byte (the fixture was accepted by the reference's own
validator when it was made), the project's validator accepts it, and planted
contract violations are rejected."""

import json
import os
import shutil
import sys

import pytest

from conftest import GOLDEN

sys.path.insert(0, GOLDEN)

import artifact_fixture  # noqa: E402
import bench_artifact  # noqa: E402

FILES = ("manifest.json", "frames.jsonl", "summary.json")


def test_producer_reproduces_golden_artifact(tmp_path):
    artifact_fixture.write(str(tmp_path))
    for name in FILES:
        with open(os.path.join(GOLDEN, "artifact_v1", name), "rb") as a, \
                open(tmp_path / name, "rb") as b:
            assert a.read() == b.read(), name
    info = bench_artifact.validate(str(tmp_path))
    assert info["frames"] == 10


def test_summary_rules():
    d = bench_artifact.distribution([5.0, 1.0, None, 3.0, 2.0, 4.0])
    assert d["count"] == 5 and d["mean"] == 3.0
    assert (d["p50"], d["p90"], d["p95"], d["p99"], d["max"]) == (3.0, 5.0, 5.0, 5.0, 5.0)
    assert bench_artifact.distribution([None, None]) is None
    man = json.load(open(os.path.join(GOLDEN, "artifact_v1", "manifest.json")))
    # frames 3 and 8 have no device timings: their paths are listed
    for m in ("preprocess_ms", "sort_ms", "gpu_complete_ms", "geometry_submit_ms", "gpu_wait_ms"):
        assert f"frames[*].{m}" in man["unavailable_fields"]
    summ = json.load(open(os.path.join(GOLDEN, "artifact_v1", "summary.json")))
    assert summ["missed_frame_count"] == 1  # frame 6 exceeds the 1 ms budget
    assert summ["distributions"]["gpu_wait_ms"] is None


def _mutated(tmp_path, name, edit):
    d = tmp_path / "art"
    shutil.copytree(os.path.join(GOLDEN, "artifact_v1"), d)
    path = d / name
    if name == "frames.jsonl":
        lines = [json.loads(x) for x in path.read_text().splitlines() if x.strip()]
        edit(lines)
        path.write_text("".join(json.dumps(x) + "\n" for x in lines))
    else:
        obj = json.loads(path.read_text())
        edit(obj)
        path.write_text(json.dumps(obj))
    return str(d)


@pytest.mark.parametrize("name,edit,msg", [
    ("summary.json", lambda s: s.update(missed_frame_count=0), "missed_frame_count"),
    ("summary.json", lambda s: s["distributions"]["call_ms"].update(p99=1.0), "call_ms.p99"),
    ("frames.jsonl", lambda f: f[2].update(call_ms=None), "call_ms is required"),
    ("frames.jsonl", lambda f: f[4].update(frame_index=7), "contiguous"),
    ("frames.jsonl", lambda f: f[5].update(elapsed_ns=1), "monotonic"),
    ("manifest.json", lambda m: m["unavailable_fields"].remove("frames[*].sort_ms"), "sort_ms"),
    ("manifest.json", lambda m: m["dataset"].update(sha256="XYZ"), "sha256"),
    ("manifest.json", lambda m: m["build"].update(repository_commit=None) or
     m["unavailable_fields"].remove("build.repository_commit"), "repository_commit"),
])
def test_planted_violations_are_rejected(tmp_path, name, edit, msg):
    d = _mutated(tmp_path, name, edit)
    with pytest.raises(bench_artifact.ArtifactError) as e:
        bench_artifact.validate(d)
    assert msg in str(e.value)
