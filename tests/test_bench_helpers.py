"""CPU tests of the bench's accounting helpers and of the oracle's coverage
bound (the value the GPU's coverage debug tap is compared with)."""

import os
import sys
import types

import numpy as np

from conftest import ROOT

sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import bench  # noqa: E402
import oracle_py  # noqa: E402


def _stats(n, visible, drawn, group):
    return [types.SimpleNamespace(visible_count=visible, drawn_count=drawn, group=g)
            for g in group[:n]]


def test_batched_preprocess_bytes_reads_each_view_set_once():
    # scene 0: 20 views (18 in group 0, 2 in group 1), scene 1: 3 views in
    # group 1; sets of at most 16 consecutive views of one scene per group:
    # (scene 0, group 0) 16 + 2 views, (scene 0, group 1) 2, (scene 1, group 1) 3
    specs = [(0, None, 10, 10)] * 20 + [(1, None, 10, 10)] * 3
    stats = _stats(23, 50, 40, [0] * 18 + [1] * 5)
    scenes = [{"positions": np.zeros((100, 3))}, {"positions": np.zeros((60, 3))}]
    planes = 12
    writes = 23 * (50 * 16 + 40 * 48)
    shape = 50 * 32 + 40 * 16 * planes

    def set_bytes(n, views):
        return n * 16 + min(views * shape, n * (32 + 16 * planes))

    want = writes + set_bytes(100, 16) + set_bytes(100, 2) + set_bytes(100, 2) + set_bytes(60, 3)
    assert bench.batched_preprocess_bytes(specs, stats, scenes, planes) == want == 141280


def test_batched_preprocess_bytes_follows_render_order_by_scene():
    # views interleaved by scene render grouped by scene (stable): the same
    # sets as when the caller sorted them
    specs = [(k % 2, None, 8, 8) for k in range(8)]
    stats = _stats(8, 10, 5, [0] * 8)
    scenes = [{"positions": np.zeros((1000, 3))}, {"positions": np.zeros((500, 3))}]
    ordered = sorted(range(8), key=lambda v: specs[v][0])
    a = bench.batched_preprocess_bytes(specs, stats, scenes, 12)
    b = bench.batched_preprocess_bytes([specs[v] for v in ordered], [stats[v] for v in ordered],
                                       scenes, 12)
    assert a == b


def test_hbm_peak_falls_back_without_measured_peaks(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "PEAKS_FILE", str(tmp_path / "absent.json"))
    assert bench.hbm_peak_gbs() == (bench.FALLBACK_HBM_GBS, "fallback")
    p = tmp_path / "peaks.json"
    p.write_text('{"hbm_gbs": 7000.5}')
    monkeypatch.setattr(bench, "PEAKS_FILE", str(p))
    assert bench.hbm_peak_gbs() == (7000.5, "measured")


def test_nearest_rank():
    v = [5.0, 1.0, 3.0, 2.0, 4.0]
    assert bench.nearest_rank(v, 0.5) == 3.0
    assert bench.nearest_rank(v, 0.99) == 5.0
    assert bench.nearest_rank(v, 0.0) == 1.0


def test_oracle_coverage_bound_matches_the_float32_restatement():
    """oracle_py.coverage_bound (what the GPU tap is pinned to) equals the
    float32 bound of tests/test_coverage_bound.py bit for bit, including the
    cap at s^2 and the -1 of a non-positive bound."""
    rng = np.random.default_rng(5)
    s = rng.uniform(0.0, 1.0, 20000).astype(np.float32)
    log2a = rng.uniform(-9.0, 0.0, 20000).astype(np.float32)
    log2a[:5] = [-8.0, -8.5, 0.0, -1e-7, -7.9999995]
    got = oracle_py.coverage_bound(s, log2a)
    import test_coverage_bound as tcb
    want = tcb.coverage_bound(log2a, s * s)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert got[0] == -1.0 and got[1] == -1.0
    assert (got[log2a > -8.0] <= (s * s)[log2a > -8.0]).all()
