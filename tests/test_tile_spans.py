"""Exact tile-row spans of the pair emission (CPU oracle only): every tile a
splat's pixels can receive weight in is emitted, the spans lie inside the
tile rect, and the FP32 tile raster is unchanged by dropping the rest."""

import math

import numpy as np
import pytest

import gsplat_scenes


def _hard_scene(seed, n=3000):
    """Near-camera splats with extreme anisotropy, alphas just above the
    1/256 threshold, large and tiny extents."""
    rng = np.random.default_rng(seed)
    pos = np.stack([rng.uniform(-2.5, 2.5, n), rng.uniform(-1.5, 1.5, n),
                    rng.uniform(0.3, 6.0, n)], axis=1).astype(np.float32)
    logit_floor = math.log((1.0 / 256.0) / (1.0 - 1.0 / 256.0))
    opacity = np.where(rng.random(n) < 0.4, logit_floor + rng.uniform(1e-4, 0.05, n),
                       rng.normal(0.0, 2.0, n)).astype(np.float32)
    base = rng.uniform(-5.0, -0.5, (n, 1))
    spread = rng.uniform(0.0, 4.5, (n, 3)) * (rng.random((n, 3)) < 0.7)
    scale = (base - spread).astype(np.float32)
    q = rng.normal(size=(n, 4)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return {"positions": pos, "opacity": opacity, "scale_xyz": scale, "rotation_xyzw": q,
            "color_dc": rng.normal(0.0, 0.5, (n, 3)).astype(np.float32), "sh_degree": 0,
            "sh_rest": None}


def _reached_tiles(fr, s):
    """Tiles holding a pixel where splat s can carry weight, in f64 with a
    slack of 1e-5 on every threshold (far above the FP32 raster's rounding)."""
    p, r = fr.proj[s], fr.rec[s]
    t = fr.tile
    x0, x1 = int(p["tile_x0"]) * t, min(int(p["tile_x1"]) * t, fr.width)
    y0, y1 = int(p["tile_y0"]) * t, min(int(p["tile_y1"]) * t, fr.height)
    px, py = np.meshgrid(np.arange(x0, x1, dtype=np.float64),
                         np.arange(y0, y1, dtype=np.float64))
    dx, dy = px - float(r["cx"]), py - float(r["cy"])
    lx = float(r["ax"]) * dx + float(r["ay"]) * dy
    ly = float(r["bx"]) * dx + float(r["by"]) * dy
    sv = float(r["s"]) * (1 + 1e-5)
    r2 = lx * lx + ly * ly
    hit = (np.abs(lx) <= sv) & (np.abs(ly) <= sv) & (r2 <= 1 + 1e-5)
    hit &= float(r["alpha"]) * np.exp(-4.5 * r2) > (1.0 / 256.0) * (1 - 1e-5)
    ty, tx = (py[hit] // t).astype(np.int64), (px[hit] // t).astype(np.int64)
    return set((ty * fr.tiles_x + tx).tolist())


CASES = [("config1", 0, 16), ("config1", 1, 8), ("hard", 2, 16), ("hard", 3, 8)]


def _frame(oracle, kind, seed, tile, exact=True):
    if kind == "config1":
        scene, cam, w, h = gsplat_scenes.config1(seed=seed)
    else:
        scene, w, h = _hard_scene(seed), 320, 200
        cam = gsplat_scenes.default_camera()
    sv = oracle.SceneView(scene)
    return sv, cam, w, h, oracle.Frame(sv, cam, w, h, tile=tile, exact=exact)


@pytest.mark.parametrize("kind,seed,tile", CASES)
def test_spans_cover_every_reached_pixel(oracle, kind, seed, tile):
    sv, cam, w, h, fr = _frame(oracle, kind, seed, tile)
    emitted = {}
    for t_, i in zip(fr.pair_tiles.tolist(), fr.pair_ids.tolist()):
        emitted.setdefault(i, set()).add(t_)
    drawn = np.nonzero(fr.proj["flags"] & 2)[0]
    checked = 0
    for s in drawn.tolist():
        p = fr.proj[s]
        if p["tile_x1"] <= p["tile_x0"] or p["tile_y1"] <= p["tile_y0"]:
            assert s not in emitted
            continue
        got = emitted.get(s, set())
        rect = {ty * fr.tiles_x + tx for ty in range(p["tile_y0"], p["tile_y1"])
                for tx in range(p["tile_x0"], p["tile_x1"])}
        assert got <= rect, s
        missing = _reached_tiles(fr, s) - got
        assert not missing, (s, sorted(missing))
        checked += 1
    assert checked > 100


@pytest.mark.parametrize("kind,seed,tile", CASES)
def test_spans_keep_the_fp32_image(oracle, kind, seed, tile):
    sv, cam, w, h, fr = _frame(oracle, kind, seed, tile)
    whole = oracle.Frame(sv, cam, w, h, tile=tile, exact=False)
    assert len(fr.pair_tiles) < len(whole.pair_tiles)
    assert np.array_equal(fr.raster_tiles_fp32(), whole.raster_tiles_fp32())
    # per tile, the exact list is the whole-rect list with entries removed
    for t in range(fr.num_tiles):
        a = fr.tile_ids[fr.ranges[t, 0]:fr.ranges[t, 1]]
        b = whole.tile_ids[whole.ranges[t, 0]:whole.ranges[t, 1]]
        assert np.array_equal(a, b[np.isin(b, a)]), t
