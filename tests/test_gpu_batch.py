"""GPU tests of the batched form: many views over several resident scenes of
uneven sizes in one call. Every view's image must equal, bit for bit, the
plain one-frame render of the same scene, camera and size (the per-tile
lists of a view are the same in the shared (view, tile, depth) key space),
whatever the launch grouping, pair-buffer re-runs, tile size or blend mode;
per-view counts must equal the oracle's."""

import numpy as np
import pytest

import gsplat_ffi as ffi
import gsplat_scenes
from conftest import assert_fp32_image

pytestmark = pytest.mark.gpu

SIZES = [(256, 256), (320, 200), (400, 300), (97, 61)]


def _scenes():
    rng = np.random.default_rng(77)
    small = gsplat_scenes.make_scene(rng, gsplat_scenes.gmm_means(rng, 3000), -3.5, 0.6, 0.5, 1.5, 1)
    mid, _, _, _ = gsplat_scenes.config1(seed=8)
    big = gsplat_scenes.make_scene(rng, gsplat_scenes.gmm_means(rng, 20000), -4.2, 0.6, 0.5, 1.5, 3)
    return [small, mid, big]


def _views(rng, count, nscenes):
    out = []
    for k in range(count):
        cam = gsplat_scenes.orbit_camera(rng, (3.0, 7.0))
        w, h = SIZES[k % len(SIZES)]
        out.append((int(rng.integers(nscenes)), cam, w, h))
    return out


def _plain(scene, cam, w, h, tile=16, blend=0):
    ctx = ffi.Context(w, h)
    ctx.set_tile_size(tile)
    ctx.set_blend_mode(blend)
    ctx.load_scene(scene)
    ctx.set_camera(cam)
    ctx.render_frame()
    return ctx


def _check_against_plain(batch, scenes, views, tile=16, blend=0, oracle=None):
    for k, (sid, cam, w, h) in enumerate(views):
        ctx = _plain(scenes[sid], cam, w, h, tile, blend)
        img = batch.readback_rgba8(k)
        assert np.array_equal(img, ctx.readback_rgba8()), f"view {k}"
        st = batch.view_stats(k)
        counts = ctx.frame_counts()
        assert st.visible_count == counts.visible and st.drawn_count == counts.drawn
        assert st.tile_pairs == counts.tile_keys
        if oracle is not None and k < 3:
            fr = oracle.Frame(oracle.SceneView(scenes[sid]), cam, w, h, tile=tile)
            assert st.visible_count == fr.visible and st.tile_pairs == len(fr.pair_tiles)
            if blend == 0:
                assert_fp32_image(img, fr.raster_tiles_fp32(), f"view {k} vs oracle")
            else:
                assert np.array_equal(img, fr.raster_unorm8()), f"view {k} vs oracle"


def test_batch_views_equal_plain_frames(oracle):
    scenes = _scenes()
    rng = np.random.default_rng(1)
    views = _views(rng, 14, len(scenes))
    with ffi.Batch() as b:
        ids = [b.add_scene(s) for s in scenes]
        assert ids == [0, 1, 2]
        t = b.render(views)
        assert t.groups == 1 and t.kernel_launches > 0 and t.device_ms > 0
        _check_against_plain(b, scenes, views, oracle=oracle)
        # a second call with other cameras reuses the workspace (graph replay
        # where the layout repeats) and stays exact
        views2 = _views(rng, 14, len(scenes))
        b.render(views2)
        _check_against_plain(b, scenes, views2)
        assert sum(b.view_stats(k).tile_pairs for k in range(14)) == b.times().tile_pairs


def test_batch_grouping_and_pair_reruns():
    scenes = _scenes()
    rng = np.random.default_rng(2)
    # Large splats close to the camera: far more pairs per splat than the
    # first prediction, so groups overflow and are re-run with larger buffers.
    r2 = np.random.default_rng(9)
    means = r2.uniform(-2, 2, (3000, 3)).astype(np.float32)
    scenes.append(gsplat_scenes.make_scene(r2, means, -0.5, 0.3, 2.0, 0.5, 0))
    views = _views(rng, 10, len(scenes))
    views += [(3, gsplat_scenes.camera((0.0, 0.0, -3.0), (0, 0, 0), 70.0), 640, 480)]
    with ffi.Batch() as b:
        for s in scenes:
            b.add_scene(s)
        b.set_limits(max_views=3)
        b.set_tile_size(8)
        t = b.render(views)
        assert t.groups == 4
        assert t.reruns >= 1
        groups = [b.view_stats(k).group for k in range(len(views))]
        # views are grouped by scene, then split in render order
        assert sorted(set(groups)) == [0, 1, 2, 3]
        assert all(groups.count(g) <= 3 for g in range(4))
        _check_against_plain(b, scenes, views, tile=8)
        t = b.render(views)  # predictions learned: no re-run the second time
        assert t.reruns == 0
        _check_against_plain(b, scenes, views, tile=8)


def test_batch_phase_timing():
    """Phase-timed renders run group by group and report per-phase device
    times summed over the groups; the images stay those of the whole-batch
    graph."""
    scenes = _scenes()
    views = _views(np.random.default_rng(31), 9, len(scenes))
    with ffi.Batch() as b:
        for s in scenes:
            b.add_scene(s)
        b.set_limits(max_views=4)
        b.render(views)
        t = b.render(views)
        assert t.groups == 3 and t.graph_launches == 1
        assert all(v == 0.0 for v in b.phase_times().values())
        ref = [b.readback_rgba8(k).copy() for k in range(len(views))]
        b.set_phase_timing(True)
        b.render(views)
        t = b.render(views)
        assert t.graph_launches == 0
        ph = b.phase_times()
        assert list(ph) == ["preprocess", "depth_sort", "emit", "tile_sort", "ranges", "raster"]
        assert all(v > 0.0 for v in ph.values()), ph
        assert sum(ph.values()) <= t.device_ms * 1.01 + 0.05
        for k in range(len(views)):
            assert np.array_equal(b.readback_rgba8(k), ref[k]), f"view {k}"
        b.set_phase_timing(False)
        t = b.render(views)
        assert t.graph_launches == 1
        assert all(v == 0.0 for v in b.phase_times().values())


@pytest.mark.parametrize("tile,blend", [(8, 0), (16, 1)])
def test_batch_tile_size_and_blend_mode(oracle, tile, blend):
    scenes = _scenes()
    rng = np.random.default_rng(3 + tile)
    views = _views(rng, 6, len(scenes))
    with ffi.Batch() as b:
        for s in scenes:
            b.add_scene(s)
        b.set_tile_size(tile)
        b.set_blend_mode(blend)
        b.render(views)
        _check_against_plain(b, scenes, views, tile, blend, oracle=oracle)


def test_batch_more_than_one_launch_of_views():
    """More views than one launch group holds (1024): split, still exact."""
    scenes = _scenes()[:2]
    rng = np.random.default_rng(4)
    views = []
    for k in range(1100):
        cam = gsplat_scenes.orbit_camera(rng, (3.0, 7.0))
        views.append((k % 2, cam, 48, 32))
    with ffi.Batch() as b:
        for s in scenes:
            b.add_scene(s)
        t = b.render(views)
        assert t.groups == 2
        pick = [0, 1, 511, 1023, 1024, 1099]
        for k in pick:
            sid, cam, w, h = views[k]
            ctx = _plain(scenes[sid], cam, w, h)
            assert np.array_equal(b.readback_rgba8(k), ctx.readback_rgba8()), k


def test_batch_errors():
    scenes = _scenes()
    with ffi.Batch() as b:
        b.add_scene(scenes[0])
        cam = gsplat_scenes.default_camera()
        with pytest.raises(ffi.GsplatError) as e:
            b.render([(5, cam, 32, 32)])
        assert e.value.code == ffi.INVALID_ARGUMENT and "unknown scene" in e.value.message
        arr = b.make_views([(0, cam, 32, 32)])
        arr[0].reserved = 1
        with pytest.raises(ffi.GsplatError) as e:
            b.render(arr)
        assert e.value.code == ffi.INVALID_ARGUMENT
        with pytest.raises(ffi.GsplatError) as e:
            b.render([(0, dict(cam, near_plane=5.0, far_plane=1.0), 32, 32)])
        assert e.value.code == ffi.INVALID_ARGUMENT
        with pytest.raises(ffi.GsplatError) as e:
            b.readback_rgba8(0)
        assert e.value.code == ffi.INVALID_ARGUMENT
        b.set_scene_budget(1 << 20)
        with pytest.raises(ffi.GsplatError) as e:
            b.add_scene(scenes[2])
        assert e.value.code == ffi.UNSUPPORTED and "budget" in e.value.message
        with pytest.raises(ffi.GsplatError) as e:
            b.set_limits(max_views=2000)
        assert e.value.code == ffi.INVALID_ARGUMENT


def test_batch_autotune_and_cache(tmp_path):
    scenes = _scenes()
    rng = np.random.default_rng(21)
    views = _views(rng, 8, len(scenes))
    cache = str(tmp_path / "tune.txt")
    with ffi.Batch() as b:
        for s in scenes:
            b.add_scene(s)
        b.render(views)
        before = [b.readback_rgba8(k).copy() for k in range(len(views))]
        r = b.autotune(views, cache, reps=1)
        assert r.candidates == 15 and not r.from_cache
        assert 0 < r.best_ms <= r.default_ms * 1.0001
        assert r.tile_size in (8, 16)
        b.render(views)
        for k in range(len(views)):
            assert np.array_equal(b.readback_rgba8(k), before[k]), k
        text = open(cache).read().splitlines()
        assert text[0] == "gsplat-cuda-autotune v1" and len(text) == 2
        assert "|blend0|" in text[1]
    with ffi.Batch() as b:
        for s in scenes:
            b.add_scene(s)
        r2 = b.autotune(views, cache)
        assert r2.from_cache and r2.candidates == 0
        assert (r2.tile_size, r2.chunk, r2.blocks_per_sm) == (r.tile_size, r.chunk, r.blocks_per_sm)
        b.render(views)
        for k in range(len(views)):
            assert np.array_equal(b.readback_rgba8(k), before[k]), k


@pytest.mark.parametrize("count", [1, 8, 9])
def test_view_table_inline_and_copied_over_graph_replays(count):
    """Runs of up to 8 views carry the view table in the first kernel's
    parameters (a replayed graph gets each run's table by a node update),
    larger runs copy it to the device: over repeated runs of one layout (the
    same scenes and sizes, so the graph is captured and replayed) with new
    cameras each time, every view equals its plain render."""
    scenes = _scenes()
    rng = np.random.default_rng(40 + count)
    layout = [(k % len(scenes), SIZES[k % len(SIZES)]) for k in range(count)]
    with ffi.Batch() as b:
        for s in scenes:
            b.add_scene(s)
        for _ in range(4):
            views = [(sid, gsplat_scenes.orbit_camera(rng, (3.0, 7.0)), w, h)
                     for sid, (w, h) in layout]
            b.render(views)
            _check_against_plain(b, scenes, views)


def test_whole_batch_is_one_graph_and_stays_exact():
    """A batch split into several launch groups runs directly the first time
    its layout is seen and as one CUDA graph (every group captured back to
    back, each group's view table a captured copy from the pinned staging
    area) once the layout repeats and the pair buffers have settled; every
    view stays equal to the plain render."""
    scenes = _scenes()
    rng = np.random.default_rng(12)
    first = _views(rng, 13, len(scenes))
    first.sort(key=lambda v: v[0])
    later = [(sid, gsplat_scenes.orbit_camera(rng, (3.0, 7.0)), w, h) for sid, _, w, h in first]
    with ffi.Batch() as b:
        for s in scenes:
            b.add_scene(s)
        b.set_limits(max_views=5, max_pairs=1 << 28, max_splats=1 << 28, max_tiles=1 << 24)
        launches = []
        for call in range(6):
            views = first if call == 0 else later  # one layout, new cameras after the first
            t = b.render(views)
            assert t.groups > 1
            launches.append(t.graph_launches)
            _check_against_plain(b, scenes, views)
        assert launches[0] == 0 and all(x == 1 for x in launches[2:]), launches
