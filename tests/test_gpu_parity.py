"""GPU parity of the CUDA SortedAlpha path against the CPU oracle, through the
C ABI. Integer and index work (visible order, tile pairs, tile ranges) must be
bit-exact; the projected records and the UNORM8 compositing mode are also
expected bit-exact because the kernels and the oracle run the same f32
operation sequence. The FP32 image equals the oracle's FP32 tile model up to
rare single steps (the raster's weight uses the hardware base-2 exponential,
the model a polynomial), and is held to the reference's own image parity
gate against the UNORM8 reference model and to <= 2/255 against the FP64
evaluation."""

import math
import os
import subprocess

import numpy as np
import pytest

import gsplat_ffi as ffi
import gsplat_scenes
from conftest import GOLDEN, ROOT, assert_fp32_image, lcg_seq

pytestmark = pytest.mark.gpu


def _ctx(w, h):
    return ffi.Context(w, h)


def _render(scene, cam, w, h, blend=0, tile=16, debug=True):
    ctx = _ctx(w, h)
    ctx.set_debug_taps(debug)
    ctx.set_blend_mode(blend)
    ctx.set_tile_size(tile)
    ctx.load_scene(scene)
    ctx.set_camera(cam)
    ctx.render_frame()
    return ctx


def _norm_ranges(r):
    """Empty tiles carry no position; compare them as (0, 0)."""
    r = np.array(r, np.uint32).copy()
    r[r[:, 0] == r[:, 1]] = 0
    return r


def _compare_stages(ctx, fr, sv):
    order = ctx.debug_order()
    assert np.array_equal(order, fr.order), "depth order"
    proj = ctx.debug_projected()
    assert proj.shape[0] == sv.n
    vis = (fr.proj["flags"] & 1) != 0
    assert np.array_equal(proj["flags"], fr.proj["flags"])
    assert np.array_equal(proj["depth"][vis].view(np.uint32), fr.proj["depth"][vis].view(np.uint32))
    drawn = (fr.proj["flags"] & 2) != 0
    for f in ("center_ndc", "axis_u", "axis_v", "color", "extent_scale"):
        a = proj[f][drawn].view(np.uint32)
        b = fr.proj[f][drawn].view(np.uint32)
        assert np.array_equal(a, b), f
    for f in ("tile_x0", "tile_y0", "tile_x1", "tile_y1"):
        assert np.array_equal(proj[f][drawn], fr.proj[f][drawn]), f
    tiles, ids = ctx.debug_tile_pairs()
    assert np.array_equal(tiles, fr.pair_tiles) and np.array_equal(ids, fr.pair_ids), "pairs"
    ranges, sorted_ids = ctx.debug_tile_ranges(fr.num_tiles)
    assert np.array_equal(_norm_ranges(ranges), _norm_ranges(fr.ranges)), "ranges"
    assert np.array_equal(sorted_ids, fr.tile_ids), "tile lists"
    counts = ctx.frame_counts()
    assert counts.visible == fr.visible and counts.drawn == fr.drawn
    assert counts.tile_keys == len(fr.pair_tiles)


def _image_metrics(img, ref8, ref64):
    d8 = np.abs(img.astype(np.int32) - ref8.astype(np.int32))
    d64 = np.abs(img.astype(np.int32) - ref64.astype(np.int32))
    rgb = d8[..., :3] / 255.0
    return {"mean_abs_rgb_vs_unorm8": float(rgb.mean()),
            "frac_over_3_255_vs_unorm8": float((rgb > 3.0 / 255.0).any(axis=-1).mean()),
            "max_vs_unorm8": int(d8.max()), "max_vs_f64": int(d64.max()),
            "mean_vs_f64": float(d64.mean() / 255.0)}


@pytest.mark.parametrize("cfg", ["config1", "config2_small"])
def test_frame_parity_stages_and_images(oracle, cfg):
    if cfg == "config1":
        scene, cam, w, h = gsplat_scenes.config1(seed=0)
    else:
        scene, cam, w, h = gsplat_scenes.config2(seed=11, n=40000)
        w, h = 960, 540
    sv = oracle.SceneView(scene)
    fr = oracle.Frame(sv, cam, w, h)
    ctx = _render(scene, cam, w, h, blend=0)
    _compare_stages(ctx, fr, sv)
    img32 = ctx.readback_rgba8()
    assert_fp32_image(img32, fr.raster_tiles_fp32(), "fp32 image vs restatement")
    ref8 = fr.raster_unorm8()
    ref64, _ = fr.raster_f64()
    m = _image_metrics(img32, ref8, ref64)
    print(cfg, m)
    assert m["mean_abs_rgb_vs_unorm8"] <= 1.0 / 255.0
    assert m["frac_over_3_255_vs_unorm8"] <= 0.001
    assert m["max_vs_f64"] <= 2
    ctx.set_blend_mode(1)
    ctx.render_frame()
    img8 = ctx.readback_rgba8()
    assert np.array_equal(img8, ref8), "unorm8 parity image vs reference model"
    ctx.close()


@pytest.mark.parametrize("cfg", ["config1", "config2_small"])
def test_raster_coverage_bound_tap(oracle, cfg):
    """The FP32 raster's own per-splat coverage bound, read through the debug
    tap, equals the oracle's bound of the same inputs bit for bit; its
    log2 alpha (the hardware logarithm) is within 4e-6 of numpy's; only splats
    in some tile list carry a value (not all of them: a tile stops staging
    chunks once every pixel is opaque)."""
    if cfg == "config1":
        scene, cam, w, h = gsplat_scenes.config1(seed=0)
    else:
        scene, cam, w, h = gsplat_scenes.config2(seed=11, n=40000)
        w, h = 960, 540
    ctx = _render(scene, cam, w, h, blend=0)
    cov = ctx.debug_coverage()
    proj = ctx.debug_projected()
    _, ids = ctx.debug_tile_pairs()
    listed = np.zeros(len(cov), bool)
    listed[np.unique(ids)] = True
    has = ~np.isnan(cov[:, 1])
    assert not (has & ~listed).any()
    assert has.sum() > 0.5 * listed.sum() and has.sum() > 100
    want = oracle.coverage_bound(proj["extent_scale"][has], cov[has, 0])
    assert np.array_equal(cov[has, 1].view(np.uint32), want.view(np.uint32))
    alpha = proj["color"][has, 3].astype(np.float64)
    assert np.abs(cov[has, 0] - np.log2(alpha)).max() <= 4e-6
    # the UNORM8 mode leaves the tap empty
    ctx.set_blend_mode(1)
    ctx.render_frame()
    assert np.isnan(ctx.debug_coverage()[:, 1]).all()
    ctx.close()


def test_full_config2_parity(oracle):
    """279,199 splats, SH3, 1920x1080: every stage bit-exact at full size (the
    FP32 image within its tolerance)."""
    import oracle_f64

    scene, cam, w, h = gsplat_scenes.config2()
    sv = oracle.SceneView(scene)
    fr = oracle.Frame(sv, cam, w, h)
    ctx = _render(scene, cam, w, h)
    _compare_stages(ctx, fr, sv)
    # the GPU's per-splat outputs against the float64 evaluation
    e = oracle_f64.output_errors(ctx.debug_projected(), oracle_f64.project(scene, cam, w, h))
    print("config2 vertex outputs vs fp64", e)
    assert e["drawn_disagree"] <= max(2, 1e-4 * e["drawn_both"])
    assert e["center_ndc"]["max_abs"] <= 2e-6 and e["color"]["max_abs"] <= 1e-6
    assert e["conic"]["mean_rel"] <= 2e-6 and e["conic"]["p999_rel"] <= 1e-4
    img = ctx.readback_rgba8()
    assert_fp32_image(img, fr.raster_tiles_fp32())
    ref8 = fr.raster_unorm8()
    ref64, _ = fr.raster_f64()
    m = _image_metrics(img, ref8, ref64)
    print("config2", m, "visible", fr.visible, "pairs", len(fr.pair_tiles))
    assert m["mean_abs_rgb_vs_unorm8"] <= 1.0 / 255.0
    assert m["frac_over_3_255_vs_unorm8"] <= 0.001
    assert m["max_vs_f64"] <= 2
    st = ctx.stats()
    assert st.visible_count == fr.visible and st.drawn_count == fr.visible
    # the UNORM8 parity mode: the reference image model, bit for bit
    ctx.set_blend_mode(1)
    ctx.render_frame()
    assert np.array_equal(ctx.readback_rgba8(), ref8), "unorm8 parity image vs reference model"
    ctx.close()


def test_conformance_minimal_ascii(kats):
    k = kats["conformance"]
    w, h = k["size"]
    for blend in (0, 1):
        ctx = _ctx(w, h)
        ctx.set_blend_mode(blend)
        ctx.load_scene_path(os.path.join(GOLDEN, "minimal_ascii.ply"))
        ctx.set_camera(ffi.lib().gsplat_camera_default())
        ctx.render_frame()
        st = ctx.stats()
        assert st.visible_count == k["visible"] and st.drawn_count == k["drawn"]
        assert st.frame_ms >= 0
        img = ctx.readback_rgba8()
        assert (img[..., 3] > 0).any()
        means = img.reshape(-1, 4).astype(np.float64).sum(0) / (w * h * 255.0)
        for c in range(4):
            assert abs(means[c] - k["channel_means"][c]) <= k["tolerance"], (blend, means)
        ctx.close()


def test_back_to_front_order_kat(kats):
    k = kats["back_to_front"]
    n = len(k["positions"])
    scene = {"positions": np.array(k["positions"], np.float32), "opacity": np.ones(n, np.float32),
             "scale_xyz": np.zeros((n, 3), np.float32),
             "rotation_xyzw": np.tile(np.float32([0, 0, 0, 1]), (n, 1)),
             "color_dc": np.tile(np.float32([0.2, 0.3, 0.4]), (n, 1)), "sh_degree": 0,
             "sh_rest": None}
    ctx = _render(scene, gsplat_scenes.default_camera(), 1280, 720)
    assert ctx.debug_order().tolist() == k["order"]
    assert ctx.stats().visible_count == k["visible"]


def test_sort_kats_and_lcg(kats, oracle):
    k = kats["sort_values_immutable"]
    assert ffi.sort_values_by_keys(k["keys"], k["values"]).tolist() == k["values_out"]
    for name in ("sort_pairs_small", "sort_gpu_small"):
        k = kats[name]
        keys, values = ffi.sort_pairs(k["keys"], k["values"])
        assert keys.tolist() == k["keys_out"] and values.tolist() == k["values_out"]
    k = kats["sort_lcg"]
    for n, seed in [(k["large_len"], k["large_seed"])] + [(m, k["edge_seed_base"] + m)
                                                          for m in k["edge_lengths"]]:
        keys = np.array(lcg_seq(seed, n), np.uint32)
        vals = np.arange(n, dtype=np.uint32)
        assert np.array_equal(ffi.sort_values_by_keys(keys, vals),
                              oracle.sort_values_by_keys(keys, vals)), n
        gk, gv = ffi.sort_pairs(keys, vals)
        ok_, ov = oracle.sort_pairs(keys, vals)
        assert np.array_equal(gk, ok_) and np.array_equal(gv, ov), n


def test_sort_gpu_radix_cases(kats, oracle):
    k = kats["gpu_radix_cases"]
    for count in k["counts"]:
        idx = np.arange(count, dtype=np.uint64)
        keys = ((idx * np.uint64(k["hash_multiplier"])) & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        keys &= np.uint32(k["key_mask"])
        keys[idx % 11 == 0] = 0
        keys[idx % 11 == 1] = 0xFFFFFFFF
        ids = (count - idx).astype(np.uint32)
        assert np.array_equal(ffi.sort_values_by_keys(keys, ids),
                              oracle.sort_values_by_keys(keys, ids)), count
    eq = k["equal_keys"]
    ids = np.arange(eq["count"], dtype=np.uint32)
    assert np.array_equal(ffi.sort_values_by_keys(np.full(eq["count"], eq["key"], np.uint32), ids), ids)


@pytest.mark.parametrize("n", [3_000_000, 5_000_001, 17_000_003])
def test_sort_large_with_ties(oracle, n):
    """Heavy ties over millions of keys; 17 M keys run the four-blocks-per-SM
    pass of sorts that leave L2."""
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 1 << 20, n, dtype=np.uint32)  # heavy ties, top byte constant
    vals = rng.permutation(n).astype(np.uint32)
    assert np.array_equal(ffi.sort_values_by_keys(keys, vals), oracle.sort_values_by_keys(keys, vals))


def test_tile_size_does_not_change_the_image(oracle):
    scene, cam, w, h = gsplat_scenes.config1(seed=3)
    a = _render(scene, cam, w, h, tile=16).readback_rgba8()
    b = _render(scene, cam, w, h, tile=8).readback_rgba8()
    assert np.array_equal(a, b)
    sv = oracle.SceneView(scene)
    fr = oracle.Frame(sv, cam, w, h, tile=8)
    ctx = _render(scene, cam, w, h, tile=8)
    _compare_stages(ctx, fr, sv)


@pytest.mark.parametrize("degree", [1, 2, 4])
def test_sh_degrees(oracle, degree):
    rng = np.random.default_rng(degree)
    n = 5000
    scene = gsplat_scenes.make_scene(rng, gsplat_scenes.gmm_means(rng, n), -4.0, 0.6, 0.5, 1.5,
                                     degree)
    cam = gsplat_scenes.camera((2.5, 0.8, -3.0), (0, 0, 0), 55.0)
    sv = oracle.SceneView(scene)
    fr = oracle.Frame(sv, cam, 400, 300)
    ctx = _render(scene, cam, 400, 300)
    _compare_stages(ctx, fr, sv)
    assert_fp32_image(ctx.readback_rgba8(), fr.raster_tiles_fp32())


def test_edge_cases(oracle):
    empty = {"positions": np.zeros((0, 3), np.float32), "opacity": np.zeros(0, np.float32),
             "scale_xyz": np.zeros((0, 3), np.float32), "rotation_xyzw": np.zeros((0, 4), np.float32),
             "color_dc": np.zeros((0, 3), np.float32), "sh_degree": 0, "sh_rest": None}
    ctx = _render(empty, gsplat_scenes.default_camera(), 64, 48)
    assert ctx.stats().visible_count == 0
    assert not ctx.readback_rgba8().any()
    assert ctx.debug_order().size == 0
    # everything behind the camera
    scene, cam, w, h = gsplat_scenes.config1(seed=1)
    back = dict(cam, rotation_xyzw=gsplat_scenes.look_at(cam["position"], (0, 0, -20)))
    ctx = _render(scene, back, w, h)
    fr = oracle.Frame(oracle.SceneView(scene), back, w, h)
    assert ctx.stats().visible_count == fr.visible
    assert_fp32_image(ctx.readback_rgba8(), fr.raster_tiles_fp32())
    # odd image sizes (partial edge tiles)
    for (w2, h2) in ((1, 1), (17, 33), (255, 1)):
        ctx = _render(scene, cam, w2, h2)
        fr = oracle.Frame(oracle.SceneView(scene), cam, w2, h2)
        assert_fp32_image(ctx.readback_rgba8(), fr.raster_tiles_fp32(), (w2, h2))


def test_large_splats_grow_pair_buffers(oracle):
    """Large splats near the camera overflow the initial pair capacity; the
    frame is re-run with larger buffers and stays exact."""
    rng = np.random.default_rng(9)
    n = 3000
    means = rng.uniform(-2, 2, (n, 3)).astype(np.float32)
    scene = gsplat_scenes.make_scene(rng, means, -0.5, 0.3, 2.0, 0.5, 0)
    cam = gsplat_scenes.camera((0.0, 0.0, -3.0), (0, 0, 0), 70.0)
    sv = oracle.SceneView(scene)
    fr = oracle.Frame(sv, cam, 640, 480, tile=8)
    ctx = _render(scene, cam, 640, 480, tile=8)
    counts = ctx.frame_counts()
    assert counts.tile_keys == len(fr.pair_tiles) > 16 * n
    assert counts.frame_reruns >= 1
    _compare_stages(ctx, fr, sv)
    assert_fp32_image(ctx.readback_rgba8(), fr.raster_tiles_fp32())


def test_repeat_frames_are_identical_and_camera_errors():
    scene, cam, w, h = gsplat_scenes.config1(seed=4)
    ctx = _render(scene, cam, w, h, debug=False)
    a = ctx.readback_rgba8().copy()
    ctx.render_frame()
    assert np.array_equal(a, ctx.readback_rgba8())
    bad = dict(cam, near_plane=10.0, far_plane=1.0)
    with pytest.raises(ffi.GsplatError) as e:
        ctx.set_camera(bad)
    assert e.value.code == ffi.INVALID_ARGUMENT
    ctx2 = _ctx(32, 32)
    with pytest.raises(ffi.GsplatError) as e:
        ctx2.render_frame()
    assert e.value.code == ffi.SCENE_NOT_LOADED
    with pytest.raises(ffi.GsplatError) as e:
        ctx2.set_auto_camera()
    assert e.value.code == ffi.SCENE_NOT_LOADED
    ctx2.load_scene(scene)
    ctx2.set_auto_camera()
    ctx2.render_frame()
    assert ctx2.stats().visible_count > 0
    ctx2.set_size(48, 40)
    ctx2.render_frame()
    assert ctx2.readback_rgba8().shape == (40, 48, 4)


def test_cuda_graph_replay_matches_direct_launches(oracle):
    """Frames replayed from the captured CUDA graph (same layout, new camera
    each frame, synchronous and enqueued) equal frames issued launch by
    launch bit for bit, and the oracle's; phase timings stay available."""
    scene, cam, w, h = gsplat_scenes.config1(seed=5)
    sv = oracle.SceneView(scene)
    rng = np.random.default_rng(11)
    cams = [gsplat_scenes.orbit_camera(rng, (4.0, 6.0)) for _ in range(4)]
    direct = _ctx(w, h)
    direct.set_cuda_graph(False)
    direct.load_scene(scene)
    graph = _ctx(w, h)
    graph.load_scene(scene)
    for c in cams:
        direct.set_camera(c)
        direct.render_frame()
        graph.set_camera(c)
        graph.render_frame()
        img = graph.readback_rgba8()
        assert np.array_equal(img, direct.readback_rgba8())
        assert_fp32_image(img, oracle.Frame(sv, c, w, h).raster_tiles_fp32())
        t = graph.phase_times()
        assert all(v >= 0.0 for v in t.values()) and sum(t.values()) > 0.0
    for c in cams:
        graph.set_camera(c)
        graph.render_frame_async()
    graph.sync()
    assert np.array_equal(graph.readback_rgba8(), direct.readback_rgba8())


def test_smaller_scene_after_larger_reuses_workspace(oracle):
    """A workspace sized by a sort above 2M keys (16 keys per thread) must
    also serve a later, smaller sort that runs 8 keys per thread and so has
    more tiles: plain context and batch lane alike."""
    rng = np.random.default_rng(31)
    big = gsplat_scenes.make_scene(rng, gsplat_scenes.gmm_means(rng, 2_300_000), -5.0, 0.5, 0.5,
                                   1.5, 0)
    small = gsplat_scenes.make_scene(rng, gsplat_scenes.gmm_means(rng, 1_200_000), -5.0, 0.5, 0.5,
                                     1.5, 0)
    cam = gsplat_scenes.camera((0.0, 0.5, -5.0), (0, 0, 0), 50.0)
    w, h = 320, 240
    ref = oracle.Frame(oracle.SceneView(small), cam, w, h).raster_tiles_fp32()
    ctx = _ctx(w, h)
    ctx.load_scene(big)
    ctx.set_camera(cam)
    ctx.render_frame()
    ctx.load_scene(small)
    ctx.render_frame()
    assert_fp32_image(ctx.readback_rgba8(), ref)
    with ffi.Batch() as b:
        b.add_scene(big)
        b.add_scene(small)
        b.render([(0, cam, w, h)])
        b.render([(1, cam, w, h)])
        assert_fp32_image(b.readback_rgba8(0), ref)


RASTER_SHAPES = [(16, c, b) for c in (256, 128, 64) for b in (0, 2, 4)] + \
    [(8, c, b) for c in (64, 32) for b in (0, 8, 16)]


def test_raster_launch_shapes_do_not_change_pixels(oracle):
    """Every tile size, chunk size and persistent-queue setting the autotuner
    may pick gives the same image bit for bit, within the FP32 tolerance of
    the oracle's."""
    scene, cam, w, h = gsplat_scenes.config1(seed=12)
    ref = oracle.Frame(oracle.SceneView(scene), cam, w + 37, h + 5).raster_tiles_fp32()
    ctx = _ctx(w + 37, h + 5)
    ctx.load_scene(scene)
    ctx.set_camera(cam)
    first = None
    for tile, chunk, bps in RASTER_SHAPES:
        ctx.set_tile_size(tile)
        ctx.set_raster_config(chunk, bps)
        ctx.render_frame()
        img = ctx.readback_rgba8()
        if first is None:
            first = img
            assert_fp32_image(img, ref)
        assert np.array_equal(img, first), (tile, chunk, bps)
    with pytest.raises(ffi.GsplatError) as e:
        ctx.set_raster_config(256, 0)  # tile size is 8 now
    assert e.value.code == ffi.INVALID_ARGUMENT
    ctx.set_tile_size(16)
    with pytest.raises(ffi.GsplatError):
        ctx.set_raster_config(96, 0)
    with pytest.raises(ffi.GsplatError):
        ctx.set_raster_config(256, 33)


def test_sort_interval_reuses_the_last_order(oracle):
    """The reference's surface sort cadence: with interval 3 the depth order
    is re-sorted on the 3rd camera change; frames in between draw the last
    sorted order with their own projection, equal to the oracle given that
    stale order. The orbit steps (0.0015 rad, 7.5 mm) stay inside the
    reference's stale-order pose bound."""
    scene, _, w, h = gsplat_scenes.config1(seed=21)
    sv = oracle.SceneView(scene)
    cams = [gsplat_scenes.camera((5.0 * math.sin(0.0015 * k), 0.3, -5.0 * math.cos(0.0015 * k)),
                                 (0, 0, 0), 50.0) for k in range(6)]
    ctx = _ctx(w, h)
    ctx.set_debug_taps(True)
    ctx.load_scene(scene)
    ctx.set_sort_interval(3)
    expect_sorted = [True, False, False, True, False, False]
    stale = None
    for k, cam in enumerate(cams):
        ctx.set_camera(cam)
        ctx.render_frame()
        counts = ctx.frame_counts()
        assert bool(counts.sort_refreshed) == expect_sorted[k], k
        own = oracle.Frame(sv, cam, w, h)
        if expect_sorted[k]:
            stale = own.order
        fr = oracle.Frame(sv, cam, w, h, order=stale)
        assert np.array_equal(ctx.debug_order(), stale), k
        assert counts.visible == own.visible  # depth-visible with this camera
        tiles, ids = ctx.debug_tile_pairs()
        assert np.array_equal(tiles, fr.pair_tiles) and np.array_equal(ids, fr.pair_ids), k
        assert_fp32_image(ctx.readback_rgba8(), fr.raster_tiles_fp32(), k)
    # interval 1: an unchanged camera reuses the order and gives the same image
    ctx.set_sort_interval(1)
    ctx.set_camera(cams[2])
    ctx.render_frame()
    assert ctx.frame_counts().sort_refreshed == 1
    img = ctx.readback_rgba8().copy()
    ctx.render_frame()
    assert ctx.frame_counts().sort_refreshed == 0
    assert np.array_equal(ctx.readback_rgba8(), img)
    # interval 0 (the context default): every frame sorts
    ctx.set_sort_interval(0)
    ctx.render_frame()
    assert ctx.frame_counts().sort_refreshed == 1
    ctx.render_frame()
    assert ctx.frame_counts().sort_refreshed == 1
    assert np.array_equal(ctx.readback_rgba8(), img)


def test_auto_camera_matches_the_oracle(oracle):
    """gsplat_context_set_auto_camera frames the scene exactly as the
    reference's context does (crates/gsplat-ffi-c/src/lib.rs:1593-1779): the
    camera read back equals the oracle's restatement bit for bit, for the
    reference's minimal_ascii.ply, the 16k and 279k synthetic scenes, and a
    portrait image (aspect below 0.6 takes the 65 degree field of view)."""
    import json

    import gsplat_scenes as gs
    with open(os.path.join(GOLDEN, "minimal_ascii_scene.json")) as f:
        minimal = gs.scene_from_json(json.load(f))
    scenes = [("minimal_ascii", minimal, 64, 64), ("config1", gs.config1(seed=0)[0], 256, 256),
              ("config2", gs.config2()[0], 1920, 1080), ("portrait", gs.config1(seed=4)[0], 200, 400)]
    for name, scene, w, h in scenes:
        ctx = _ctx(w, h)
        ctx.load_scene(scene)
        ctx.set_auto_camera()
        got = ctx.camera().to_dict()
        want = oracle.auto_camera(scene["positions"], w, h)
        for k in ("position", "rotation_xyzw", "vertical_fov_radians", "near_plane", "far_plane"):
            a = np.asarray(got[k], np.float32).view(np.uint32)
            b = np.asarray(want[k], np.float32).view(np.uint32)
            assert np.array_equal(a, b), (name, k, got[k], want[k])
        ctx.render_frame()
        assert ctx.stats().visible_count > 0, name
        ctx.close()
    # the PLY path keeps the host positions the framing reads
    ctx = _ctx(64, 64)
    ctx.load_scene_path(os.path.join(GOLDEN, "minimal_ascii.ply"))
    ctx.set_auto_camera()
    want = oracle.auto_camera(minimal["positions"], 64, 64)
    assert np.array_equal(np.asarray(ctx.camera().to_dict()["position"], np.float32),
                          np.asarray(want["position"], np.float32))
    ctx.close()


def test_sort_interval_pose_bound(oracle):
    """A reused order is dropped, and the frame sorted, as soon as the camera
    leaves the reference's stale-order pose bound of the camera the order was
    sorted for (surface_session.rs:23-24, 1255-1272): rotation above 0.01 rad,
    or translation above 2% of the scene's bounding-box diagonal."""
    scene, _, w, h = gsplat_scenes.config1(seed=22)
    sv = oracle.SceneView(scene)
    pos = scene["positions"].astype(np.float32)
    ext = pos.max(axis=0) - pos.min(axis=0)
    diag = float(np.sqrt(np.float32((ext * ext).sum())))
    base = (0.0, 0.3, -5.0)
    ctx = _ctx(w, h)
    ctx.set_debug_taps(True)
    ctx.load_scene(scene)
    ctx.set_sort_interval(8)

    def frame(cam, expect_sorted):
        ctx.set_camera(cam)
        ctx.render_frame()
        assert bool(ctx.frame_counts().sort_refreshed) == expect_sorted, cam
        return ctx.debug_order()

    frame(gsplat_scenes.camera(base, (0, 0, 0), 50.0), True)  # first frame sorts
    # inside the bound: 0.006 rad of yaw, translation well under 2% of the diagonal
    yaw = 0.003
    small = gsplat_scenes.camera((5.0 * math.sin(yaw), 0.3, -5.0 * math.cos(yaw)), (0, 0, 0), 50.0)
    frame(small, False)
    # rotation beyond 0.01 rad from the sorted camera (the look-at turns ~0.02 rad)
    yaw = 0.02
    turned = gsplat_scenes.camera((5.0 * math.sin(yaw), 0.3, -5.0 * math.cos(yaw)), (0, 0, 0), 50.0)
    order = frame(turned, True)
    assert np.array_equal(order, oracle.Frame(sv, turned, w, h).order)
    # translation beyond 2% of the diagonal with the same rotation
    shifted = dict(turned, position=[turned["position"][0], turned["position"][1] + 0.03 * diag,
                                     turned["position"][2]])
    order = frame(shifted, True)
    assert np.array_equal(order, oracle.Frame(sv, shifted, w, h).order)
    # a move of 1% of the diagonal stays inside the bound: the order is reused
    near = dict(shifted, position=[shifted["position"][0] + 0.01 * diag, shifted["position"][1],
                                   shifted["position"][2]])
    assert np.array_equal(frame(near, False), order)


def test_benchmark_artifact_from_rendered_frames(tmp_path):
    """Real frames through the C ABI recorded as a v1 benchmark artifact
    (the reference's contract) pass the contract checks."""
    import bench_artifact

    scene, cam, w, h = gsplat_scenes.config1(seed=14)
    ctx = _ctx(w, h)
    ctx.load_scene(scene)
    rng = np.random.default_rng(3)
    cams = [gsplat_scenes.orbit_camera(rng, (4.0, 6.0)) for _ in range(12)]
    out = np.empty(w * h * 4, np.uint8)
    frames = bench_artifact.record_frames(ctx, cams, out, "gpu-test-run")
    assert all(f["gpu_complete_ms"] > 0 and f["call_ms"] > 0 for f in frames)
    assert all(f["visible"] > 0 for f in frames)
    manifest = {
        "run_id": "gpu-test-run",
        "identity": {k: "2026-12-01T00:00:00Z" for k in (
            "started_at_utc", "ended_at_utc", "measurement_started_at_utc",
            "measurement_ended_at_utc")} | {"series_id": "gpu-test"},
        "build": {"repository_commit": None, "dirty": None, "profile": "release",
                  "package_version": "0.1.0"},
        "dataset": {"id": "config1-seed14", "sha256": "2" * 64, "bytes": 1, "splat_count": 16384,
                    "sh_degree": 0},
        "trace": {"id": "orbit", "sha256": "3" * 64},
        "renderer": {"implementation": "gsplat-rs-b200-cuda", "path": "sorted_alpha_cuda_tiles",
                     "backend": "cuda-sm_100a", "sort_policy": "gpu_every_frame"},
        "display": {"width": w, "height": h, "dpr": 1.0, "refresh_hz": 60.0,
                    "frame_budget_ms": 16.7, "refresh_hz_source": "configured",
                    "frame_budget_source": "configured"},
        "environment": {"platform": "x", "os": "x", "device": "B200", "browser": None,
                        "adapter": "B200", "driver": None},
        "unavailable_fields": ["build.repository_commit", "build.dirty", "environment.browser",
                               "environment.driver"],
    }
    bench_artifact.write_artifact(str(tmp_path), manifest, frames, 0, 16.7)
    assert bench_artifact.validate(str(tmp_path))["frames"] == 12


def test_c_smoke_programs_run():
    exe = os.path.join(ROOT, "tests", "ffi", "_build_smoke")
    subprocess.run(["gcc", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "ffi", "ffi_smoke_cuda.c"), "-o", exe,
                    "-L", os.path.dirname(ffi.LIB_PATH), "-lgsplat_ffi_c",
                    "-Wl,-rpath," + os.path.dirname(ffi.LIB_PATH)], check=True)
    try:
        r = subprocess.run([exe], cwd=ROOT, capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        assert "ffi smoke ok" in r.stdout
    finally:
        os.remove(exe)
    ref = os.path.join(ROOT, "oracle", "_ref", "ffi_smoke")
    if os.path.exists(ref):
        r = subprocess.run([ref, os.path.join(GOLDEN, "minimal_ascii.ply")], cwd=ROOT,
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        assert "ffi smoke ok" in r.stdout


def test_async_readback_pipeline_equals_synchronous_frames():
    """Frames enqueued back to back, each read back asynchronously into its
    own host buffer while the next renders (two device images alternate),
    equal frame-by-frame synchronous renders; sizes change in between."""
    scene, _, w, h = gsplat_scenes.config1(seed=13)
    rng = np.random.default_rng(2)
    cams = [gsplat_scenes.orbit_camera(rng, (4.0, 6.0)) for _ in range(7)]
    ref = []
    with ffi.Context(w, h) as ctx:
        ctx.load_scene(scene)
        for c in cams:
            ctx.set_camera(c)
            ctx.render_frame()
            ref.append(ctx.readback_rgba8())
    with ffi.Context(w, h) as ctx:
        ctx.load_scene(scene)
        outs = [np.zeros(w * h * 4, np.uint8) for _ in cams]
        for c, out in zip(cams, outs):
            ctx.set_camera(c)
            ctx.render_frame_async()
            ctx.readback_rgba8_async(out)
        ctx.sync()
        for k, out in enumerate(outs):
            assert np.array_equal(out.reshape(h, w, 4), ref[k]), k
        # a resize in the middle of the pipeline, then synchronous frames again
        ctx.set_size(w + 16, h - 8)
        ctx.set_camera(cams[0])
        ctx.render_frame_async()
        big = np.zeros((w + 16) * (h - 8) * 4, np.uint8)
        ctx.readback_rgba8_async(big)
        ctx.sync()
        ctx.render_frame()
        assert np.array_equal(ctx.readback_rgba8().reshape(-1), big)


@pytest.mark.parametrize("lanes", [2, 3, 4, 8])
def test_frame_lanes_equal_single_lane_frames(lanes):
    """Frames that overlap on the device over `lanes` pipelines (one stream,
    workspace and image each) give, frame by frame, the single-lane images:
    async frames with async readbacks, a synchronous frame among them (its
    counters and debug order are the last frame's), a larger scene that
    overflows a lane's pair buffers on a synchronous frame, and a return to
    one lane."""
    scene, _, w, h = gsplat_scenes.config1(seed=17)
    rng = np.random.default_rng(lanes)
    cams = [gsplat_scenes.orbit_camera(rng, (4.0, 6.0)) for _ in range(11)]
    ref, orders = [], []
    with ffi.Context(w, h) as ctx:
        ctx.set_debug_taps(True)
        ctx.load_scene(scene)
        for c in cams:
            ctx.set_camera(c)
            ctx.render_frame()
            ref.append(ctx.readback_rgba8().copy())
            orders.append(ctx.debug_order().copy())
    with ffi.Context(w, h) as ctx:
        ctx.set_debug_taps(True)
        ctx.load_scene(scene)
        ctx.set_frame_lanes(lanes)
        outs = [np.zeros(w * h * 4, np.uint8) for _ in cams]
        for rep in range(2):
            for k, (c, out) in enumerate(zip(cams, outs)):
                ctx.set_camera(c)
                if k == 5:
                    ctx.render_frame()
                    assert np.array_equal(ctx.debug_order(), orders[k])
                    assert ctx.stats().visible_count == len(orders[k])
                else:
                    ctx.render_frame_async()
                ctx.readback_rgba8_async(out)
            ctx.sync()
            assert np.array_equal(ctx.debug_order(), orders[-1])
            for k, out in enumerate(outs):
                assert np.array_equal(out.reshape(h, w, 4), ref[k]), (rep, k)
        big, bcam, bw, bh = gsplat_scenes.config2(seed=5, n=60000)
        ctx.load_scene(big)
        ctx.set_size(bw // 2, bh // 2)
        ctx.set_camera(bcam)
        ctx.render_frame()
        want = ctx.readback_rgba8().copy()
        for _ in range(2 * lanes):
            ctx.render_frame_async()
        ctx.sync()
        assert np.array_equal(ctx.readback_rgba8(), want)
        ctx.set_frame_lanes(1)
        ctx.render_frame_async()
        ctx.sync()
        assert np.array_equal(ctx.readback_rgba8(), want)
