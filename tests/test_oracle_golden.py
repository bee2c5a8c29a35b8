"""Pins the CPU oracle to the reference's own known-answer tests (CPU only)."""

import math

import numpy as np
import pytest

import gsplat_scenes
from conftest import lcg_seq


def _expected_desc_stable(keys, values):
    # sort_by(key desc) then ties in input order (Rust sort_by is stable).
    order = sorted(range(len(keys)), key=lambda i: (-int(keys[i]), i))
    return [keys[i] for i in order], [values[i] for i in order]


def test_sort_pairs_small(oracle, kats):
    k = kats["sort_pairs_small"]
    keys, values = oracle.sort_pairs(k["keys"], k["values"])
    assert keys.tolist() == k["keys_out"] and values.tolist() == k["values_out"]
    k = kats["sort_gpu_small"]
    keys, values = oracle.sort_pairs(k["keys"], k["values"])
    assert keys.tolist() == k["keys_out"] and values.tolist() == k["values_out"]


def test_sort_values_by_immutable_keys(oracle, kats):
    k = kats["sort_values_immutable"]
    assert oracle.sort_values_by_keys(k["keys"], k["values"]).tolist() == k["values_out"]


def test_sort_lcg_large_and_edge_lengths(oracle, kats):
    k = kats["sort_lcg"]
    cases = [(k["large_len"], k["large_seed"])] + [
        (n, k["edge_seed_base"] + n) for n in k["edge_lengths"]]
    for n, seed in cases:
        keys = lcg_seq(seed, n)
        values = list(range(n))
        # sort_pairs orders by key desc, then value asc (= index asc here).
        ek, ev = _expected_desc_stable(keys, values)
        got_k, got_v = oracle.sort_pairs(keys, values)
        assert got_k.tolist() == ek and got_v.tolist() == ev, n
        assert oracle.sort_values_by_keys(keys, values).tolist() == ev, n


def test_sort_gpu_radix_cases_stable(oracle, kats):
    k = kats["gpu_radix_cases"]
    for count in k["counts"]:
        keys, ids = [], []
        for index in range(count):
            m = index % 11
            if m == 0:
                key = 0
            elif m == 1:
                key = 0xFFFFFFFF
            else:
                key = ((index * k["hash_multiplier"]) & 0xFFFFFFFF) & k["key_mask"]
            keys.append(key)
            ids.append(count - index)
        ek, ev = _expected_desc_stable(keys, ids)
        assert oracle.sort_values_by_keys(keys, ids).tolist() == ev, count
    eq = k["equal_keys"]
    ids = list(range(eq["count"]))
    assert oracle.sort_values_by_keys([eq["key"]] * eq["count"], ids).tolist() == ids


def test_radix_count_simd_matches_scalar(oracle):
    # radix.rs:242-263: len 10,003, seed 11, hi/lo words from the LCG.
    seq = lcg_seq(11, 2 * 10003)
    vals = np.array([(seq[2 * i] << 32) | seq[2 * i + 1] for i in range(10003)], np.uint64)
    for shift in range(0, 64, 8):
        assert np.array_equal(oracle.radix_count(vals, shift, True),
                              oracle.radix_count(vals, shift, False)), shift


def test_back_to_front_order(oracle, kats):
    k = kats["back_to_front"]
    cam = gsplat_scenes.default_camera()
    keys, ids = oracle.preprocess_visible(np.array(k["positions"], np.float32), cam)
    assert len(ids) == k["visible"]
    assert oracle.sort_values_by_keys(keys, ids).tolist() == k["order"]


def test_camera_validation(oracle):
    cam = gsplat_scenes.default_camera()
    assert oracle.camera_validate(cam) == 0
    bad = dict(cam, near_plane=10.0, far_plane=1.0)
    assert oracle.camera_validate(bad) == 1
    assert oracle.camera_validate(dict(cam, rotation_xyzw=[0, 0, 0, 0])) == 1
    assert oracle.camera_validate(dict(cam, rotation_xyzw=[0, 0, 0, 2.0])) == 1
    assert oracle.camera_validate(dict(cam, vertical_fov_radians=math.pi)) == 1
    assert oracle.camera_validate(dict(cam, position=[float("nan"), 0, 0])) == 1


def _single(position, scale, rot, opacity=1.0, dc=(0.2, 0.3, 0.4)):
    return {"positions": np.array([position], np.float32), "opacity": np.array([opacity], np.float32),
            "scale_xyz": np.array([scale], np.float32), "rotation_xyzw": np.array([rot], np.float32),
            "color_dc": np.array([dc], np.float32), "sh_degree": 0, "sh_rest": None}


def _axes(proj):
    u, v = proj["axis_u"][0], proj["axis_v"][0]
    return float(np.hypot(*u)), float(np.hypot(*v)), float(u[0] * v[0] + u[1] * v[1])


def test_covariance_axes_nonzero_and_anisotropic(oracle):
    # lib.rs:4443-4462: cov diag(0.02, 0.005, 0.002) at camera-space (0.2, -0.1, 2).
    cam = gsplat_scenes.default_camera()
    scale = [0.5 * math.log(0.02), 0.5 * math.log(0.005), 0.5 * math.log(0.002)]
    sv = oracle.SceneView(_single([0.2, -0.1, 2.0], scale, [0, 0, 0, 1]))
    fr = oracle.Frame(sv, cam, 1280, 720)
    lu, lv, _ = _axes(fr.proj)
    assert lu > 0 and lv > 0 and lu > lv


def test_oriented_axes_orthogonal(oracle):
    # lib.rs:4464-4496
    qz = math.sqrt(0.5)
    cam = gsplat_scenes.default_camera()
    sv = oracle.SceneView(_single([0, 0, 2.0], [0.8, -0.4, -0.4], [0, 0, qz, qz]))
    inst, _ = oracle.build_instances(sv, cam, 1280, 720, [0])
    assert inst.shape[0] == 1
    u, v = inst[0, 2:4], inst[0, 4:6]
    assert np.hypot(*u) > np.hypot(*v) and abs(float(u @ v)) < 1e-4
    fr = oracle.Frame(sv, cam, 1280, 720)
    lu, lv, dot = _axes(fr.proj)
    assert lu > lv and abs(dot) < 1e-4


def test_partial_offscreen_splat_kept(oracle):
    # lib.rs:4498-4528
    cam = gsplat_scenes.default_camera()
    sv = oracle.SceneView(_single([2.3, 0, 1.0], [2.0, 2.0, 2.0], [0, 0, 0, 1]))
    inst, _ = oracle.build_instances(sv, cam, 1280, 720, [0])
    assert inst.shape[0] == 1
    cx, ext = inst[0, 0], abs(inst[0, 2]) + abs(inst[0, 4])
    assert cx > 2.0 and cx - ext <= 1.0
    fr = oracle.Frame(sv, cam, 1280, 720)
    assert fr.proj["flags"][0] & 2


def test_conformance_minimal_ascii(oracle, kats, minimal_scene):
    k = kats["conformance"]
    w, h = k["size"]
    sv = oracle.SceneView(minimal_scene)
    assert sv.validate() == 0
    fr = oracle.Frame(sv, gsplat_scenes.default_camera(), w, h)
    assert fr.visible == k["visible"]
    img = fr.raster_unorm8()
    assert (img[..., 3] > 0).any()
    means = img.reshape(-1, 4).astype(np.float64).sum(0) / (w * h * 255.0)
    for c in range(4):
        assert abs(means[c] - k["channel_means"][c]) <= k["tolerance"], (c, means)
    # the FP64 evaluation and the FP32 front-to-back tile raster agree too
    img64, _ = fr.raster_f64()
    img32 = fr.raster_tiles_fp32()
    assert np.abs(img64.astype(int) - img.astype(int)).max() <= 2
    assert np.abs(img32.astype(int) - img64.astype(int)).max() <= 1


def test_wgsl_restatement_matches_cpu_builder(oracle):
    """The WGSL vertex-stage restatement and the reference's CPU instance
    builder agree: geometry bit for bit, colour up to SH summation order."""
    scene, cam, w, h = gsplat_scenes.config2(seed=7, n=4000)
    sv = oracle.SceneView(scene)
    fr = oracle.Frame(sv, cam, w, h)
    inst, idx = oracle.build_instances(sv, cam, w, h, fr.order)
    drawn = fr.proj["flags"] & 2
    assert len(idx) == int(np.count_nonzero(drawn))
    p = fr.proj[idx]
    assert np.array_equal(inst[:, 0:2], p["center_ndc"])
    assert np.array_equal(inst[:, 2:4], p["axis_u"])
    assert np.array_equal(inst[:, 4:6], p["axis_v"])
    assert np.abs(inst[:, 8:12] - p["color"]).max() < 2e-6


def test_two_stage_tile_order_equals_u64_key_sort(oracle):
    """Emission in depth order then a stable sort by tile equals one stable
    sort of 64-bit (tile, ~depth bits) keys emitted in id order."""
    scene, cam, w, h = gsplat_scenes.config1(seed=5)
    sv = oracle.SceneView(scene)
    fr = oracle.Frame(sv, cam, w, h)
    # the emitted pairs, regrouped in id order (emission order within an id)
    by_id = np.argsort(fr.pair_ids, kind="stable")
    tiles = fr.pair_tiles[by_id].astype(np.uint64)
    ids = fr.pair_ids[by_id]
    dbits = np.maximum(fr.proj["depth"][ids], np.float32(0.0)).view(np.uint32)
    keys = (tiles << np.uint64(32)) | (~dbits).astype(np.uint64)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(ids[order], fr.tile_ids)
    assert np.array_equal((keys[order] >> np.uint64(32)).astype(np.uint32),
                          np.sort(fr.pair_tiles, kind="stable"))


def test_exp_neg_accuracy(oracle):
    xs = np.linspace(-4.5, 0.0, 20001, dtype=np.float32)
    got = np.array([oracle.exp_neg(float(x)) for x in xs], np.float64)
    ref = np.exp(xs.astype(np.float64))
    assert np.max(np.abs(got - ref) / ref) < 5e-7


def test_fp32_tile_raster_vs_reference_models(oracle):
    scene, cam, w, h = gsplat_scenes.config1(seed=0)
    sv = oracle.SceneView(scene)
    fr = oracle.Frame(sv, cam, w, h)
    ref8 = fr.raster_unorm8().astype(np.int32)
    f64, _ = fr.raster_f64()
    fast = fr.raster_tiles_fp32().astype(np.int32)
    d64 = np.abs(fast - f64.astype(np.int32))
    d8 = np.abs(fast - ref8)
    assert d64.max() <= 2 and (d64 > 1).mean() < 1e-4
    # the reference's own image-parity gate (lib.rs:3520-3537)
    rgb = d8[..., :3] / 255.0
    assert rgb.mean() <= 1.0 / 255.0
    assert (rgb > 3.0 / 255.0).any(axis=-1).mean() <= 0.001


def _f32_bits(values):
    return np.asarray(values, np.float32).view(np.uint32)


def test_look_at_rotation_matches_the_oracle(oracle):
    """The product's camera_rotation_looking_at (host code, no GPU) equals the
    oracle's restatement of crates/gsplat-ffi-c/src/lib.rs:1679-1733 bit for
    bit, including forward vectors near +-Y (the alternative up vector) and
    a target on the camera (the +Z fallback)."""
    import gsplat_ffi as ffi

    rng = np.random.default_rng(31)
    cases = [((0.0, 0.0, -5.0), (0.0, 0.0, 0.0)), ((0.0, 5.0, 0.0), (0.0, 0.0, 0.0)),
             ((0.0, -5.0, 0.01), (0.0, 0.0, 0.0)), ((1.0, 2.0, 3.0), (1.0, 2.0, 3.0)),
             ((3.0, 0.0, 0.0), (-3.0, 0.0, 0.0))]
    for _ in range(500):
        cases.append((tuple(rng.normal(0, 5, 3)), tuple(rng.normal(0, 1, 3))))
    for pos, tgt in cases:
        pos32 = np.float32(pos)
        tgt32 = np.float32(tgt)
        want = oracle.camera_look_at(pos32, tgt32)
        got = ffi.camera_look_at([float(v) for v in pos32], [float(v) for v in tgt32], 1.0)
        assert np.array_equal(_f32_bits(list(got.rotation_xyzw)), _f32_bits(want)), (pos, tgt)


def test_vertex_outputs_against_fp64(oracle):
    """The float32 vertex stage (the oracle's, which the CUDA kernel equals bit
    for bit, tests/test_gpu_parity.py) against a float64 evaluation of the
    same reference math (oracle/oracle_f64.py), per output: means2d (NDC
    centres, absolute), the premultiplied colour (absolute) and the conic of
    the clamped axes (relative). Both draw the same splats."""
    import gsplat_scenes
    import oracle_f64

    for scene, cam, w, h in (gsplat_scenes.config1(seed=0),
                             gsplat_scenes.config2(seed=11, n=40000)[:2] + (960, 540)):
        sv = oracle.SceneView(scene)
        fr = oracle.Frame(sv, cam, w, h)
        ref = oracle_f64.project(scene, cam, w, h)
        e = oracle_f64.output_errors(fr.proj, ref)
        print(e)
        assert e["drawn_both"] > 0
        assert e["drawn_disagree"] <= max(2, 1e-4 * e["drawn_both"])
        assert e["center_ndc"]["max_abs"] <= 2e-6
        assert e["color"]["max_abs"] <= 1e-6
        assert e["conic"]["mean_rel"] <= 2e-6 and e["conic"]["p999_rel"] <= 1e-4
