"""Packed resident scenes on the GPU (the reference's 20-byte hot record and
i8 SH sidecar, packed_atlas.rs, decoded per frame by the preprocess kernel):
the encoding equals the oracle's bit for bit, every frame stage of a packed
scene equals the oracle's frame of the decoded scene, the image stays within
the reference's image-parity gate of the full-precision scene, and batches
and the server mix packed and plane-format scenes with every view equal to
its plain render."""

import numpy as np
import pytest

import gsplat_ffi as ffi
import gsplat_scenes
from conftest import assert_fp32_image
from test_gpu_parity import _compare_stages

pytestmark = pytest.mark.gpu


def _scene(kind, seed=0):
    if kind == "c1":
        scene, cam, w, h = gsplat_scenes.config1(seed=seed)
    elif kind == "c2":
        scene, cam, w, h = gsplat_scenes.config2(seed=seed, n=30_000)
        w, h = 640, 360
    else:
        degree = int(kind[-1])
        rng = np.random.default_rng(seed)
        scene = gsplat_scenes.make_scene(rng, gsplat_scenes.gmm_means(rng, 8000), -4.0, 0.8, 0.5,
                                         1.5, degree)
        cam = gsplat_scenes.camera((0.0, 0.5, -4.0), (0.0, 0.0, 0.0), 55.0)
        w, h = 400, 300
    return scene, cam, w, h


def _packed_ctx(scene, cam, w, h, debug=True):
    ctx = ffi.Context(w, h)
    ctx.set_debug_taps(debug)
    ctx.load_scene_packed(scene)
    ctx.set_camera(cam)
    ctx.render_frame()
    return ctx


@pytest.mark.parametrize("kind", ["c1", "c2", "sh1", "sh2"])
def test_packed_encoding_and_stages_equal_the_oracle(oracle, kind):
    scene, cam, w, h = _scene(kind, seed=4)
    sv = oracle.PackedSceneView(scene)
    with _packed_ctx(scene, cam, w, h) as ctx:
        table, hot, side = ctx.debug_packed_scene()
        assert np.array_equal(table[:11].view(np.uint32), sv.header.view(np.uint32))
        assert np.array_equal(hot.reshape(-1), sv.hot[:5 * sv.n])
        if sv.degree > 0:
            assert np.array_equal(side.reshape(-1), sv.sidecar[:48 * sv.n])
        fr = oracle.Frame(sv, cam, w, h)
        _compare_stages(ctx, fr, sv)
        assert_fp32_image(ctx.readback_rgba8(), fr.raster_tiles_fp32())


def test_packed_image_passes_the_reference_gate_against_the_full_scene():
    """Quantisation error only: the reference's image-parity gate
    (lib.rs:3520-3537) between the packed and the full-precision render."""
    scene, cam, w, h = gsplat_scenes.config2(seed=2)
    with ffi.Context(w, h) as full, ffi.Context(w, h) as packed:
        full.load_scene(scene)
        packed.load_scene_packed(scene)
        for ctx in (full, packed):
            ctx.set_camera(cam)
            ctx.render_frame()
        a = full.readback_rgba8().astype(np.int32)
        b = packed.readback_rgba8().astype(np.int32)
    rgb = np.abs(a - b)[..., :3] / 255.0
    assert rgb.mean() <= 1.0 / 255.0
    assert (rgb > 3.0 / 255.0).any(axis=-1).mean() <= 0.001


def test_degree_four_is_not_packed():
    rng = np.random.default_rng(1)
    scene = gsplat_scenes.make_scene(rng, gsplat_scenes.gmm_means(rng, 100), -4.0, 0.8, 0.5, 1.5, 4)
    with ffi.Context(64, 64) as ctx:
        with pytest.raises(ffi.GsplatError) as e:
            ctx.load_scene_packed(scene)
        assert e.value.code == ffi.UNSUPPORTED


def test_batch_and_server_mix_packed_and_plane_scenes():
    s_full, cam0, _, _ = _scene("sh2", seed=8)
    s_pack, cam1, _, _ = _scene("c1", seed=9)
    rng = np.random.default_rng(3)
    views = []
    for k in range(12):
        sid = k % 3
        cam = gsplat_scenes.orbit_camera(rng, (3.0, 6.0))
        views.append((sid, cam, [(320, 240), (256, 256), (200, 120)][k % 3]))

    def plain(sid, cam, w, h):
        with ffi.Context(w, h) as ctx:
            if sid == 0:
                ctx.load_scene(s_full)
            else:
                ctx.load_scene_packed(s_full if sid == 2 else s_pack)
            ctx.set_camera(cam)
            ctx.render_frame()
            return ctx.readback_rgba8()

    refs = [plain(sid, cam, w, h) for sid, cam, (w, h) in views]
    with ffi.Batch() as b:
        assert b.add_scene(s_full) == 0
        assert b.add_scene_packed(s_pack) == 1
        assert b.add_scene_packed(s_full) == 2
        arr = ffi.Batch.make_views([(sid, cam, w, h) for sid, cam, (w, h) in views])
        b.render(arr)
        for k in range(len(views)):
            assert np.array_equal(b.readback_rgba8(k), refs[k]), k
    with ffi.Server(lanes=2, max_views=8) as srv:
        srv.add_scene(s_full)
        srv.add_scene_packed(s_pack)
        srv.add_scene_packed(s_full)
        ids = [srv.submit(sid, cam, w, h) for sid, cam, (w, h) in views]
        for k, rid in enumerate(ids):
            srv.wait(rid)
            assert np.array_equal(srv.read_rgba8(rid), refs[k]), k
            srv.release(rid)
