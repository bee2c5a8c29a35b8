"""The sort/raster stress frame on the GPU against the oracle: 3,000,000 SH3
splats (a uniform 10^3 box plus a dense core), the camera inside the volume,
3840x2160 — 2.7 M depth-visible splats and 208 M tile pairs, where the depth
keys and pairs no longer fit the L2 cache and tile lists reach 34 k entries.

Integer and index work is compared bit for bit over the whole frame: the
visible and drawn counts, the depth order, every projected record, every
emitted (tile, splat) pair, the tile ranges and the per-tile lists. The FP32
image is compared with the oracle's FP32 tile model over the whole frame
(within the tolerance of tests/conftest.py::assert_fp32_image). The UNORM8
parity image is compared bit for bit with the reference image model on three
bands of 16 rows (top, middle, bottom): the reference model walks all 2.7 M
splats for every band, so the whole frame would take minutes on the host."""

import numpy as np
import pytest

import gsplat_ffi as ffi
import gsplat_scenes
from conftest import assert_fp32_image

pytestmark = pytest.mark.gpu

BANDS = [(0, 16), (1072, 1088), (2144, 2160)]


@pytest.fixture(scope="module")
def frame3(oracle):
    scene, cam, w, h = gsplat_scenes.config3()
    sv = oracle.SceneView(scene)
    fr = oracle.Frame(sv, cam, w, h)
    return scene, cam, w, h, sv, fr


def test_config3_stages_bit_exact(frame3):
    scene, cam, w, h, sv, fr = frame3
    ctx = ffi.Context(w, h)
    ctx.set_debug_taps(True)
    ctx.load_scene(scene)
    ctx.set_camera(cam)
    ctx.render_frame()
    counts = ctx.frame_counts()
    assert counts.visible == fr.visible and counts.drawn == fr.drawn
    assert counts.tile_keys == len(fr.pair_tiles)
    assert np.array_equal(ctx.debug_order(), fr.order), "depth order"
    proj = ctx.debug_projected()
    drawn = (fr.proj["flags"] & 2) != 0
    assert np.array_equal(proj["flags"], fr.proj["flags"])
    for f in ("center_ndc", "axis_u", "axis_v", "color", "extent_scale"):
        assert np.array_equal(proj[f][drawn].view(np.uint32), fr.proj[f][drawn].view(np.uint32)), f
    del proj
    tiles, ids = ctx.debug_tile_pairs()
    assert np.array_equal(tiles, fr.pair_tiles), "pair tiles"
    assert np.array_equal(ids, fr.pair_ids), "pair ids"
    del tiles, ids
    ranges, sorted_ids = ctx.debug_tile_ranges(fr.num_tiles)
    r = np.array(ranges, np.uint32)
    want = np.array(fr.ranges, np.uint32)
    empty = want[:, 0] == want[:, 1]
    assert np.array_equal(r[~empty], want[~empty]), "tile ranges"
    assert np.all(r[empty, 0] == r[empty, 1])
    assert np.array_equal(sorted_ids, fr.tile_ids), "tile lists"
    del sorted_ids
    ctx.close()


def test_config3_images(frame3):
    scene, cam, w, h, sv, fr = frame3
    ctx = ffi.Context(w, h)
    ctx.load_scene(scene)
    ctx.set_camera(cam)
    ctx.render_frame()
    assert_fp32_image(ctx.readback_rgba8(), fr.raster_tiles_fp32(), "fp32 image, whole frame")
    ctx.set_blend_mode(1)
    ctx.render_frame()
    img8 = ctx.readback_rgba8()
    for y0, y1 in BANDS:
        ref8 = fr.raster_unorm8(rows=(y0, y1))
        assert np.array_equal(img8[y0:y1], ref8[y0:y1]), ("unorm8 band", y0, y1)
    ctx.close()
