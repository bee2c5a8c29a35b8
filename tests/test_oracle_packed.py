"""Pins the oracle's packed resident format (20-byte hot record + i8 SH
sidecar) to the reference's own packed_atlas tests
(crates/gsplat-render-wgpu/src/packed_atlas.rs:633-880): the same sample scene
and the same round-trip bounds, checked through encode + decode (CPU only)."""

import math

import numpy as np
import pytest


def sample_scene(count, sh_degree):
    # packed_atlas.rs:633-656 (sample_scene)
    i = np.arange(count, dtype=np.float32)
    pos = np.stack([i * np.float32(0.01), np.sin(i * np.float32(0.02)),
                    np.float32(1.0) + i * np.float32(0.001)], axis=1).astype(np.float32)
    scene = {"positions": pos, "opacity": np.zeros(count, np.float32),
             "scale_xyz": np.tile(np.array([-2.0, -1.5, -1.0], np.float32), (count, 1)),
             "rotation_xyzw": np.tile(np.array([0, 0, 0, 1], np.float32), (count, 1)),
             "color_dc": np.tile(np.array([0.2, -0.1, 0.4], np.float32), (count, 1)),
             "sh_degree": sh_degree, "sh_rest": None}
    if sh_degree > 0:
        stride = ((sh_degree + 1) ** 2 - 1) * 3
        k = np.arange(count * stride)
        scene["sh_rest"] = (((k % 17).astype(np.float32) - 8.0) * np.float32(0.02)).astype(np.float32)
    return scene


def test_record_sizes_and_reduction(oracle):
    sv = oracle.PackedSceneView(sample_scene(16, 3))
    assert sv.hot.size // sv.n * 4 == 20 and sv.sidecar.size // sv.n == 48
    # 64 + 180 bytes of the reference's direct path vs 68 packed
    assert abs((64 + 180) / 68 - 244.0 / 68.0) < 1e-12
    # this renderer's resident planes: 3 x 16 B geometry + 12 x 16 B colour (SH3)
    assert (3 + 12) * 16 / 68 > 3.5


def test_header_matches_the_range_scans(oracle):
    # packed_atlas.rs:728-739: metadata scans equal the packing's ranges
    sc = sample_scene(8, 3)
    sc["scale_xyz"][0] = [-7.0, -2.0, 4.0]
    sc["scale_xyz"][7] = [5.0, -3.0, 2.0]
    sv = oracle.PackedSceneView(sc)
    assert sv.header[6] == np.float32(-7.0)
    assert sv.header[7] == np.float32(5.0) - np.float32(-7.0)
    rest = sc["sh_rest"].reshape(8, 3, 15)
    for ch in range(3):
        assert sv.header[8 + ch] == np.abs(rest[:, ch, :]).max()


def test_position_roundtrip(oracle):
    # packed_atlas.rs:753-769
    sc = sample_scene(8, 0)
    sv = oracle.PackedSceneView(sc)
    assert np.abs(sv.pos.reshape(-1, 3) - sc["positions"]).max() < 1e-3


@pytest.mark.parametrize("q", [
    [0.0, 0.0, 0.0, 1.0], [0.1, -0.2, 0.3, 0.9], [0.5, 0.5, 0.5, 0.5], [-0.3, 0.1, 0.2, 0.9],
    [0.9, -0.2, 0.1, -0.3], [-0.7, 0.1, 0.2, 0.1], [0.1, 0.8, -0.2, -0.4]])
def test_rotation_roundtrip_through_the_covariance(oracle, q):
    # packed_atlas.rs:771-797: orientation survives the smallest-three packing
    # (q and -q alike); checked on the decoded covariance R diag(s^2) R^T.
    sc = sample_scene(1, 0)
    sc["rotation_xyzw"][0] = q
    sc["scale_xyz"][0] = [-1.0, -2.0, -3.0]
    sv = oracle.PackedSceneView(sc)
    qn = np.asarray(q, np.float64) / np.linalg.norm(q)
    x, y, z, w = qn
    R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                  [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                  [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
    S = np.diag(np.exp(2 * np.array([-1.0, -2.0, -3.0])))
    want = R @ S @ R.T
    c = sv.cov.astype(np.float64)
    got = np.array([[c[0], c[1], c[2]], [c[1], c[3], c[4]], [c[2], c[4], c[5]]])
    assert np.abs(got - want).max() < 0.03 * np.abs(want).max()


def test_sh_sidecar_roundtrip(oracle):
    # packed_atlas.rs:799-846
    for degree in range(4):
        sc = sample_scene(4, degree)
        sv = oracle.PackedSceneView(sc)
        if degree == 0:
            assert not sv.sidecar.any()
            continue
        assert np.abs(sv.rest - sc["sh_rest"]).max() < 0.03
        pc = (degree + 1) ** 2 - 1
        side = sv.sidecar.reshape(-1, 48)[:, :45].reshape(-1, 3, 15)
        assert not side[:, :, pc:].any()


def test_colour_opacity_and_scale_codecs(oracle):
    # packed_atlas.rs:860-891 (rgb10 and codec round trips)
    sc = sample_scene(5, 0)
    sc["opacity"][:] = [-4.0, -1.0, 0.0, 1.0, 3.0]
    sc["scale_xyz"][:, 0] = [-4.0, -1.0, 0.0, 1.0, 3.0]
    sv = oracle.PackedSceneView(sc)
    assert np.isfinite(sv.alpha[:5]).all()
    want_alpha = 1.0 / (1.0 + np.exp(-sc["opacity"].astype(np.float64)))
    assert np.abs(sv.alpha[:5] - want_alpha).max() <= 0.5 / 255 + 1e-6
    # baked DC colour: C0 dc + 0.5 within one RGB10 step
    c0 = 0.28209479177387814
    rgb = c0 * sc["color_dc"].astype(np.float64) + 0.5
    got = c0 * sv.dc.reshape(-1, 3).astype(np.float64) + 0.5
    assert np.abs(got - rgb).max() < 1.0 / 1023 + 1e-6
    # log scales within 0.01 (range -4..3 over 1,023 steps): x axis of an
    # identity rotation is the first variance
    dec = 0.5 * np.log(sv.cov.reshape(-1, 6)[:, 0].astype(np.float64))
    assert np.abs(dec - sc["scale_xyz"][:, 0]).max() < 0.01
    assert math.isfinite(float(sv.extent[:5].sum()))


def test_refined_constant_division_is_exact_over_the_decode_ranges(oracle):
    """The CUDA packed decode divides by its constants as a product with
    RN(1/d) and one fma correction; over every dividend it meets, that equals
    the IEEE quotient the oracle (and the reference) computes."""
    ints = lambda lo, hi: np.arange(lo, hi + 1, dtype=np.float32)
    assert oracle.const_div_mismatches(127.0, ints(-127, 127)) == 0
    assert oracle.const_div_mismatches(255.0, ints(0, 255)) == 0
    assert oracle.const_div_mismatches(1023.0, ints(0, 1023)) == 0
    assert oracle.const_div_mismatches(65535.0, ints(0, 65535)) == 0
    levels = ints(0, 1023) / np.float32(1023.0) - np.float32(0.5)
    assert oracle.const_div_mismatches(np.float32(0.28209479177387814), levels) == 0
