"""PLY ingestion on the device (gsplat_context_load_scene_path with a binary
body): the resident scene planes equal the host load path's (gsplat_ply_load,
then the host precompute and upload) bit for bit, for both byte orders, every
PLY scalar type, extra and duplicate properties, SH degrees 0-4 and bodies
spanning several chunks; the loader's error codes and messages are kept, and a
failed load leaves the previous scene in place."""

import numpy as np
import pytest

import gsplat_ffi as ffi
import gsplat_scenes

pytestmark = pytest.mark.gpu

PLY_TYPES = {np.dtype("i1"): "char", np.dtype("u1"): "uchar", np.dtype("i2"): "short",
             np.dtype("u2"): "ushort", np.dtype("i4"): "int", np.dtype("u4"): "uint",
             np.dtype("f4"): "float", np.dtype("f8"): "double"}


def write_ply(path, props, big_endian=False, vertices=None, truncate=0):
    """props: list of (name, numpy dtype, values[n]) in record order."""
    n = len(props[0][2]) if vertices is None else vertices
    order = ">" if big_endian else "<"
    rec = np.dtype([(f"p{k}", order + np.dtype(dt).str[1:]) for k, (_, dt, _) in enumerate(props)])
    body = np.zeros(len(props[0][2]), rec)
    for k, (_, dt, vals) in enumerate(props):
        body[f"p{k}"] = np.asarray(vals).astype(dt)
    fmt = "binary_big_endian" if big_endian else "binary_little_endian"
    head = f"ply\nformat {fmt} 1.0\ncomment written by the ingestion test\nelement vertex {n}\n"
    head += "".join(f"property {PLY_TYPES[np.dtype(dt)]} {name}\n" for name, dt, _ in props)
    head += "end_header\n"
    data = body.tobytes()
    with open(path, "wb") as f:
        f.write(head.encode())
        f.write(data[:len(data) - truncate])


def scene_props(rng, n, degree, types=None, extra=True):
    """Standard 3DGS vertex properties with random values of the given types."""
    types = types or {}
    t = lambda name: types.get(name, np.float32)
    props = [("x", t("pos"), rng.normal(0, 1, n)), ("y", t("pos"), rng.normal(0, 1, n)),
             ("z", t("pos"), rng.normal(0, 1, n) + 4.0)]
    if extra:
        props += [("nx", np.float32, np.zeros(n)), ("ny", np.float32, np.zeros(n)),
                  ("nz", np.float32, np.zeros(n))]
    props += [(f"f_dc_{k}", t("dc"), rng.normal(0, 0.5, n)) for k in range(3)]
    rest = 3 * ((degree + 1) ** 2 - 1)
    props += [(f"f_rest_{k}", t("rest"), rng.normal(0, 0.2, n)) for k in range(rest)]
    props += [("opacity", t("opacity"), rng.normal(0.5, 2.0, n))]
    props += [(f"scale_{k}", t("scale"), rng.normal(-4.0, 1.0, n)) for k in range(3)]
    q = rng.normal(size=(n, 4))
    props += [(f"rot_{k}", t("rot"), q[:, k]) for k in range(4)]
    if extra:
        props += [("label", np.uint8, rng.integers(0, 255, n))]
    return props


def _planes(ctx):
    return ctx.debug_scene()


def _host_planes(path, w=64, h=64):
    with ffi.Context(w, h) as ctx:
        ctx.load_scene(ffi.ply_load(path))
        return _planes(ctx)


def _device_planes(path, w=64, h=64):
    with ffi.Context(w, h) as ctx:
        ctx.load_scene_path(path)
        return _planes(ctx)


def _same_bits(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("degree,big,types", [
    (3, False, None),
    (0, False, None),
    (1, True, None),
    (2, False, {"pos": np.float64, "rot": np.int16, "dc": np.int32, "opacity": np.int8}),
    (4, True, {"pos": np.float64, "scale": np.float64, "rest": np.float64, "rot": np.uint16}),
])
def test_device_decode_equals_host_path(tmp_path, degree, big, types):
    rng = np.random.default_rng(100 + degree)
    path = str(tmp_path / "scene.ply")
    write_ply(path, scene_props(rng, 3001, degree, types), big_endian=big)
    assert _same_bits(_device_planes(path), _host_planes(path))


def test_multi_chunk_body_and_rendering(tmp_path):
    """A 300,000-vertex SH3 body (several 32 MiB chunks): equal planes, and
    the same image and visible count through both paths."""
    rng = np.random.default_rng(7)
    path = str(tmp_path / "big.ply")
    write_ply(path, scene_props(rng, 300_000, 3))
    cam = gsplat_scenes.camera((0.0, 0.5, -3.0), (0.0, 0.0, 4.0), 60.0)
    out = []
    for device in (True, False):
        with ffi.Context(320, 240) as ctx:
            if device:
                ctx.load_scene_path(path)
            else:
                ctx.load_scene(ffi.ply_load(path))
            ctx.set_camera(cam)
            ctx.render_frame()
            out.append((_planes(ctx), ctx.readback_rgba8(), ctx.stats().visible_count))
    assert _same_bits(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1]) and out[0][2] == out[1][2] > 0


def test_duplicate_names_and_infinite_opacity(tmp_path):
    rng = np.random.default_rng(3)
    n = 257
    props = scene_props(rng, n, 1)
    op = np.array(props[[p[0] for p in props].index("opacity")][2], np.float32)
    op[::7] = np.inf
    op[3::7] = -np.inf
    props = [(name, dt, op if name == "opacity" else v) for name, dt, v in props]
    # a later duplicate of "x" overrides the earlier one
    props.append(("x", np.float32, rng.normal(5, 1, n)))
    path = str(tmp_path / "dup.ply")
    write_ply(path, props)
    dev, host = _device_planes(path), _host_planes(path)
    assert _same_bits(dev, host)
    alpha = dev[:4 * n].reshape(-1, 4)[:, 3]
    # +-inf logits are read as +-16
    assert alpha[0] > 0.9999 and 0.0 < alpha[3] < 1e-6


def test_ascii_body_still_loads(tmp_path):
    path = str(tmp_path / "a.ply")
    with open(path, "w") as f:
        f.write("ply\nformat ascii 1.0\nelement vertex 2\n")
        for p in ("x", "y", "z", "opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1",
                  "rot_2", "rot_3", "f_dc_0", "f_dc_1", "f_dc_2"):
            f.write(f"property float {p}\n")
        f.write("end_header\n")
        f.write("0 0 3 1 -3 -3 -3 1 0 0 0 0.5 0.5 0.5\n")
        f.write("0.2 0.1 4 2 -2 -3 -3 1 0.1 0 0 0.1 0.2 0.3\n")
    assert _same_bits(_device_planes(path), _host_planes(path))


@pytest.mark.parametrize("field,where", [("rot_2", 11), ("f_rest_5", 900), ("f_dc_1", 0),
                                         ("x", 2999), ("scale_1", 1500), ("opacity", 42)])
def test_non_finite_values_fail_like_the_loader(tmp_path, field, where):
    rng = np.random.default_rng(5)
    props = scene_props(rng, 3000, 1)
    props = [(name, dt, np.where(np.arange(3000) == where, np.nan, v) if name == field else v)
             for name, dt, v in props]
    path = str(tmp_path / "nan.ply")
    write_ply(path, props)
    good = str(tmp_path / "good.ply")
    write_ply(good, scene_props(rng, 100, 0))
    with ffi.Context(64, 64) as ctx:
        ctx.load_scene_path(good)
        before = _planes(ctx)
        with pytest.raises(ffi.GsplatError) as e:
            ctx.load_scene_path(path)
        assert e.value.code == ffi.PARSE_FAILED
        assert "failed to parse numeric value" in e.value.message
        assert _same_bits(_planes(ctx), before)  # the previous scene stays loaded
        ctx.render_frame()
    with pytest.raises(ffi.GsplatError) as e:
        ffi.ply_load(path)
    assert e.value.code == ffi.PARSE_FAILED


def test_header_and_body_errors(tmp_path):
    rng = np.random.default_rng(9)
    cases = []
    p = str(tmp_path / "short.ply")
    write_ply(p, scene_props(rng, 50, 0), truncate=3)
    cases.append((p, ffi.PARSE_FAILED))
    p = str(tmp_path / "missing.ply")
    write_ply(p, [pr for pr in scene_props(rng, 50, 0) if pr[0] != "scale_2"])
    cases.append((p, ffi.PARSE_FAILED))
    p = str(tmp_path / "many.ply")
    write_ply(p, scene_props(rng, 4, 0), vertices=5_000_001)
    cases.append((p, ffi.UNSUPPORTED))
    cases.append((str(tmp_path / "absent.ply"), ffi.NOT_FOUND))
    with ffi.Context(64, 64) as ctx:
        for path, code in cases:
            with pytest.raises(ffi.GsplatError) as e:
                ctx.load_scene_path(path)
            assert e.value.code == code, path
            with pytest.raises(ffi.GsplatError) as e2:
                ffi.ply_load(path)
            assert e2.value.code == code, path
            # same message, after the entry point's own prefix
            assert e.value.message.split(": ", 1)[-1] == e2.value.message.split(": ", 1)[-1], path


def test_written_scene_loads_as_the_in_memory_scene(tmp_path):
    """gsplat_scenes.write_ply inverts the loader's conversions, so the device
    ingestion of the file gives the planes of the in-memory scene."""
    scene, cam, w, h = gsplat_scenes.config2(seed=3, n=20_000)
    path = str(tmp_path / "c2.ply")
    gsplat_scenes.write_ply(path, scene)
    with ffi.Context(64, 64) as ctx:
        ctx.load_scene(scene)
        mem = _planes(ctx)
    assert _same_bits(_device_planes(path), mem)
