"""Host-side checks of libgsplat_ffi_c.so that need no GPU: the library loads
and exports every symbol of include/*.h, the v0.1 ABI defaults and error
semantics, and the PLY loader against the reference's known answers."""

import ctypes
import json
import os
import re
import subprocess

import numpy as np
import pytest

import gsplat_ffi as ffi
import gsplat_scenes
from conftest import GOLDEN, ROOT


def _header_functions():
    names = set()
    for h in ("gsplat.h", "gsplat_cuda.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(gsplat_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_header_symbol():
    L = ffi.lib()
    declared = _header_functions()
    assert len(declared) >= 50
    for name in declared:
        assert hasattr(L, name), name
    assert declared == set(ffi.exported_names())
    out = subprocess.run(["nm", "-D", "--defined-only", ffi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (gsplat_[a-z0-9_]+)", out))
    assert declared <= exported


def test_abi_struct_sizes():
    assert ctypes.sizeof(ffi.GsplatConfig) == 12
    assert ctypes.sizeof(ffi.GsplatStats) == 24
    assert ctypes.sizeof(ffi.GsplatCamera) == 40
    assert ffi.PROJECTED_DTYPE.itemsize == 64
    assert ctypes.sizeof(ffi.GsplatBatchView) == 56
    assert ctypes.sizeof(ffi.GsplatBatchViewStats) == 16
    assert ctypes.sizeof(ffi.GsplatBatchTimes) == 32
    assert ctypes.sizeof(ffi.GsplatServeConfig) == 48
    assert ctypes.sizeof(ffi.GsplatTuneResult) == 32
    assert ctypes.sizeof(ffi.GsplatRequestInfo) == 32
    assert ctypes.sizeof(ffi.GsplatServeStats) == 176


def test_versions_defaults_and_messages(oracle):
    L = ffi.lib()
    assert (L.gsplat_version_major(), L.gsplat_version_minor()) == (0, 1)
    msgs = {0: b"ok", 1: b"invalid argument", 2: b"not found", 3: b"parse failed",
            4: b"unsupported", 5: b"scene not loaded", 100: b"internal error", 7: b"unknown error"}
    for code, text in msgs.items():
        assert L.gsplat_error_message(code) == text
    cfg = L.gsplat_config_default()
    assert (cfg.width, cfg.height, cfg.mode) == (1280, 720, 0)
    cam = L.gsplat_camera_default()
    ref = gsplat_scenes.default_camera()
    assert list(cam.position) == [0, 0, 0] and list(cam.rotation_xyzw) == [0, 0, 0, 1]
    assert np.float32(cam.vertical_fov_radians) == np.float32(ref["vertical_fov_radians"])
    assert np.float32(cam.near_plane) == np.float32(0.01) and cam.far_plane == 1000.0
    assert oracle.camera_validate(cam.to_dict()) == 0


def test_create_errors_without_gpu():
    L = ffi.lib()
    out = ctypes.c_void_p(1)
    assert L.gsplat_context_create(ffi.GsplatConfig(1280, 720, 1), ctypes.byref(out)) == 1
    assert not out.value
    assert L.gsplat_context_create(ffi.GsplatConfig(0, 720, 0), ctypes.byref(out)) == 1
    assert L.gsplat_context_create(ffi.GsplatConfig(1280, 720, 0), None) == 1
    assert "out_ctx is null" in ffi.last_error()
    rc = L.gsplat_context_create(ffi.GsplatConfig(64, 64, 0), ctypes.byref(out))
    if rc == 4:  # no usable CUDA device here: same code as a missing wgpu adapter
        assert not out.value
        assert "unavailable" in ffi.last_error()
    else:
        assert rc == 0
        L.gsplat_context_destroy(out)


def test_null_context_arguments():
    L = ffi.lib()
    cam = L.gsplat_camera_default()
    assert L.gsplat_context_set_camera(None, cam) == 1
    assert "ctx is null" in ffi.last_error()
    assert L.gsplat_context_set_auto_camera(None) == 1
    assert L.gsplat_context_load_scene_path(None, b"x.ply") == 1
    assert L.gsplat_context_render_frame(None) == 1
    st = ffi.GsplatStats()
    assert L.gsplat_context_get_stats(None, ctypes.byref(st)) == 1
    L.gsplat_context_destroy(None)
    assert L.gsplat_context_readback_rgba8(None, None, 0) == 1


def test_batch_null_and_no_gpu_errors():
    L = ffi.lib()
    assert L.gsplat_batch_create(None) == 1
    assert "out_batch is null" in ffi.last_error()
    L.gsplat_batch_destroy(None)
    assert L.gsplat_batch_render(None, None, 0) == 1
    assert "batch is null" in ffi.last_error()
    t = ffi.GsplatBatchTimes()
    assert L.gsplat_batch_get_times(None, ctypes.byref(t)) == 1
    assert L.gsplat_batch_set_phase_timing(None, 1) == 1
    ms = (ctypes.c_float * 6)()
    assert L.gsplat_batch_get_phase_times(None, ms, 6) == 1
    assert "batch is null" in ffi.last_error()
    out = ctypes.c_void_p(1)
    rc = L.gsplat_batch_create(ctypes.byref(out))
    if rc == 4:
        assert not out.value and "unavailable" in ffi.last_error()
    else:
        assert rc == 0
        L.gsplat_batch_destroy(out)


def test_server_null_and_no_gpu_errors():
    L = ffi.lib()
    assert L.gsplat_server_create(None, None) == 1
    L.gsplat_server_destroy(None)
    rid = ctypes.c_uint64()
    assert L.gsplat_server_submit(None, None, ctypes.byref(rid)) == 1
    assert "server is null" in ffi.last_error()
    cfg = ffi.GsplatServeConfig(0, 0, 9, 0, 0, 0, 0, 0, 0, 0)  # lanes must be 1..8
    out = ctypes.c_void_p(1)
    assert L.gsplat_server_create(ctypes.byref(cfg), ctypes.byref(out)) == 1
    assert not out.value
    cfg.lanes = 0
    rc = L.gsplat_server_create(ctypes.byref(cfg), ctypes.byref(out))
    if rc == 4:
        assert not out.value and "unavailable" in ffi.last_error()
    else:
        assert rc == 0
        L.gsplat_server_destroy(out)


def test_surface_renderer_is_unsupported():
    L = ffi.lib()
    out = ctypes.c_void_p(1)
    assert L.gsplat_surface_renderer_create_android(None, b"x.ply", 64, 64, ctypes.byref(out)) == 4
    assert not out.value
    assert L.gsplat_surface_renderer_render_frame(None) == 4
    L.gsplat_surface_renderer_destroy(None)


def test_ply_minimal_ascii_matches_golden_scene():
    got = ffi.ply_load(os.path.join(GOLDEN, "minimal_ascii.ply"))
    with open(os.path.join(GOLDEN, "minimal_ascii_scene.json")) as f:
        ref = gsplat_scenes.scene_from_json(json.load(f))
    for k in ("positions", "opacity", "scale_xyz", "rotation_xyzw", "color_dc"):
        assert np.array_equal(got[k], ref[k]), k
    assert got["sh_degree"] == 0 and got["sh_rest"] is None


def test_ply_minimal_binary_loads():
    got = ffi.ply_load(os.path.join(GOLDEN, "minimal_binary.ply"))
    assert got["positions"].shape[0] > 0
    assert np.all(np.isfinite(got["positions"]))


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_bytes(text.encode() if isinstance(text, str) else text)
    return str(p)


HEADER = ("ply\nformat ascii 1.0\nelement vertex 1\n" + "".join(
    f"property float {n}\n" for n in ["x", "y", "z", "opacity", "scale_0", "scale_1", "scale_2",
                                       "rot_0", "rot_1", "rot_2", "rot_3", "f_dc_0", "f_dc_1",
                                       "f_dc_2"]))


def test_ply_quaternion_kat(tmp_path, kats):
    k = kats["ply_quat"]
    got = ffi.ply_load(_write(tmp_path, "q.ply", k["ply"]))
    assert np.array_equal(got["rotation_xyzw"][0], np.float32(k["rotation_xyzw"]))
    assert np.array_equal(got["positions"][0], np.float32([0.0, -0.1, 1.0]))


def test_ply_sh_rest_kat(tmp_path, kats):
    k = kats["ply_sh_deg1"]
    body = "".join(f"property float f_rest_{i}\n" for i in range(9)) + "end_header\n"
    row = "0.0 0.1 1.0 0.9 1.0 1.1 1.2 1.0 0.0 0.0 0.0 0.2 0.3 0.4 " + " ".join(
        str(v) for v in k["rest_in"]) + "\n"
    got = ffi.ply_load(_write(tmp_path, "sh.ply", HEADER + body + row))
    assert got["sh_degree"] == 1
    assert got["sh_rest"][0].tolist() == [np.float32(v) for v in k["rest_out"]]
    # an incomplete f_rest set is ignored (degree 0, no rest)
    bad = "property float f_rest_0\nend_header\n" + "0 0.1 1 0.9 1 1.1 1.2 1 0 0 0 0.2 0.3 0.4 0.125\n"
    got = ffi.ply_load(_write(tmp_path, "sh0.ply", HEADER + bad))
    assert got["sh_degree"] == 0 and got["sh_rest"] is None


def test_ply_errors(tmp_path, kats):
    row = "0.0 0.1 1.0 0.9 1.0 1.1 1.2 1.0 0.0 0.0 0.0 0.2 0.3 0.4\n"
    ok = HEADER + "end_header\n" + row
    L = ffi.lib()

    def code(text, name="e.ply"):
        h = ctypes.c_void_p()
        rc = L.gsplat_ply_load(_write(tmp_path, name, text).encode(), ctypes.byref(h))
        if rc == 0:
            L.gsplat_host_scene_destroy(h)
        return rc

    assert code(ok) == 0
    assert code(ok.replace("property float opacity\n", "")) == 3
    assert "opacity" in ffi.last_error()
    assert code(ok.replace("0.0 0.1", "NaN 0.1", 1)) == 3
    assert code(ok.replace("element vertex 1", "element vertex 2")) == 3
    assert code(ok.replace("format ascii 1.0", "format ascii 2.0")) == 4
    assert code(ok.replace("property float x\n", "property list uchar int x\n")) == 4
    assert code(ok.replace("element vertex 1", "element vertex 5000001")) == 4
    assert code("not a ply\n") == 3
    h = ctypes.c_void_p()
    assert L.gsplat_ply_load(b"/nonexistent/file.ply", ctypes.byref(h)) == 2
    # infinite opacity logits clamp to +-16 (gsplat-io-ply lib.rs:18, 993-1004)
    got = ffi.ply_load(_write(tmp_path, "inf.ply", ok.replace(" 0.9 1.0 1.1", " inf 1.0 1.1", 1)))
    assert got["opacity"][0] == kats["opacity_logit_limit"]["value"]


def test_ply_binary_endianness_roundtrip(tmp_path):
    names = ["x", "y", "z", "opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1",
             "rot_2", "rot_3", "f_dc_0", "f_dc_1", "f_dc_2"]
    rng = np.random.default_rng(3)
    vals = rng.normal(size=(5, len(names))).astype(np.float32)
    out = {}
    for fmt, dt in (("binary_little_endian", "<f4"), ("binary_big_endian", ">f4")):
        head = f"ply\nformat {fmt} 1.0\nelement vertex 5\n" + "".join(
            f"property float {n}\n" for n in names) + "end_header\n"
        p = _write(tmp_path, fmt + ".ply", head.encode() + vals.astype(dt).tobytes())
        out[fmt] = ffi.ply_load(p)
    a, b = out["binary_little_endian"], out["binary_big_endian"]
    for k in ("positions", "opacity", "scale_xyz", "rotation_xyzw", "color_dc"):
        assert np.array_equal(a[k], b[k])
    assert np.array_equal(a["positions"][:, 1], -vals[:, 1])
    assert np.array_equal(a["rotation_xyzw"][:, 3], vals[:, 7])


def test_camera_look_at_matches_generator():
    c = ffi.camera_look_at([4.0, 0.5, -3.0], [0.0, 0.0, 0.0], 0.8)
    q = np.array(gsplat_scenes.look_at([4.0, 0.5, -3.0], [0.0, 0.0, 0.0]))
    assert np.allclose(np.array(c.rotation_xyzw), q, atol=1e-5)


def test_own_c_smoke_compiles(tmp_path):
    exe = tmp_path / "smoke"
    subprocess.run(["gcc", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "ffi", "ffi_smoke_cuda.c"), "-o", str(exe),
                    "-L", os.path.dirname(ffi.LIB_PATH), "-lgsplat_ffi_c",
                    "-Wl,-rpath," + os.path.dirname(ffi.LIB_PATH)], check=True)
    r = subprocess.run([str(exe)], cwd=ROOT, capture_output=True, text=True)
    assert r.returncode in (0, 3), r.stderr


def test_reference_c_smoke_links_unchanged():
    """The reference's own tests/ffi/ffi_smoke.c, built by oracle/Makefile
    (ref-smoke) from the reference tree, links against this library."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ffi_smoke")
    if not os.path.exists(exe):
        pytest.skip("reference smoke binary not built (reference tree absent)")
    r = subprocess.run([exe, os.path.join(GOLDEN, "minimal_ascii.ply")], capture_output=True,
                       text=True)
    assert r.returncode in (0, 3), r.stderr
