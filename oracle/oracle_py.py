"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker or the timed CPU
baseline, never as part of the product.
"""

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)


class OrcCamera(ctypes.Structure):
    _fields_ = [("position", ctypes.c_float * 3), ("rotation_xyzw", ctypes.c_float * 4),
                ("vertical_fov_radians", ctypes.c_float), ("near_plane", ctypes.c_float),
                ("far_plane", ctypes.c_float)]


class OrcScene(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64), ("sh_degree", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("positions", _f32p), ("opacity", _f32p),
                ("scale_xyz", _f32p), ("rotation_xyzw", _f32p), ("color_dc", _f32p),
                ("sh_rest", _f32p)]


class OrcFrameParams(ctypes.Structure):
    _fields_ = [("cam", ctypes.c_float * 3), ("view_rot", ctypes.c_float * 9)] + [
        (n, ctypes.c_float) for n in ("f", "aspect", "tan_half_fovy", "lim_x", "lim_y", "fx", "fy",
                                      "blur_x", "blur_y", "near_plane", "far_plane", "half_w",
                                      "half_h", "sx", "sy")] + [
        (n, ctypes.c_uint32) for n in ("width", "height", "tile", "tiles_x", "tiles_y",
                                       "sh_degree")]


class OrcFrameTiming(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("preprocess_ms", "sort_ms", "project_ms",
                                                "raster_ms", "total_ms")] + [
        ("visible", ctypes.c_uint64), ("drawn", ctypes.c_uint64)]


# Same layout as OrcProjected / GsplatProjectedSplat (64 bytes).
PROJECTED_DTYPE = np.dtype([("center_ndc", "<f4", 2), ("axis_u", "<f4", 2), ("axis_v", "<f4", 2),
                            ("color", "<f4", 4), ("extent_scale", "<f4"), ("depth", "<f4"),
                            ("flags", "<u4"), ("tile_x0", "<u2"), ("tile_y0", "<u2"),
                            ("tile_x1", "<u2"), ("tile_y1", "<u2"), ("reserved", "<u4")])
RECORD_DTYPE = np.dtype([(n, "<f4") for n in ("cx", "cy", "ax", "ay", "bx", "by", "s", "alpha",
                                               "cr", "cg", "cb", "log2a")])
assert PROJECTED_DTYPE.itemsize == 64 and RECORD_DTYPE.itemsize == 48

_lib = None


def build():
    """Compile the oracle with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_camera_validate.argtypes = [ctypes.POINTER(OrcCamera)]
        L.orc_camera_validate.restype = ctypes.c_int32
        L.orc_scene_validate.argtypes = [ctypes.POINTER(OrcScene), ctypes.c_uint64]
        L.orc_scene_validate.restype = ctypes.c_int32
        L.orc_view_rotation.argtypes = [_f32p, _f32p]
        L.orc_auto_camera.argtypes = [_f32p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.POINTER(OrcCamera)]
        L.orc_auto_camera.restype = ctypes.c_int32
        L.orc_camera_look_at.argtypes = [_f32p, _f32p, _f32p]
        L.orc_camera_look_at.restype = None
        L.orc_quat_inverse.argtypes = [_f32p, _f32p]
        L.orc_frame_params.argtypes = [ctypes.POINTER(OrcCamera), ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.POINTER(OrcFrameParams)]
        L.orc_pack_scene.argtypes = [ctypes.c_void_p, _f32p, _u32p, ctypes.c_void_p]
        L.orc_pack_scene.restype = None
        L.orc_unpack_scene.argtypes = [ctypes.c_uint64, ctypes.c_uint32, _f32p, _u32p,
                                       ctypes.c_void_p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p]
        L.orc_unpack_scene.restype = None
        L.orc_const_div_mismatches.argtypes = [ctypes.c_float, _f32p, ctypes.c_uint64]
        L.orc_const_div_mismatches.restype = ctypes.c_uint64
        L.orc_precompute_alpha.argtypes = [_f32p, ctypes.c_uint64, _f32p]
        L.orc_precompute_extent_scale.argtypes = [_f32p, ctypes.c_uint64, _f32p]
        L.orc_precompute_cov.argtypes = [_f32p, _f32p, ctypes.c_uint64, _f32p]
        L.orc_preprocess_visible.argtypes = [_f32p, ctypes.c_uint64, ctypes.POINTER(OrcCamera),
                                             _u32p, _u32p]
        L.orc_preprocess_visible.restype = ctypes.c_uint64
        L.orc_sort_values_by_keys.argtypes = [_u32p, _u32p, ctypes.c_uint64]
        L.orc_sort_pairs.argtypes = [_u32p, _u32p, ctypes.c_uint64]
        L.orc_radix_count.argtypes = [_u64p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int32,
                                      _u64p]
        L.orc_pack_pairs.argtypes = [_u32p, _u32p, ctypes.c_uint64, ctypes.c_int32, _u64p]
        L.orc_project_all.argtypes = [ctypes.POINTER(OrcScene), _f32p, _f32p, _f32p,
                                      ctypes.POINTER(OrcFrameParams), ctypes.c_void_p,
                                      ctypes.c_void_p]
        L.orc_build_instances.argtypes = [ctypes.POINTER(OrcScene), _f32p, _f32p,
                                          ctypes.POINTER(OrcCamera), ctypes.c_uint32,
                                          ctypes.c_uint32, _u32p, ctypes.c_uint64, _f32p, _u32p]
        L.orc_build_instances.restype = ctypes.c_uint64
        L.orc_emit_tile_pairs.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _u32p, ctypes.c_uint64,
                                          ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u32p,
                                          _u32p, ctypes.c_uint64]
        L.orc_emit_tile_pairs.restype = ctypes.c_uint64
        L.orc_tile_lists.argtypes = [_u32p, _u32p, ctypes.c_uint64, ctypes.c_uint32, _u32p, _u32p]
        L.orc_sort_u64_pairs_stable.argtypes = [_u64p, _u32p, ctypes.c_uint64]
        L.orc_exp_neg.argtypes = [ctypes.c_float]
        L.orc_exp_neg.restype = ctypes.c_float
        L.orc_raster_unorm8.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _u32p, ctypes.c_uint64,
                                        ctypes.c_uint32, ctypes.c_uint32, _u8p, ctypes.c_int32]
        L.orc_raster_f64.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _u32p, ctypes.c_uint64,
                                     ctypes.c_uint32, ctypes.c_uint32, _u8p, _f64p, ctypes.c_int32]
        L.orc_raster_unorm8_rows.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _u32p,
                                             ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                             _u8p, ctypes.c_int32, ctypes.c_uint32,
                                             ctypes.c_uint32]
        L.orc_raster_f64_rows.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _u32p, ctypes.c_uint64,
                                          ctypes.c_uint32, ctypes.c_uint32, _u8p, _f64p,
                                          ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32]
        L.orc_raster_tiles_fp32_rows.argtypes = [ctypes.c_void_p, _u32p, _u32p, ctypes.c_uint32,
                                                 ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                                 _u8p, ctypes.c_int32, ctypes.c_uint32,
                                                 ctypes.c_uint32]
        L.orc_raster_tiles_fp32.argtypes = [ctypes.c_void_p, _u32p, _u32p, ctypes.c_uint32,
                                            ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                            _u8p, ctypes.c_int32]
        L.orc_render_reference_frame.argtypes = [ctypes.POINTER(OrcScene), _f32p, _f32p, _f32p,
                                                 ctypes.POINTER(OrcCamera), ctypes.c_uint32,
                                                 ctypes.c_uint32, ctypes.c_uint32, _u8p,
                                                 ctypes.c_int32, ctypes.POINTER(OrcFrameTiming)]
        L.orc_render_reference_frame.restype = ctypes.c_int32
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def camera(cam):
    """cam: dict or object with position, rotation_xyzw, fov, near, far."""
    c = OrcCamera()
    c.position[:] = [float(v) for v in cam["position"]]
    c.rotation_xyzw[:] = [float(v) for v in cam["rotation_xyzw"]]
    c.vertical_fov_radians = float(cam["vertical_fov_radians"])
    c.near_plane = float(cam["near_plane"])
    c.far_plane = float(cam["far_plane"])
    return c


class SceneView:
    """Keeps contiguous f32 copies of a scene alive for the C side."""

    def __init__(self, scene):
        self.n = int(scene["positions"].shape[0])
        self.pos = np.ascontiguousarray(scene["positions"], np.float32).reshape(-1)
        self.opa = np.ascontiguousarray(scene["opacity"], np.float32).reshape(-1)
        self.scl = np.ascontiguousarray(scene["scale_xyz"], np.float32).reshape(-1)
        self.rot = np.ascontiguousarray(scene["rotation_xyzw"], np.float32).reshape(-1)
        self.dc = np.ascontiguousarray(scene["color_dc"], np.float32).reshape(-1)
        rest = scene.get("sh_rest")
        self.rest = None if rest is None else np.ascontiguousarray(rest, np.float32).reshape(-1)
        self.degree = int(scene["sh_degree"])
        s = OrcScene()
        s.count = self.n
        s.sh_degree = self.degree
        s.positions = _p(self.pos, _f32p)
        s.opacity = _p(self.opa, _f32p)
        s.scale_xyz = _p(self.scl, _f32p)
        s.rotation_xyzw = _p(self.rot, _f32p)
        s.color_dc = _p(self.dc, _f32p)
        s.sh_rest = _p(self.rest, _f32p) if self.rest is not None else None
        self.c = s
        n1 = max(self.n, 1)
        self.alpha = np.zeros(n1, np.float32)
        self.extent = np.zeros(n1, np.float32)
        self.cov = np.zeros(6 * n1, np.float32)
        L = lib()
        L.orc_precompute_alpha(_p(self.opa, _f32p), self.n, _p(self.alpha, _f32p))
        L.orc_precompute_extent_scale(_p(self.alpha, _f32p), self.n, _p(self.extent, _f32p))
        L.orc_precompute_cov(_p(self.scl, _f32p), _p(self.rot, _f32p), self.n, _p(self.cov, _f32p))

    def validate(self):
        rest_len = 0 if self.rest is None else self.rest.size
        return lib().orc_scene_validate(ctypes.byref(self.c), rest_len)


class PackedSceneView(SceneView):
    """A scene in the packed resident format (20-byte hot record + i8 SH
    sidecar, packed_atlas.rs), decoded as the CUDA renderer decodes it: the
    frame stages then see an ordinary scene with the decoded values."""

    def __init__(self, scene):
        super().__init__(scene)
        if self.degree > 3:
            raise ValueError("the packed format holds SH degree <= 3")
        L = lib()
        n1 = max(self.n, 1)
        self.header = np.zeros(11, np.float32)
        self.hot = np.zeros(5 * n1, np.uint32)
        self.sidecar = np.zeros(48 * n1, np.int8)
        L.orc_pack_scene(ctypes.byref(self.c), _p(self.header, _f32p), _p(self.hot, _u32p),
                         self.sidecar.ctypes.data)
        pc = (self.degree + 1) ** 2 - 1
        self.pos = np.zeros(3 * n1, np.float32)
        self.dc = np.zeros(3 * n1, np.float32)
        self.rest = np.zeros(3 * pc * n1, np.float32) if pc else None
        L.orc_unpack_scene(self.n, self.degree, _p(self.header, _f32p), _p(self.hot, _u32p),
                           self.sidecar.ctypes.data, _p(self.pos, _f32p), _p(self.alpha, _f32p),
                           _p(self.extent, _f32p), _p(self.cov, _f32p), _p(self.dc, _f32p),
                           _p(self.rest, _f32p) if pc else None)
        self.pos = self.pos[:3 * self.n]
        self.c.positions = _p(self.pos, _f32p)
        self.c.color_dc = _p(self.dc, _f32p)
        self.c.sh_rest = _p(self.rest, _f32p) if pc else None


def camera_validate(cam):
    return lib().orc_camera_validate(ctypes.byref(camera(cam)))


def auto_camera(positions, width, height):
    """gsplat_context_set_auto_camera's camera for a scene (dict of floats)."""
    pos = np.ascontiguousarray(positions, np.float32).reshape(-1)
    c = OrcCamera()
    rc = lib().orc_auto_camera(_p(pos, _f32p), pos.size // 3, width, height, ctypes.byref(c))
    if rc != 0:
        raise ValueError("empty scene")
    return {"position": list(c.position), "rotation_xyzw": list(c.rotation_xyzw),
            "vertical_fov_radians": c.vertical_fov_radians, "near_plane": c.near_plane,
            "far_plane": c.far_plane}


def camera_look_at(position, target):
    p = np.ascontiguousarray(position, np.float32)
    t = np.ascontiguousarray(target, np.float32)
    q = np.zeros(4, np.float32)
    lib().orc_camera_look_at(_p(p, _f32p), _p(t, _f32p), _p(q, _f32p))
    return q


def view_rotation(q):
    q = np.asarray(q, np.float32)
    out = np.zeros(9, np.float32)
    lib().orc_view_rotation(_p(q, _f32p), _p(out, _f32p))
    return out.reshape(3, 3)


def frame_params(cam, width, height, tile=16, sh_degree=0):
    p = OrcFrameParams()
    lib().orc_frame_params(ctypes.byref(camera(cam)), width, height, tile, sh_degree,
                           ctypes.byref(p))
    return p


def preprocess_visible(positions, cam):
    pos = np.ascontiguousarray(positions, np.float32).reshape(-1)
    n = pos.size // 3
    keys = np.zeros(max(n, 1), np.uint32)
    idx = np.zeros(max(n, 1), np.uint32)
    v = lib().orc_preprocess_visible(_p(pos, _f32p), n, ctypes.byref(camera(cam)),
                                     _p(keys, _u32p), _p(idx, _u32p))
    if v == 2**64 - 1:
        raise ValueError("invalid camera")
    return keys[:v].copy(), idx[:v].copy()


def sort_values_by_keys(keys, values):
    keys = np.ascontiguousarray(keys, np.uint32)
    values = np.array(values, np.uint32)
    if len(keys) != len(values):
        raise ValueError("length mismatch")
    lib().orc_sort_values_by_keys(_p(keys, _u32p), _p(values, _u32p), len(keys))
    return values


def sort_pairs(keys, values):
    keys = np.array(keys, np.uint32)
    values = np.array(values, np.uint32)
    lib().orc_sort_pairs(_p(keys, _u32p), _p(values, _u32p), len(keys))
    return keys, values


def radix_count(values, shift, simd):
    values = np.ascontiguousarray(values, np.uint64)
    out = np.zeros(256, np.uint64)
    lib().orc_radix_count(_p(values, _u64p), len(values), shift, int(simd), _p(out, _u64p))
    return out


class Frame:
    """Oracle evaluation of one SortedAlpha frame, stage by stage."""

    def __init__(self, sv, cam, width, height, tile=16, order=None, exact=True):
        """`order`: a back-to-front id list to draw instead of this camera's
        own (a stale order, as the reference's surface session draws between
        sort refreshes); every splat is still projected with `cam`.
        `exact`: tile pairs from exact row spans (the CUDA design) or, when
        false, from whole tile rects."""
        L = lib()
        self.width, self.height, self.tile = width, height, tile
        self.params = frame_params(cam, width, height, tile, sv.degree)
        self.keys, self.visible_ids = preprocess_visible(sv.pos.reshape(-1, 3), cam)
        if order is None:
            self.order = sort_values_by_keys(self.keys, self.visible_ids.copy())
        else:
            self.order = np.ascontiguousarray(order, np.uint32)
        n1 = max(sv.n, 1)
        self.proj = np.zeros(n1, PROJECTED_DTYPE)
        self.rec = np.zeros(n1, RECORD_DTYPE)
        L.orc_project_all(ctypes.byref(sv.c), _p(sv.alpha, _f32p), _p(sv.extent, _f32p),
                          _p(sv.cov, _f32p), ctypes.byref(self.params),
                          self.proj.ctypes.data, self.rec.ctypes.data)
        self.tiles_x = self.params.tiles_x
        self.tiles_y = self.params.tiles_y
        self.num_tiles = self.tiles_x * self.tiles_y
        v = len(self.order)
        order = np.ascontiguousarray(self.order, np.uint32) if v else np.zeros(1, np.uint32)
        k = L.orc_emit_tile_pairs(self.proj.ctypes.data, self.rec.ctypes.data, _p(order, _u32p), v,
                                  self.tiles_x, tile, int(exact), None, None, 0)
        self.pair_tiles = np.zeros(max(k, 1), np.uint32)
        self.pair_ids = np.zeros(max(k, 1), np.uint32)
        L.orc_emit_tile_pairs(self.proj.ctypes.data, self.rec.ctypes.data, _p(order, _u32p), v,
                              self.tiles_x, tile, int(exact), _p(self.pair_tiles, _u32p),
                              _p(self.pair_ids, _u32p), k)
        self.pair_tiles = self.pair_tiles[:k]
        self.pair_ids = self.pair_ids[:k]
        self.ranges = np.zeros(2 * self.num_tiles, np.uint32)
        self.tile_ids = np.zeros(max(k, 1), np.uint32)
        L.orc_tile_lists(_p(np.ascontiguousarray(self.pair_tiles) if k else np.zeros(1, np.uint32),
                            _u32p),
                         _p(np.ascontiguousarray(self.pair_ids) if k else np.zeros(1, np.uint32),
                            _u32p),
                         k, self.num_tiles, _p(self.ranges, _u32p), _p(self.tile_ids, _u32p))
        self.tile_ids = self.tile_ids[:k]
        self.ranges = self.ranges.reshape(-1, 2)
        self._order_c = order

    @property
    def visible(self):
        return len(self.order)

    @property
    def drawn(self):
        return int(np.count_nonzero(self.proj["flags"] & 2))

    # rows=(y0, y1): only those rows are composited (the others stay zero)

    def raster_unorm8(self, threads=8, rows=None):
        out = np.zeros(self.width * self.height * 4, np.uint8)
        y0, y1 = rows if rows else (0, self.height)
        lib().orc_raster_unorm8_rows(self.rec.ctypes.data, self.proj.ctypes.data,
                                     _p(self._order_c, _u32p), self.visible, self.width,
                                     self.height, _p(out, _u8p), threads, y0, y1)
        return out.reshape(self.height, self.width, 4)

    def raster_f64(self, threads=8, rows=None):
        out = np.zeros(self.width * self.height * 4, np.uint8)
        acc = np.zeros(self.width * self.height * 4, np.float64)
        y0, y1 = rows if rows else (0, self.height)
        lib().orc_raster_f64_rows(self.rec.ctypes.data, self.proj.ctypes.data,
                                  _p(self._order_c, _u32p), self.visible, self.width, self.height,
                                  _p(out, _u8p), _p(acc, _f64p), threads, y0, y1)
        return out.reshape(self.height, self.width, 4), acc.reshape(self.height, self.width, 4)

    def raster_tiles_fp32(self, threads=8, rows=None):
        out = np.zeros(self.width * self.height * 4, np.uint8)
        ids = self.tile_ids if len(self.tile_ids) else np.zeros(1, np.uint32)
        y0, y1 = rows if rows else (0, self.height)
        lib().orc_raster_tiles_fp32_rows(self.rec.ctypes.data,
                                         _p(np.ascontiguousarray(self.ranges.reshape(-1)), _u32p),
                                         _p(np.ascontiguousarray(ids), _u32p), self.width,
                                         self.height, self.tile, self.tiles_x, _p(out, _u8p),
                                         threads, y0, y1)
        return out.reshape(self.height, self.width, 4)


def build_instances(sv, cam, width, height, indices):
    idx = np.ascontiguousarray(indices, np.uint32)
    m = len(idx)
    out = np.zeros(12 * max(m, 1), np.float32)
    out_idx = np.zeros(max(m, 1), np.uint32)
    k = lib().orc_build_instances(ctypes.byref(sv.c), _p(sv.alpha, _f32p), _p(sv.cov, _f32p),
                                  ctypes.byref(camera(cam)), width, height,
                                  _p(idx if m else np.zeros(1, np.uint32), _u32p), m,
                                  _p(out, _f32p), _p(out_idx, _u32p))
    return out[:12 * k].reshape(k, 12), out_idx[:k]


def render_reference_frame(sv, cam, width, height, threads=8, rows=0):
    """The reference SortedAlpha frame on the host CPU; returns (rgba, timing).
    rows > 0 composites only the top `rows` rows (a bounded sample)."""
    out = np.zeros(width * height * 4, np.uint8)
    t = OrcFrameTiming()
    rc = lib().orc_render_reference_frame(ctypes.byref(sv.c), _p(sv.alpha, _f32p),
                                          _p(sv.extent, _f32p), _p(sv.cov, _f32p),
                                          ctypes.byref(camera(cam)), width, height, rows,
                                          _p(out, _u8p), threads, ctypes.byref(t))
    if rc != 0:
        raise ValueError("invalid camera")
    return out.reshape(height, width, 4), t


def coverage_bound(s, log2a):
    """FP32-mode coverage bound on r^2 per splat, in float32 (each operation
    rounded like the tile model in oracle_render.cpp, orc_raster_tiles_fp32):
    the reference's fragment rule (crates/gsplat-render-wgpu/shaders/
    splat_surface_direct.wgsl:336-369) keeps w = alpha e^(-4.5 r^2) > 1/256
    and |local| <= s, i.e. r^2 < (log2 alpha + 8) / (4.5 log2 e) and
    r^2 <= s^2; the bound is the largest float below the first, capped at the
    second, and -1 when the first is not positive."""
    s = np.asarray(s, np.float32)
    log2a = np.asarray(log2a, np.float32)
    s2 = s * s
    wlim = (log2a + np.float32(8.0)) / np.float32(6.49212768)
    below = np.nextafter(wlim, np.float32(0.0))
    return np.where(wlim > np.float32(0.0), np.fmin(s2, below), np.float32(-1.0)).astype(np.float32)


def exp_neg(x):
    return lib().orc_exp_neg(float(x))


def const_div_mismatches(d, x):
    x = np.ascontiguousarray(x, np.float32)
    return int(lib().orc_const_div_mismatches(float(d), _p(x, _f32p), x.size))
