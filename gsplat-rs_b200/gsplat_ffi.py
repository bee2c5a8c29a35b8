"""ctypes binding of libgsplat_ffi_c.so (gsplat.h v0.1 + gsplat_cuda.h).

`Context` mirrors the reference Renderer/`gsplat_context_*` surface
(crates/gsplat-ffi-c/src/lib.rs:322-570): create / set_camera /
load_scene_path / render_frame / get_stats, plus the additive readback,
in-memory scene load and debug taps. Errors raise GsplatError carrying the
GsplatErrorCode and gsplat_last_error_message().

The library is the CUDA product; there is no fallback: when the shared
library is missing, `lib()` raises.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# GSPLAT_FFI_LIB selects another build of the library (tuning variants).
LIB_PATH = os.environ.get("GSPLAT_FFI_LIB") or os.path.join(HERE, "lib", "libgsplat_ffi_c.so")

OK = 0
INVALID_ARGUMENT = 1
NOT_FOUND = 2
PARSE_FAILED = 3
UNSUPPORTED = 4
SCENE_NOT_LOADED = 5
INTERNAL = 100

BLEND_FP32 = 0
BLEND_UNORM8 = 1


class GsplatConfig(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("mode", ctypes.c_uint32)]


class GsplatStats(ctypes.Structure):
    _fields_ = [("frame_ms", ctypes.c_float), ("preprocess_ms", ctypes.c_float),
                ("sort_ms", ctypes.c_float), ("raster_ms", ctypes.c_float),
                ("visible_count", ctypes.c_uint32), ("drawn_count", ctypes.c_uint32)]


class GsplatCamera(ctypes.Structure):
    _fields_ = [("position", ctypes.c_float * 3), ("rotation_xyzw", ctypes.c_float * 4),
                ("vertical_fov_radians", ctypes.c_float), ("near_plane", ctypes.c_float),
                ("far_plane", ctypes.c_float)]

    @classmethod
    def from_dict(cls, d):
        c = cls()
        c.position[:] = [float(v) for v in d["position"]]
        c.rotation_xyzw[:] = [float(v) for v in d["rotation_xyzw"]]
        c.vertical_fov_radians = float(d["vertical_fov_radians"])
        c.near_plane = float(d["near_plane"])
        c.far_plane = float(d["far_plane"])
        return c

    def to_dict(self):
        return {"position": list(self.position), "rotation_xyzw": list(self.rotation_xyzw),
                "vertical_fov_radians": self.vertical_fov_radians,
                "near_plane": self.near_plane, "far_plane": self.far_plane}


class GsplatSurfaceSortStats(ctypes.Structure):
    _fields_ = [("camera_revision", ctypes.c_uint64), ("applied_order_revision", ctypes.c_uint64),
                ("scheduled_revision", ctypes.c_uint64), ("completed_revision", ctypes.c_uint64),
                ("presented_order_revision_lag", ctypes.c_uint32),
                ("observed_result_revision_lag", ctypes.c_uint32), ("flags", ctypes.c_uint32)]


_f32p = ctypes.POINTER(ctypes.c_float)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u8p = ctypes.POINTER(ctypes.c_uint8)


class GsplatSceneDesc(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64), ("sh_degree", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("positions", _f32p), ("opacity", _f32p),
                ("scale_xyz", _f32p), ("rotation_xyzw", _f32p), ("color_dc", _f32p),
                ("sh_rest", _f32p)]


class GsplatFrameCounts(ctypes.Structure):
    _fields_ = [("visible", ctypes.c_uint64), ("drawn", ctypes.c_uint64),
                ("tile_keys", ctypes.c_uint64), ("key_capacity", ctypes.c_uint64),
                ("tiles_x", ctypes.c_uint32), ("tiles_y", ctypes.c_uint32),
                ("tile_size", ctypes.c_uint32), ("blend_mode", ctypes.c_uint32),
                ("preprocess_ms", ctypes.c_float), ("sort_ms", ctypes.c_float),
                ("raster_ms", ctypes.c_float), ("frame_ms", ctypes.c_float),
                ("frame_reruns", ctypes.c_uint32), ("sort_refreshed", ctypes.c_uint32)]


class GsplatBatchView(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_uint32), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("camera", GsplatCamera)]


class GsplatBatchViewStats(ctypes.Structure):
    _fields_ = [("visible_count", ctypes.c_uint32), ("drawn_count", ctypes.c_uint32),
                ("tile_pairs", ctypes.c_uint32), ("group", ctypes.c_uint32)]


class GsplatBatchTimes(ctypes.Structure):
    _fields_ = [("device_ms", ctypes.c_float), ("wall_ms", ctypes.c_float),
                ("groups", ctypes.c_uint32), ("reruns", ctypes.c_uint32),
                ("kernel_launches", ctypes.c_uint32), ("graph_launches", ctypes.c_uint32),
                ("tile_pairs", ctypes.c_uint64)]


class GsplatServeConfig(ctypes.Structure):
    _fields_ = [("scene_budget_bytes", ctypes.c_uint64), ("work_budget_bytes", ctypes.c_uint64),
                ("lanes", ctypes.c_uint32), ("max_views_per_batch", ctypes.c_uint32),
                ("tile_size", ctypes.c_uint32), ("raster_chunk", ctypes.c_uint32),
                ("raster_blocks_per_sm", ctypes.c_uint32), ("result_pool_mib", ctypes.c_uint32),
                ("max_queue_ms", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class GsplatTuneResult(ctypes.Structure):
    _fields_ = [("tile_size", ctypes.c_uint32), ("chunk", ctypes.c_uint32),
                ("blocks_per_sm", ctypes.c_uint32), ("candidates", ctypes.c_uint32),
                ("best_ms", ctypes.c_float), ("default_ms", ctypes.c_float),
                ("from_cache", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class GsplatRequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_uint32), ("error_code", ctypes.c_int32),
                ("batch_views", ctypes.c_uint32), ("visible_count", ctypes.c_uint32),
                ("drawn_count", ctypes.c_uint32), ("tile_pairs", ctypes.c_uint32),
                ("latency_ms", ctypes.c_float), ("queue_ms", ctypes.c_float)]


class GsplatServeStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("reruns", ctypes.c_uint64), ("peak_admitted_bytes", ctypes.c_uint64),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
                ("views_per_s", ctypes.c_double), ("mean_batch_views", ctypes.c_double),
                ("device_ms", ctypes.c_double), ("launch_ms", ctypes.c_double),
                ("retire_ms", ctypes.c_double), ("graph_captures", ctypes.c_uint64),
                ("pinned_slabs", ctypes.c_uint64), ("capture_ms", ctypes.c_double),
                ("pinned_alloc_ms", ctypes.c_double), ("workspace_regrowths", ctypes.c_uint64),
                ("regrowth_ms", ctypes.c_double), ("shed", ctypes.c_uint64)]


REQUEST_QUEUED, REQUEST_RUNNING, REQUEST_DONE, REQUEST_FAILED = 0, 1, 2, 3

PROJECTED_DTYPE = np.dtype([("center_ndc", "<f4", 2), ("axis_u", "<f4", 2), ("axis_v", "<f4", 2),
                            ("color", "<f4", 4), ("extent_scale", "<f4"), ("depth", "<f4"),
                            ("flags", "<u4"), ("tile_x0", "<u2"), ("tile_y0", "<u2"),
                            ("tile_x1", "<u2"), ("tile_y1", "<u2"), ("reserved", "<u4")])

# (name, restype, argtypes) of every exported function.
_SIGS = [
    ("gsplat_version_major", ctypes.c_uint32, []),
    ("gsplat_version_minor", ctypes.c_uint32, []),
    ("gsplat_error_message", ctypes.c_char_p, [ctypes.c_int32]),
    ("gsplat_last_error_message", ctypes.c_char_p, []),
    ("gsplat_config_default", GsplatConfig, []),
    ("gsplat_camera_default", GsplatCamera, []),
    ("gsplat_context_create", ctypes.c_int32, [GsplatConfig, ctypes.POINTER(ctypes.c_void_p)]),
    ("gsplat_context_destroy", None, [ctypes.c_void_p]),
    ("gsplat_context_set_camera", ctypes.c_int32, [ctypes.c_void_p, GsplatCamera]),
    ("gsplat_context_set_auto_camera", ctypes.c_int32, [ctypes.c_void_p]),
    ("gsplat_context_load_scene_path", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_char_p]),
    ("gsplat_context_render_frame", ctypes.c_int32, [ctypes.c_void_p]),
    ("gsplat_context_get_stats", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(GsplatStats)]),
    ("gsplat_surface_renderer_create_android", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32,
      ctypes.POINTER(ctypes.c_void_p)]),
    ("gsplat_surface_renderer_create_android_with_geometry_path", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
      ctypes.POINTER(ctypes.c_void_p)]),
    ("gsplat_surface_renderer_create_uikit", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32,
      ctypes.POINTER(ctypes.c_void_p)]),
    ("gsplat_surface_renderer_create_uikit_with_geometry_path", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32,
      ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p)]),
    ("gsplat_surface_renderer_destroy", None, [ctypes.c_void_p]),
    ("gsplat_surface_renderer_resize", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]),
    ("gsplat_surface_renderer_set_sort_interval", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_surface_renderer_set_geometry_path", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_surface_renderer_set_gpu_preproject", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_surface_renderer_set_gpu_preproject_double_buffer", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_surface_renderer_set_async_sort", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_surface_renderer_set_async_geometry", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_surface_renderer_set_instance_buffer_count", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_surface_renderer_set_frame_latency", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_surface_renderer_reset_camera", ctypes.c_int32, [ctypes.c_void_p]),
    ("gsplat_surface_renderer_orbit", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_float, ctypes.c_float]),
    ("gsplat_surface_renderer_zoom", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_float]),
    ("gsplat_surface_renderer_pan", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_float, ctypes.c_float]),
    ("gsplat_surface_renderer_render_frame", ctypes.c_int32, [ctypes.c_void_p]),
    ("gsplat_surface_renderer_get_stats", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(GsplatStats)]),
    ("gsplat_surface_renderer_get_sort_stats", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.POINTER(GsplatSurfaceSortStats)]),
    ("gsplat_context_set_size", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]),
    ("gsplat_context_get_config", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(GsplatConfig)]),
    ("gsplat_context_get_camera", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(GsplatCamera)]),
    ("gsplat_context_set_blend_mode", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_context_set_tile_size", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_context_set_debug_taps", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_context_set_cuda_graph", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_context_set_raster_config", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]),
    ("gsplat_context_set_sort_interval", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_context_set_frame_lanes", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_context_load_scene_buffers", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.POINTER(GsplatSceneDesc)]),
    ("gsplat_context_readback_rgba8", ctypes.c_int32, [ctypes.c_void_p, _u8p, ctypes.c_uint64]),
    ("gsplat_context_readback_rgba8_async", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]),
    ("gsplat_context_get_frame_counts", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.POINTER(GsplatFrameCounts)]),
    ("gsplat_context_get_phase_times", ctypes.c_int32,
     [ctypes.c_void_p, _f32p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]),
    ("gsplat_context_render_frame_async", ctypes.c_int32, [ctypes.c_void_p]),
    ("gsplat_context_sync", ctypes.c_int32, [ctypes.c_void_p]),
    ("gsplat_context_get_stream", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("gsplat_context_debug_order", ctypes.c_int32,
     [ctypes.c_void_p, _u32p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    ("gsplat_context_debug_scene", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    ("gsplat_context_debug_packed_scene", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
      ctypes.POINTER(ctypes.c_uint64)]),
    ("gsplat_context_load_scene_packed", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p]),
    ("gsplat_batch_add_scene_packed", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32)]),
    ("gsplat_server_add_scene_packed", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32)]),
    ("gsplat_context_debug_coverage", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    ("gsplat_context_debug_projected", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    ("gsplat_context_debug_tile_pairs", ctypes.c_int32,
     [ctypes.c_void_p, _u32p, _u32p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    ("gsplat_context_debug_tile_ranges", ctypes.c_int32,
     [ctypes.c_void_p, _u32p, ctypes.c_uint64, _u32p, ctypes.c_uint64,
      ctypes.POINTER(ctypes.c_uint64)]),
    ("gsplat_cuda_sort_values_by_keys", ctypes.c_int32, [_u32p, _u32p, ctypes.c_uint64]),
    ("gsplat_cuda_sort_pairs", ctypes.c_int32, [_u32p, _u32p, ctypes.c_uint64]),
    ("gsplat_cuda_sort_values_by_keys_noalloc", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]),
    ("gsplat_batch_create", ctypes.c_int32, [ctypes.POINTER(ctypes.c_void_p)]),
    ("gsplat_batch_destroy", None, [ctypes.c_void_p]),
    ("gsplat_batch_set_scene_budget", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint64]),
    ("gsplat_batch_add_scene_buffers", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.POINTER(GsplatSceneDesc), _u32p]),
    ("gsplat_batch_add_scene_path", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_char_p, _u32p]),
    ("gsplat_batch_set_tile_size", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_batch_set_blend_mode", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_batch_set_limits", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
    ("gsplat_batch_set_raster_config", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]),
    ("gsplat_batch_autotune", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.POINTER(GsplatBatchView), ctypes.c_uint32, ctypes.c_char_p,
      ctypes.c_uint32, ctypes.POINTER(GsplatTuneResult)]),
    ("gsplat_batch_render", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.POINTER(GsplatBatchView), ctypes.c_uint32]),
    ("gsplat_batch_get_times", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(GsplatBatchTimes)]),
    ("gsplat_batch_set_phase_timing", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("gsplat_batch_get_phase_times", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.c_uint32]),
    ("gsplat_batch_get_view_stats", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(GsplatBatchViewStats)]),
    ("gsplat_batch_readback_rgba8", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint32, _u8p, ctypes.c_uint64]),
    ("gsplat_batch_image_device", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p),
      ctypes.POINTER(ctypes.c_uint64)]),
    ("gsplat_batch_get_stream", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("gsplat_server_create", ctypes.c_int32,
     [ctypes.POINTER(GsplatServeConfig), ctypes.POINTER(ctypes.c_void_p)]),
    ("gsplat_server_destroy", None, [ctypes.c_void_p]),
    ("gsplat_server_add_scene_buffers", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.POINTER(GsplatSceneDesc), _u32p]),
    ("gsplat_server_add_scene_path", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_char_p, _u32p]),
    ("gsplat_server_submit", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.POINTER(GsplatBatchView), ctypes.POINTER(ctypes.c_uint64)]),
    ("gsplat_server_poll", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(GsplatRequestInfo)]),
    ("gsplat_server_wait", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(GsplatRequestInfo)]),
    ("gsplat_server_read_rgba8", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint64, _u8p, ctypes.c_uint64]),
    ("gsplat_server_release", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint64]),
    ("gsplat_server_get_stats", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(GsplatServeStats)]),
    ("gsplat_server_reset_stats", ctypes.c_int32, [ctypes.c_void_p]),
    ("gsplat_ply_load", ctypes.c_int32, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("gsplat_host_scene_destroy", None, [ctypes.c_void_p]),
    ("gsplat_host_scene_view", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(GsplatSceneDesc)]),
    ("gsplat_camera_look_at", ctypes.c_int32,
     [_f32p, _f32p, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.POINTER(GsplatCamera)]),
    ("gsplat_cuda_device_info", ctypes.c_int32,
     [ctypes.c_char_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32),
      ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]),
    ("gsplat_cuda_measure_fp32_peak", ctypes.c_int32,
     [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
]

_lib = None


def lib():
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with gsplat-rs_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_names():
    return [s[0] for s in _SIGS]


class GsplatError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{message} (code {code})")
        self.code = code
        self.message = message


def check(rc):
    if rc != 0:
        raise GsplatError(rc, lib().gsplat_last_error_message().decode())
    return rc


def last_error():
    return lib().gsplat_last_error_message().decode()


class SceneDesc:
    """Keeps contiguous f32 copies of a SceneBuffers-shaped dict alive."""

    def __init__(self, scene):
        n = int(np.asarray(scene["positions"]).reshape(-1, 3).shape[0])
        self.arrays = {}
        for k in ("positions", "opacity", "scale_xyz", "rotation_xyzw", "color_dc"):
            self.arrays[k] = np.ascontiguousarray(scene[k], np.float32).reshape(-1)
        rest = scene.get("sh_rest")
        self.arrays["sh_rest"] = None if rest is None else np.ascontiguousarray(rest, np.float32).reshape(-1)
        d = GsplatSceneDesc()
        d.count = n
        d.sh_degree = int(scene["sh_degree"])
        for k in ("positions", "opacity", "scale_xyz", "rotation_xyzw", "color_dc"):
            setattr(d, k, self.arrays[k].ctypes.data_as(_f32p))
        d.sh_rest = self.arrays["sh_rest"].ctypes.data_as(_f32p) if self.arrays["sh_rest"] is not None else None
        self.desc = d


class Context:
    """One GsplatContext: an offscreen SortedAlpha renderer on the current GPU."""

    def __init__(self, width=1280, height=720, mode=0):
        self.ptr = ctypes.c_void_p()
        check(lib().gsplat_context_create(GsplatConfig(width, height, mode), ctypes.byref(self.ptr)))
        self.width, self.height = width, height

    def close(self):
        if self.ptr:
            lib().gsplat_context_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_camera(self, cam):
        c = cam if isinstance(cam, GsplatCamera) else GsplatCamera.from_dict(cam)
        check(lib().gsplat_context_set_camera(self.ptr, c))

    def camera(self):
        c = GsplatCamera()
        check(lib().gsplat_context_get_camera(self.ptr, ctypes.byref(c)))
        return c

    def set_auto_camera(self):
        check(lib().gsplat_context_set_auto_camera(self.ptr))

    def set_size(self, width, height):
        check(lib().gsplat_context_set_size(self.ptr, width, height))
        self.width, self.height = width, height

    def set_blend_mode(self, mode):
        check(lib().gsplat_context_set_blend_mode(self.ptr, mode))

    def set_tile_size(self, tile):
        check(lib().gsplat_context_set_tile_size(self.ptr, tile))

    def set_debug_taps(self, on=True):
        check(lib().gsplat_context_set_debug_taps(self.ptr, 1 if on else 0))

    def set_cuda_graph(self, on=True):
        check(lib().gsplat_context_set_cuda_graph(self.ptr, 1 if on else 0))

    def set_raster_config(self, chunk, blocks_per_sm=0):
        check(lib().gsplat_context_set_raster_config(self.ptr, chunk, blocks_per_sm))

    def set_sort_interval(self, interval):
        check(lib().gsplat_context_set_sort_interval(self.ptr, interval))

    def set_frame_lanes(self, lanes):
        check(lib().gsplat_context_set_frame_lanes(self.ptr, lanes))

    def load_scene_path(self, path):
        check(lib().gsplat_context_load_scene_path(self.ptr, os.fsencode(path)))

    def load_scene(self, scene):
        sd = SceneDesc(scene)
        check(lib().gsplat_context_load_scene_buffers(self.ptr, ctypes.byref(sd.desc)))

    def load_scene_packed(self, scene):
        """The scene in the packed resident format (SH degree <= 3)."""
        sd = SceneDesc(scene)
        check(lib().gsplat_context_load_scene_packed(self.ptr, ctypes.byref(sd.desc)))

    def debug_packed_scene(self):
        """(table[1292] float32, hot (n, 5) uint32, sidecar (n, 48) int8 or None)."""
        n = ctypes.c_uint64()
        check(lib().gsplat_context_debug_packed_scene(self.ptr, None, None, None,
                                                      ctypes.byref(n)))
        table = np.zeros(1292, np.float32)
        hot = np.zeros((max(n.value, 1), 5), np.uint32)
        side = np.zeros((max(n.value, 1), 48), np.int8)
        check(lib().gsplat_context_debug_packed_scene(self.ptr, table.ctypes.data, hot.ctypes.data,
                                                      side.ctypes.data, ctypes.byref(n)))
        return table, hot[:n.value], side[:n.value]

    def render_frame(self):
        check(lib().gsplat_context_render_frame(self.ptr))

    def stats(self):
        s = GsplatStats()
        check(lib().gsplat_context_get_stats(self.ptr, ctypes.byref(s)))
        return s

    def frame_counts(self):
        c = GsplatFrameCounts()
        check(lib().gsplat_context_get_frame_counts(self.ptr, ctypes.byref(c)))
        return c

    PHASES = ("preprocess", "depth_sort", "emit", "tile_sort", "ranges", "raster")

    def phase_times(self):
        out = (ctypes.c_float * 16)()
        n = ctypes.c_uint32()
        check(lib().gsplat_context_get_phase_times(self.ptr, out, 16, ctypes.byref(n)))
        return dict(zip(self.PHASES, [out[k] for k in range(n.value)]))

    def readback_rgba8_async(self, out):
        """Enqueue the last frame's RGBA8 copy into `out` (a uint8 array of
        width*height*4 bytes, ideally pinned); it lands by the next sync()."""
        check(lib().gsplat_context_readback_rgba8_async(self.ptr, out.ctypes.data, out.nbytes))

    def render_frame_async(self):
        check(lib().gsplat_context_render_frame_async(self.ptr))

    def sync(self):
        check(lib().gsplat_context_sync(self.ptr))

    def stream(self):
        s = ctypes.c_void_p()
        check(lib().gsplat_context_get_stream(self.ptr, ctypes.byref(s)))
        return s.value

    def readback_rgba8(self, out=None):
        n = self.width * self.height * 4
        if out is None:
            out = np.empty(n, np.uint8)
        check(lib().gsplat_context_readback_rgba8(self.ptr, out.ctypes.data_as(_u8p), out.nbytes))
        return out.reshape(self.height, self.width, 4)

    def debug_order(self):
        n = ctypes.c_uint64()
        check(lib().gsplat_context_debug_order(self.ptr, None, 0, ctypes.byref(n)))
        out = np.empty(max(n.value, 1), np.uint32)
        check(lib().gsplat_context_debug_order(self.ptr, out.ctypes.data_as(_u32p), n.value,
                                               ctypes.byref(n)))
        return out[:n.value]

    def debug_scene(self):
        """The resident scene planes as float32: pos_alpha (n, 4), cov_a (n, 4),
        cov_b (n, 4) and the colour planes (planes, n, 4)."""
        n = ctypes.c_uint64()
        check(lib().gsplat_context_debug_scene(self.ptr, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), np.float32)
        check(lib().gsplat_context_debug_scene(self.ptr, out.ctypes.data, n.value,
                                               ctypes.byref(n)))
        return out[:n.value]

    def debug_projected(self):
        n = ctypes.c_uint64()
        check(lib().gsplat_context_debug_projected(self.ptr, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), PROJECTED_DTYPE)
        check(lib().gsplat_context_debug_projected(self.ptr, out.ctypes.data, n.value,
                                                   ctypes.byref(n)))
        return out[:n.value]

    def debug_coverage(self):
        """(n, 2) float32: log2 alpha and the coverage bound the FP32 raster
        used per splat (NaN for splats in no tile list)."""
        n = ctypes.c_uint64()
        check(lib().gsplat_context_debug_coverage(self.ptr, None, 0, ctypes.byref(n)))
        out = np.zeros((max(n.value, 1), 2), np.float32)
        check(lib().gsplat_context_debug_coverage(self.ptr, out.ctypes.data, n.value,
                                                  ctypes.byref(n)))
        return out[:n.value]

    def debug_tile_pairs(self):
        n = ctypes.c_uint64()
        check(lib().gsplat_context_debug_tile_pairs(self.ptr, None, None, 0, ctypes.byref(n)))
        t = np.empty(max(n.value, 1), np.uint32)
        i = np.empty(max(n.value, 1), np.uint32)
        check(lib().gsplat_context_debug_tile_pairs(self.ptr, t.ctypes.data_as(_u32p),
                                                    i.ctypes.data_as(_u32p), n.value,
                                                    ctypes.byref(n)))
        return t[:n.value], i[:n.value]

    def debug_tile_ranges(self, num_tiles):
        n = ctypes.c_uint64()
        r = np.empty(2 * num_tiles, np.uint32)
        check(lib().gsplat_context_debug_tile_ranges(self.ptr, r.ctypes.data_as(_u32p), r.size,
                                                     None, 0, ctypes.byref(n)))
        ids = np.empty(max(n.value, 1), np.uint32)
        check(lib().gsplat_context_debug_tile_ranges(self.ptr, r.ctypes.data_as(_u32p), r.size,
                                                     ids.ctypes.data_as(_u32p), ids.size,
                                                     ctypes.byref(n)))
        return r.reshape(-1, 2), ids[:n.value]


class Batch:
    """One GsplatBatch: resident scenes and many views rendered per call."""

    def __init__(self):
        self.ptr = ctypes.c_void_p()
        check(lib().gsplat_batch_create(ctypes.byref(self.ptr)))
        self.sizes = []

    def close(self):
        if self.ptr:
            lib().gsplat_batch_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_scene_budget(self, nbytes):
        check(lib().gsplat_batch_set_scene_budget(self.ptr, int(nbytes)))

    def add_scene(self, scene):
        sd = SceneDesc(scene)
        sid = ctypes.c_uint32()
        check(lib().gsplat_batch_add_scene_buffers(self.ptr, ctypes.byref(sd.desc), ctypes.byref(sid)))
        return sid.value

    def add_scene_packed(self, scene):
        sd = SceneDesc(scene)
        sid = ctypes.c_uint32()
        check(lib().gsplat_batch_add_scene_packed(self.ptr, ctypes.byref(sd.desc), ctypes.byref(sid)))
        return sid.value

    def add_scene_path(self, path):
        sid = ctypes.c_uint32()
        check(lib().gsplat_batch_add_scene_path(self.ptr, os.fsencode(path), ctypes.byref(sid)))
        return sid.value

    def set_tile_size(self, tile):
        check(lib().gsplat_batch_set_tile_size(self.ptr, tile))

    def set_blend_mode(self, mode):
        check(lib().gsplat_batch_set_blend_mode(self.ptr, mode))

    def set_limits(self, max_views=0, max_pairs=0, max_splats=0, max_tiles=0):
        check(lib().gsplat_batch_set_limits(self.ptr, max_views, max_pairs, max_splats, max_tiles))

    def set_raster_config(self, chunk, blocks_per_sm=0):
        check(lib().gsplat_batch_set_raster_config(self.ptr, chunk, blocks_per_sm))

    def autotune(self, views, cache_path=None, reps=3):
        arr = views if isinstance(views, ctypes.Array) else self.make_views(views)
        r = GsplatTuneResult()
        check(lib().gsplat_batch_autotune(self.ptr, arr, len(arr),
                                          os.fsencode(cache_path) if cache_path else None, reps,
                                          ctypes.byref(r)))
        return r

    @staticmethod
    def make_views(views):
        """views: iterable of (scene, camera, width, height)."""
        views = list(views)
        arr = (GsplatBatchView * len(views))()
        for k, (sid, cam, w, h) in enumerate(views):
            arr[k].scene, arr[k].width, arr[k].height, arr[k].reserved = sid, w, h, 0
            arr[k].camera = cam if isinstance(cam, GsplatCamera) else GsplatCamera.from_dict(cam)
        return arr

    def render(self, views):
        arr = views if isinstance(views, ctypes.Array) else self.make_views(views)
        check(lib().gsplat_batch_render(self.ptr, arr, len(arr)))
        self.sizes = [(arr[k].width, arr[k].height) for k in range(len(arr))]
        return self.times()

    def times(self):
        t = GsplatBatchTimes()
        check(lib().gsplat_batch_get_times(self.ptr, ctypes.byref(t)))
        return t

    def set_phase_timing(self, on):
        check(lib().gsplat_batch_set_phase_timing(self.ptr, 1 if on else 0))

    def phase_times(self):
        """Per-phase device ms of the last render (zeros unless phase-timed)."""
        out = (ctypes.c_float * len(Context.PHASES))()
        check(lib().gsplat_batch_get_phase_times(self.ptr, out, len(out)))
        return dict(zip(Context.PHASES, [float(x) for x in out]))

    def view_stats(self, view):
        s = GsplatBatchViewStats()
        check(lib().gsplat_batch_get_view_stats(self.ptr, view, ctypes.byref(s)))
        return s

    def readback_rgba8(self, view, out=None):
        w, h = self.sizes[view] if view < len(self.sizes) else (1, 1)
        if out is None:
            out = np.empty(w * h * 4, np.uint8)
        check(lib().gsplat_batch_readback_rgba8(self.ptr, view, out.ctypes.data_as(_u8p), out.nbytes))
        return out.reshape(h, w, 4)

    def image_device(self, view):
        p, n = ctypes.c_void_p(), ctypes.c_uint64()
        check(lib().gsplat_batch_image_device(self.ptr, view, ctypes.byref(p), ctypes.byref(n)))
        return p.value, n.value

    def stream(self):
        s = ctypes.c_void_p()
        check(lib().gsplat_batch_get_stream(self.ptr, ctypes.byref(s)))
        return s.value


class Server:
    """One GsplatServer: resident scenes and a continuous-batching request loop."""

    def __init__(self, lanes=0, max_views=0, tile=0, scene_budget=0, work_budget=0,
                 raster_chunk=0, raster_blocks_per_sm=0, result_pool_mib=0, max_queue_ms=0):
        cfg = GsplatServeConfig(scene_budget, work_budget, lanes, max_views, tile, raster_chunk,
                                raster_blocks_per_sm, result_pool_mib, max_queue_ms, 0)
        self.ptr = ctypes.c_void_p()
        check(lib().gsplat_server_create(ctypes.byref(cfg), ctypes.byref(self.ptr)))
        self.sizes = {}

    def close(self):
        if self.ptr:
            lib().gsplat_server_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, scene):
        sd = SceneDesc(scene)
        sid = ctypes.c_uint32()
        check(lib().gsplat_server_add_scene_buffers(self.ptr, ctypes.byref(sd.desc), ctypes.byref(sid)))
        return sid.value

    def add_scene_packed(self, scene):
        sd = SceneDesc(scene)
        sid = ctypes.c_uint32()
        check(lib().gsplat_server_add_scene_packed(self.ptr, ctypes.byref(sd.desc), ctypes.byref(sid)))
        return sid.value

    def submit(self, scene, cam, width, height):
        v = GsplatBatchView()
        v.scene, v.width, v.height, v.reserved = scene, width, height, 0
        v.camera = cam if isinstance(cam, GsplatCamera) else GsplatCamera.from_dict(cam)
        rid = ctypes.c_uint64()
        check(lib().gsplat_server_submit(self.ptr, ctypes.byref(v), ctypes.byref(rid)))
        self.sizes[rid.value] = (width, height)
        return rid.value

    def poll(self, rid):
        i = GsplatRequestInfo()
        check(lib().gsplat_server_poll(self.ptr, rid, ctypes.byref(i)))
        return i

    def wait(self, rid, timeout_ms=60000):
        i = GsplatRequestInfo()
        check(lib().gsplat_server_wait(self.ptr, rid, timeout_ms, ctypes.byref(i)))
        return i

    def read_rgba8(self, rid, out=None):
        w, h = self.sizes.get(rid, (1, 1))
        if out is None:
            out = np.empty(w * h * 4, np.uint8)
        check(lib().gsplat_server_read_rgba8(self.ptr, rid, out.ctypes.data_as(_u8p), out.nbytes))
        return out.reshape(h, w, 4)

    def release(self, rid):
        check(lib().gsplat_server_release(self.ptr, rid))
        self.sizes.pop(rid, None)

    def stats(self):
        s = GsplatServeStats()
        check(lib().gsplat_server_get_stats(self.ptr, ctypes.byref(s)))
        return s

    def reset_stats(self):
        check(lib().gsplat_server_reset_stats(self.ptr))


def sort_values_by_keys(keys, values):
    keys = np.ascontiguousarray(keys, np.uint32)
    values = np.array(values, np.uint32)
    if len(keys) != len(values):
        raise ValueError("key/value length mismatch")
    check(lib().gsplat_cuda_sort_values_by_keys(keys.ctypes.data_as(_u32p),
                                                values.ctypes.data_as(_u32p), len(keys)))
    return values


def sort_pairs(keys, values):
    keys = np.array(keys, np.uint32)
    values = np.array(values, np.uint32)
    check(lib().gsplat_cuda_sort_pairs(keys.ctypes.data_as(_u32p), values.ctypes.data_as(_u32p),
                                       len(keys)))
    return keys, values


def ply_load(path):
    """Parse a PLY file on the host; returns a SceneBuffers-shaped dict."""
    h = ctypes.c_void_p()
    check(lib().gsplat_ply_load(os.fsencode(path), ctypes.byref(h)))
    try:
        d = GsplatSceneDesc()
        check(lib().gsplat_host_scene_view(h, ctypes.byref(d)))
        n = d.count

        def arr(p, m):
            return np.ctypeslib.as_array(p, shape=(m,)).copy() if m else np.zeros(0, np.float32)

        out = {"positions": arr(d.positions, 3 * n).reshape(-1, 3),
               "opacity": arr(d.opacity, n),
               "scale_xyz": arr(d.scale_xyz, 3 * n).reshape(-1, 3),
               "rotation_xyzw": arr(d.rotation_xyzw, 4 * n).reshape(-1, 4),
               "color_dc": arr(d.color_dc, 3 * n).reshape(-1, 3),
               "sh_degree": int(d.sh_degree), "sh_rest": None}
        if d.sh_rest:
            width = 3 * ((d.sh_degree + 1) ** 2 - 1)
            out["sh_rest"] = arr(d.sh_rest, n * width).reshape(n, width)
        return out
    finally:
        lib().gsplat_host_scene_destroy(h)


def camera_look_at(position, target, fov, near=0.01, far=1000.0):
    p = (ctypes.c_float * 3)(*position)
    t = (ctypes.c_float * 3)(*target)
    c = GsplatCamera()
    check(lib().gsplat_camera_look_at(p, t, fov, near, far, ctypes.byref(c)))
    return c


def measure_fp32_peak():
    """The device's measured FP32 FMA throughput: (TFLOP/s, best launch ms)."""
    t, ms = ctypes.c_double(), ctypes.c_double()
    check(lib().gsplat_cuda_measure_fp32_peak(ctypes.byref(t), ctypes.byref(ms)))
    return t.value, ms.value


def device_info():
    name = ctypes.create_string_buffer(256)
    sm, ma, mi = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    check(lib().gsplat_cuda_device_info(name, 256, ctypes.byref(sm), ctypes.byref(ma), ctypes.byref(mi)))
    return {"name": name.value.decode(), "sm_count": sm.value, "cc": (ma.value, mi.value)}
