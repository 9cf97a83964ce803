"""ctypes binding of libnan_b200.so (the C ABI in include/nan_b200.h).

There is no fallback: importing a tracer class without the compiled library
raises, so no CPU path can stand in for the CUDA kernels by accident.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("NAN_B200_LIBRARY", PKG / "libnan_b200.so"))

NAN_OK = 0
NAN_ERR_INVALID_ARGUMENT = 1
NAN_ERR_OUT_OF_MEMORY = 2
NAN_ERR_LIMIT = 3
NAN_ERR_CUDA = 4
NAN_ERR_NO_SCENE = 5

_STATUS_NAMES = {
    NAN_ERR_INVALID_ARGUMENT: "invalid argument",
    NAN_ERR_OUT_OF_MEMORY: "out of memory",
    NAN_ERR_LIMIT: "device limit hit",
    NAN_ERR_CUDA: "CUDA error",
    NAN_ERR_NO_SCENE: "no scene",
}


class NanError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class NanLighting(ctypes.Structure):
    _fields_ = [
        ("sun_direction", ctypes.c_float * 3),
        ("sun_cos_half_angle", ctypes.c_float),
        ("sun_color", ctypes.c_float * 3),
        ("sun_intensity", ctypes.c_float),
        ("sun_transmittance", ctypes.c_float * 3),
        ("ray_t_max", ctypes.c_float),
        ("sky_radiance", ctypes.c_float * 3),
        ("flags", ctypes.c_uint32),
        ("sky_view_lut", ctypes.c_void_p),
        ("sky_view_width", ctypes.c_uint32),
        ("sky_view_height", ctypes.c_uint32),
        ("sky_view_up", ctypes.c_float * 3),
        ("sky_view_horizon_angle", ctypes.c_float),
    ]


class NanCamera(ctypes.Structure):
    _fields_ = [
        ("position", ctypes.c_float * 3),
        ("jitter_x", ctypes.c_float),
        ("image_u", ctypes.c_float * 3),
        ("jitter_y", ctypes.c_float),
        ("image_v", ctypes.c_float * 3),
        ("near_clip", ctypes.c_float),
        ("image_w", ctypes.c_float * 3),
        ("far_clip", ctypes.c_float),
    ]


class NanSceneDesc(ctypes.Structure):
    _fields_ = [
        ("vertices", ctypes.c_void_p),
        ("vertex_count", ctypes.c_uint32),
        ("indices", ctypes.c_void_p),
        ("index_triangle_count", ctypes.c_uint32),
        ("mesh_descs", ctypes.c_void_p),
        ("mesh_count", ctypes.c_uint32),
        ("instance_descs", ctypes.c_void_p),
        ("instance_count", ctypes.c_uint32),
        ("transforms", ctypes.c_void_p),
        ("inverse_transposes", ctypes.c_void_p),
        ("transform_count", ctypes.c_uint32),
        ("materials", ctypes.c_void_p),
        ("material_count", ctypes.c_uint32),
    ]


class NanSceneInfo(ctypes.Structure):
    _fields_ = [
        ("triangle_count", ctypes.c_uint32),
        ("node_count", ctypes.c_uint32),
        ("leaf_count", ctypes.c_uint32),
        ("max_depth", ctypes.c_uint32),
        ("device_bytes", ctypes.c_uint64),
        ("build_ms", ctypes.c_double),
        ("sah_cost", ctypes.c_double),
    ]


class NanMeshColorsDesc(ctypes.Structure):
    _fields_ = [
        ("face_infos", ctypes.c_void_p),
        ("face_count", ctypes.c_uint32),
        ("instance_infos", ctypes.c_void_p),
        ("side_infos", ctypes.c_void_p),
        ("instance_count", ctypes.c_uint32),
        ("surface_prefix", ctypes.c_void_p),
        ("total_surface_texels", ctypes.c_uint32),
        ("payload_count", ctypes.c_uint32),
        ("compensation", ctypes.c_void_p),
    ]


class NanTuning(ctypes.Structure):
    _fields_ = [
        ("integrator", ctypes.c_uint32),
        ("trace_blocks_per_sm", ctypes.c_uint32),
        ("max_paths_in_flight", ctypes.c_uint32),
        ("bvh_builder", ctypes.c_uint32),
        ("bvh_width", ctypes.c_uint32),
        ("kernel_timing", ctypes.c_uint32),
        ("ray_order", ctypes.c_uint32),
        ("traversal", ctypes.c_uint32),
    ]


class NanKernelTimes(ctypes.Structure):
    _fields_ = [
        ("extend_ms", ctypes.c_double),
        ("shadow_ms", ctypes.c_double),
        ("stage_ms", ctypes.c_double),
        ("extend_launches", ctypes.c_uint64),
        ("shadow_launches", ctypes.c_uint64),
        ("stage_launches", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class NanCacheConfig(ctypes.Structure):
    _fields_ = [
        ("bounds_min", ctypes.c_float * 3),
        ("bounds_max", ctypes.c_float * 3),
        ("log2_table", ctypes.c_uint32),
        ("base_resolution", ctypes.c_uint32),
        ("max_resolution", ctypes.c_uint32),
        ("learning_rate", ctypes.c_float),
        ("beta1", ctypes.c_float),
        ("beta2", ctypes.c_float),
        ("epsilon", ctypes.c_float),
        ("loss_epsilon", ctypes.c_float),
        ("table_update", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32 * 3),
    ]


class NanCachedFrame(ctypes.Structure):
    _fields_ = [
        ("queries", ctypes.c_void_p),
        ("query_weights", ctypes.c_void_p),
        ("query_count", ctypes.c_void_p),
        ("train_points", ctypes.c_void_p),
        ("train_queries", ctypes.c_void_p),
        ("train_count", ctypes.c_uint32),
        ("train_offset", ctypes.c_uint32),
        ("train_stride", ctypes.c_uint32),
        ("train_stride_inverse", ctypes.c_uint32),
        ("cache_vertex", ctypes.c_uint32),
    ]


class NanProbeSet(ctypes.Structure):
    _fields_ = [
        ("scene", ctypes.c_void_p),
        ("probes", ctypes.c_void_p),
        ("probe_count", ctypes.c_uint32),
        ("probe_instances", ctypes.c_void_p),
        ("probe_instance_count", ctypes.c_uint32),
        ("values", ctypes.c_void_p),
        ("sample_counts", ctypes.c_void_p),
        ("self_hits", ctypes.c_void_p),
        ("radial", ctypes.c_void_p),
        ("compensation", ctypes.c_void_p),
        ("lighting", NanLighting),
    ]


class NanBatchTuning(ctypes.Structure):
    _fields_ = [
        ("stack_depth", ctypes.c_uint32),
        ("blocks_per_sm", ctypes.c_uint32),
        ("units_per_grab", ctypes.c_uint32),
        ("min_blocks_per_sm", ctypes.c_uint32),
    ]


class NanProbeLayoutDesc(ctypes.Structure):
    _fields_ = [
        ("probes", ctypes.c_void_p),
        ("probe_count", ctypes.c_uint32),
        ("node_count", ctypes.c_uint32),
        ("nodes", ctypes.c_void_p),
        ("instances", ctypes.c_void_p),
        ("instance_count", ctypes.c_uint32),
        ("triangle_vertex_probe_count", ctypes.c_uint32),
        ("triangle_vertex_probes", ctypes.c_void_p),
    ]


class NanProbeResolveOptions(ctypes.Structure):
    _fields_ = [
        ("debug_view", ctypes.c_uint32),
        ("min_gather_count", ctypes.c_uint32),
        ("use_vertex_fallback", ctypes.c_uint32),
        ("use_vertex_lighting", ctypes.c_uint32),
        ("use_radial_visibility", ctypes.c_uint32),
        ("frame_index", ctypes.c_uint32),
        ("max_density_multiplier", ctypes.c_float),
        ("vertex_lighting_rgbm_range", ctypes.c_float),
        ("vertex_lighting_rgbm", ctypes.c_void_p),
        ("vertex_lighting_target", ctypes.c_void_p),
        ("vertex_lighting_triangle_map", ctypes.c_void_p),
        ("vertex_lighting_instance_offsets", ctypes.c_void_p),
        ("vertex_lighting_vertex_count", ctypes.c_uint32),
        ("vertex_lighting_triangle_record_count", ctypes.c_uint32),
    ]


class NanWseOptions(ctypes.Structure):
    _fields_ = [("normal_cosine_threshold", ctypes.c_float), ("plane_distance_scale", ctypes.c_float)]


class NanRepairOptions(ctypes.Structure):
    _fields_ = [("min_gather_count", ctypes.c_uint32), ("max_repair_count", ctypes.c_uint32),
                ("normal_cosine_threshold", ctypes.c_float), ("weight_epsilon", ctypes.c_float)]


class NanSupportOptions(ctypes.Structure):
    _fields_ = [("normal_cosine_threshold", ctypes.c_float), ("weight_epsilon", ctypes.c_float),
                ("max_density_multiplier", ctypes.c_float), ("reserved", ctypes.c_float)]


INTEGRATORS = {"wavefront": 0, "megakernel": 1}
BVH_BUILDERS = {"sah": 0, "lbvh": 1, "ploc": 2}


class NanCounters(ctypes.Structure):
    _fields_ = [
        ("extend_rays", ctypes.c_uint64),
        ("shadow_rays", ctypes.c_uint64),
        ("units", ctypes.c_uint64),
        ("paths", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


# (name, restype, argtypes) of every entry point declared in include/nan_b200.h.
_VP, _U32, _I, _U64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_uint64
EXPORTS = {
    "nan_last_error": (ctypes.c_char_p, []),
    "nan_version": (_I, []),
    "nan_ctx_create": (_I, [_I, ctypes.POINTER(_VP)]),
    "nan_ctx_destroy": (_I, [_VP]),
    "nan_ctx_check": (_I, [_VP, _VP]),
    "nan_ctx_read_counters": (_I, [_VP, ctypes.POINTER(NanCounters), _I, _VP]),
    "nan_ctx_launch_count": (_U64, [_VP]),
    "nan_ctx_reserve": (_I, [_VP, _U64]),
    "nan_wavefront_bytes_per_path": (_U64, []),
    "nan_ctx_read_kernel_times": (_I, [_VP, ctypes.POINTER(NanKernelTimes), _I]),
    "nan_ctx_set_area_lights": (_I, [_VP, _VP, _U32, ctypes.c_float]),
    "nan_ctx_configure": (_I, [_VP, ctypes.POINTER(NanTuning)]),
    "nan_scene_build": (_I, [_VP, ctypes.POINTER(NanSceneDesc), _VP]),
    "nan_scene_build_noalloc": (_I, [_VP, ctypes.POINTER(NanSceneDesc), _VP, _U64, _VP, _U64, _VP, _U64, _VP]),
    "nan_scene_info": (_I, [_VP, ctypes.POINTER(NanSceneInfo)]),
    "nan_scene_world_triangles": (_I, [_VP, _VP, _VP]),
    "nan_intersect": (_I, [_VP, _VP, _U32, _VP, _VP, _VP]),
    "nan_occluded": (_I, [_VP, _VP, _U32, _VP, _VP]),
    "nan_visibility_ray_table": (_I, [_U32, _VP]),
    "nan_visibility_sh16": (_I, [_VP, _VP, _VP, _U32, _VP, _U32, ctypes.c_float, ctypes.c_float, _VP, _VP, _VP]),
    "nan_trace_screen": (_I, [_VP, _VP, _U32, _U32, _U32, _U32, ctypes.POINTER(NanCamera),
                              ctypes.POINTER(NanLighting), _VP]),
    "nan_accumulate": (_I, [_VP, _VP, _VP, _VP, _U32, _U32, _I, _VP]),
    "nan_trace_texels": (_I, [_VP, ctypes.POINTER(NanMeshColorsDesc), _VP, _U32, _U32, _U32, _I,
                              ctypes.POINTER(NanLighting), _U32, _U32, _VP]),
    "nan_trace_probes": (_I, [_VP, _VP, _VP, _VP, _VP, _VP, _U32, _VP, _U32, _U32, _U32, _U32, _I,
                              ctypes.POINTER(NanLighting), _U32, _U32, _VP, _VP]),
    "nan_pack_rgb9e5": (_I, [_VP, _VP, _VP, _U32, _VP]),
    "nan_cache_sizes": (_I, [ctypes.POINTER(NanCacheConfig), ctypes.POINTER(_U64), ctypes.POINTER(_U64)]),
    "nan_cache_create": (_I, [_VP, ctypes.POINTER(NanCacheConfig), ctypes.POINTER(_VP)]),
    "nan_cache_destroy": (_I, [_VP]),
    "nan_cache_set_params": (_I, [_VP, _VP, _VP, _VP]),
    "nan_cache_get_params": (_I, [_VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "nan_cache_infer": (_I, [_VP, _VP, _U32, _VP, _VP]),
    "nan_cache_backward": (_I, [_VP, _VP, _VP, _U32, _U32, _VP]),
    "nan_cache_step": (_I, [_VP, _VP]),
    "nan_cache_set_learning_rate": (_I, [_VP, ctypes.c_float]),
    "nan_cache_train": (_I, [_VP, _VP, _VP, _U32, _U32, _VP]),
    "nan_batch_create": (_I, [_VP, _VP, _U32, ctypes.POINTER(_VP)]),
    "nan_batch_destroy": (_I, [_VP]),
    "nan_batch_info": (_I, [_VP, ctypes.POINTER(_U32), ctypes.POINTER(_U32), ctypes.POINTER(NanBatchTuning)]),
    "nan_batch_set_tuning": (_I, [_VP, ctypes.POINTER(NanBatchTuning)]),
    "nan_batch_set_mode": (_I, [_VP, _U32]),
    "nan_batch_trace_probes": (_I, [_VP, _U32, _U32, _U32, _I, _VP]),
    "nan_batch_autotune": (_I, [_VP, _U32, _U32, _VP, ctypes.POINTER(NanBatchTuning), ctypes.POINTER(ctypes.c_float)]),
    "nan_batch_capture": (_I, [_VP, _U32, _I, _U32, _U32, _VP]),
    "nan_batch_replay": (_I, [_VP, _U32, _VP]),
    "nan_resolve_mesh_colors": (_I, [_VP, ctypes.POINTER(NanMeshColorsDesc), _VP, _I, _VP, _U32, _U32,
                                     ctypes.POINTER(NanCamera), ctypes.POINTER(NanLighting), _VP]),
    "nan_filter_mesh_colors": (_I, [_VP, ctypes.POINTER(NanMeshColorsDesc), _VP, _VP, _VP, _VP, ctypes.c_float,
                                    ctypes.c_float, _VP]),
    "nan_trace_probes_prt": (_I, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _U32, _VP, _U32, _U32, _U32, _U32, _I,
                                  ctypes.POINTER(NanLighting), _U32, _U32, _VP]),
    "nan_prt_project_lighting": (_I, [_VP, _VP, _U32, ctypes.POINTER(NanLighting), _VP]),
    "nan_prt_evaluate": (_I, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _U32, _VP]),
    "nan_resolve_probes": (_I, [_VP, ctypes.POINTER(NanProbeLayoutDesc), _VP, _VP, _VP, _VP,
                                ctypes.POINTER(NanProbeResolveOptions), _VP, _U32, _U32, ctypes.POINTER(NanCamera),
                                ctypes.POINTER(NanLighting), _VP]),
    "nan_deficit_repair": (_I, [_VP, _VP, _VP, _VP, _U32, _VP, _VP, _VP, _U32, _VP, _VP, _VP, _U32, _VP, _U32,
                                ctypes.POINTER(NanRepairOptions), _VP, ctypes.POINTER(_U32), _VP, _VP, _VP, _VP, _VP,
                                _VP, ctypes.POINTER(_U32), _VP]),
    "nan_estimate_support": (_I, [_VP, _VP, _VP, _VP, _VP, _U32, _VP, _VP, _VP, _U32, _VP, _U32,
                                  ctypes.POINTER(NanSupportOptions), _VP, _VP, _VP]),
    "nan_wse_eliminate": (_I, [_VP, _VP, _VP, _VP, _U32, _VP, _VP, ctypes.POINTER(NanWseOptions), _VP, _VP,
                               ctypes.POINTER(_U32), _VP]),
    "nan_wse_eliminate_adaptive": (_I, [_VP, _VP, _VP, _VP, _VP, _U32, _VP, _VP, ctypes.POINTER(NanWseOptions), _VP,
                                        _VP, ctypes.POINTER(_U32), _VP]),
    "nan_build_point_octrees": (_I, [_VP, _VP, _VP, _U32, _U32, _U32, _VP, _U32, _VP, _VP, _VP, _VP]),
    "nan_filter_audit_repair": (_I, [_VP, _VP, _VP, _VP, _U32, _VP, _VP, _VP, _U32, _VP, _U32, _U32, _VP,
                                     ctypes.c_double, _VP, ctypes.POINTER(_U32), _VP, ctypes.POINTER(_U32), _VP]),
    "nan_trace_points": (_I, [_VP, _VP, _U32, _VP, _U32, _U32, _U32, _U32, ctypes.POINTER(NanLighting), _VP]),
    "nan_trace_screen_cached": (_I, [_VP, _VP, _VP, _U32, _U32, _U32, ctypes.POINTER(NanCamera),
                                     ctypes.POINTER(NanLighting), ctypes.POINTER(NanCachedFrame), _VP]),
}

_lib: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    """Load libnan_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m nan_b200.build` "
                "(there is no CPU fallback for the tracer)"
            )
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (restype, argtypes) in EXPORTS.items():
            fn = getattr(handle, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = handle
    return _lib


def check(status: int) -> None:
    if status != NAN_OK:
        message = lib().nan_last_error()
        raise NanError(status, message.decode() if message else "")


def stream_handle(command_encoder) -> int | None:
    """Map the reference's command_encoder argument to a CUDA stream handle.

    Accepts None (the current torch stream), a torch.cuda.Stream, or a raw
    cudaStream_t integer.
    """
    import torch

    if command_encoder is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(command_encoder, int):
        return command_encoder
    if hasattr(command_encoder, "cuda_stream"):
        return command_encoder.cuda_stream
    raise TypeError(f"cannot use {type(command_encoder).__name__} as a CUDA stream")


def ptr(tensor) -> int:
    return int(tensor.data_ptr()) if tensor is not None else 0


class Context:
    """Owns one NanContext (device status word, counters, BVH)."""

    def __init__(self, device_index: int = 0):
        handle = ctypes.c_void_p()
        check(lib().nan_ctx_create(int(device_index), ctypes.byref(handle)))
        self.handle = handle
        self.device_index = int(device_index)

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            lib().nan_ctx_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, stream=None) -> None:
        check(lib().nan_ctx_check(self.handle, stream_handle(stream)))

    def read_counters(self, reset: bool = False, stream=None) -> dict:
        c = NanCounters()
        check(lib().nan_ctx_read_counters(self.handle, ctypes.byref(c), int(reset), stream_handle(stream)))
        return c.as_dict()

    @property
    def launch_count(self) -> int:
        return int(lib().nan_ctx_launch_count(self.handle))

    def reserve(self, scratch_bytes: int) -> None:
        """Grow the wavefront scratch arena to at least scratch_bytes."""
        check(lib().nan_ctx_reserve(self.handle, int(scratch_bytes)))

    def reserve_paths(self, paths: int) -> None:
        """Scratch for `paths` wavefront paths in flight (plus control words)."""
        per = int(lib().nan_wavefront_bytes_per_path())
        self.reserve(int(paths) * per + (1 << 22))

    def read_kernel_times(self, reset: bool = False) -> dict:
        """Device milliseconds of the wavefront stages recorded while
        kernel_timing is on (waits for their events)."""
        t = NanKernelTimes()
        check(lib().nan_ctx_read_kernel_times(self.handle, ctypes.byref(t), int(reset)))
        return t.as_dict()

    def configure(self, integrator: str = "wavefront", trace_blocks_per_sm: int = 0,
                  max_paths_in_flight: int = 0, bvh_builder: str = "sah", bvh_width: int = 2,
                  kernel_timing: bool = False, ray_order: int = 0, traversal: int = 0) -> None:
        t = NanTuning()
        t.ray_order = int(ray_order)
        t.traversal = int(traversal)
        t.kernel_timing = int(bool(kernel_timing))
        t.bvh_builder = BVH_BUILDERS[bvh_builder]
        t.bvh_width = 8 if int(bvh_width) == 8 else 2
        t.integrator = INTEGRATORS[integrator]
        t.trace_blocks_per_sm = int(trace_blocks_per_sm)
        t.max_paths_in_flight = int(max_paths_in_flight)
        check(lib().nan_ctx_configure(self.handle, ctypes.byref(t)))
