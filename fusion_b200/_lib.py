"""ctypes binding of libfusion_b200.so (include/fusion_b200.h).

Loading fails loudly when the library is missing or when no CUDA device is
present: there is no CPU fallback for any entry point.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfusion_b200.so")

FB_OK, FB_EINVAL, FB_ENOMEM, FB_ECUDA, FB_ETRACK_LOST = 0, 1, 2, 3, 4
FB_FORM_REFERENCE, FB_FORM_PRECISION = 0, 1

ERR_FLAGS = {
    0x1: "heap_exhausted", 0x2: "excess_full", 0x4: "request_set_full", 0x8: "coord_range",
    0x10: "new_list_full", 0x20: "visible_full", 0x40: "sequential_insert", 0x80: "timeout", 0x100: "normal_w",
}


class Config(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int),
        ("fx", ctypes.c_float), ("fy", ctypes.c_float), ("cx", ctypes.c_float), ("cy", ctypes.c_float),
        ("depth_scale", ctypes.c_float), ("depth_cutoff", ctypes.c_float),
        ("voxel_size", ctypes.c_float), ("trunc_dist", ctypes.c_float),
        ("depth_min", ctypes.c_float), ("depth_max", ctypes.c_float),
        ("num_buckets", ctypes.c_int), ("num_excess", ctypes.c_int), ("num_blocks", ctypes.c_int),
        ("iters", ctypes.c_int * 3),
        ("form", ctypes.c_int),
    ]


class FrameResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int), ("tracked", ctypes.c_int), ("tracker_state", ctypes.c_int),
        ("fused", ctypes.c_int),
        ("no_visible", ctypes.c_uint32), ("no_allocated", ctypes.c_uint32), ("no_new", ctypes.c_uint32),
        ("error_flags", ctypes.c_uint32),
        ("icp_error", ctypes.c_float), ("icp_count", ctypes.c_float),
        ("rgb_error", ctypes.c_float), ("rgb_count", ctypes.c_float),
        ("pose", ctypes.c_double * 16),
        ("frame_id", ctypes.c_uint64),
    ]


class MapStats(ctypes.Structure):
    _fields_ = [
        ("heap_counter", ctypes.c_int32), ("entry_ptr", ctypes.c_int32),
        ("no_allocated", ctypes.c_uint32), ("no_visible", ctypes.c_uint32), ("no_new", ctypes.c_uint32),
        ("no_tiles", ctypes.c_uint32), ("error_flags", ctypes.c_uint32), ("sequential", ctypes.c_int32),
    ]


class KeypointStats(ctypes.Structure):
    _fields_ = [("keys", ctypes.c_uint32), ("matches", ctypes.c_uint32), ("bootstrap", ctypes.c_int32),
                ("relocalised", ctypes.c_int32), ("keyframes", ctypes.c_uint32), ("map_keys", ctypes.c_uint32)]


class Image(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("pitch", ctypes.c_size_t), ("cols", ctypes.c_int),
                ("rows", ctypes.c_int)]


class FrameInput(ctypes.Structure):
    _fields_ = [("depth", ctypes.c_void_p), ("depth_pitch", ctypes.c_size_t), ("rgb", ctypes.c_void_p),
                ("rgb_pitch", ctypes.c_size_t), ("on_device", ctypes.c_int)]


# name -> (restype, argtypes)
_vp, _i, _f, _sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_size_t
_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.c_void_p
SIGNATURES = {
    "fb_default_config": (None, [ctypes.POINTER(Config), _i, _i]),
    "fb_status_string": (ctypes.c_char_p, [_i]),
    "fb_last_error": (ctypes.c_char_p, []),
    "fb_session_bytes": (_sz, [ctypes.POINTER(Config)]),
    "fb_graph_exec_stats": (None, [ctypes.POINTER(ctypes.c_longlong)] * 3),
    "fb_session_create": (_i, [ctypes.POINTER(Config), _vp, ctypes.POINTER(_vp)]),
    "fb_session_destroy": (_i, [_vp]),
    "fb_session_reset": (_i, [_vp]),
    "fb_grab_frame": (_i, [_vp, _vp, _sz, _vp, _sz, _i, ctypes.POINTER(FrameResult)]),
    "fb_stage_frame": (_i, [_vp, _vp, _sz, _vp, _sz]),
    "fb_get_pose": (_i, [_vp, _vp]),
    "fb_session_set_profiling": (_i, [_vp, _i]),
    "fb_session_set_graphs": (_i, [_vp, _i]),
    "fb_session_stage_times": (_i, [_vp, _vp, _vp, _i]),
    "fb_session_set_raycast_tile": (_i, [_vp, _i, _i]),
    "fb_session_prepare": (_i, [_vp, _i]),
    "fb_session_prepare_some": (_i, [_vp, _i, _i, ctypes.POINTER(ctypes.c_int)]),
    "fb_render_image": (_i, [ctypes.POINTER(Image), ctypes.POINTER(Image), _vp, ctypes.POINTER(Image), _vp]),
    "fb_depth_to_image": (_i, [ctypes.POINTER(Image), ctypes.POINTER(Image), _vp]),
    "fb_rgb_to_rgba": (_i, [ctypes.POINTER(Image), ctypes.POINTER(Image), _vp]),
    "fb_session_set_keypoints": (_i, [_vp, _i]),
    "fb_session_keypoint_stats": (_i, [_vp, ctypes.POINTER(KeypointStats)]),
    "fb_download_keypoints": (_i, [_vp, _i, _vp, _vp, _vp, _vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]),
    "fb_match_descriptors": (_i, [_vp, ctypes.c_uint32, _vp, ctypes.c_uint32, _vp, _vp, _vp]),
    "fb_pose_estimate": (_i, [_vp, _vp, ctypes.c_uint32, _i, _i, ctypes.c_uint64, _vp, _vp,
                              ctypes.POINTER(ctypes.c_int)]),
    "fb_write_map_file": (_i, [_vp, ctypes.c_char_p]),
    "fb_read_map_file": (_i, [_vp, ctypes.c_char_p]),
    "fb_session_set_mapping": (_i, [_vp, _i]),
    "fb_render_top_down": (_i, [_vp, _f, ctypes.POINTER(Image), ctypes.POINTER(Image), ctypes.POINTER(Image),
                                ctypes.POINTER(ctypes.c_int), _vp]),
    "fb_mesh_scene": (_i, [_vp, _vp, _vp, _vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), _vp]),
    "fb_mesh_case_table": (_i, [_vp, _vp]),
    "fb_write_ply": (_i, [ctypes.c_char_p, _vp, _vp, _vp, ctypes.c_uint64]),
    "fb_save_mesh": (_i, [_vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64)]),
    "fb_snapshot_bytes": (_i, [_vp, ctypes.POINTER(_sz)]),
    "fb_snapshot": (_i, [_vp, _vp, _sz, ctypes.POINTER(_sz)]),
    "fb_restore": (_i, [_vp, _vp, _sz]),
    "fb_batch_create": (_i, [_vp, ctypes.POINTER(_vp)]),
    "fb_batch_destroy": (_i, [_vp]),
    "fb_batch_set_mode": (_i, [_vp, _i]),
    "fb_batch_reserve": (_i, [_vp, _sz]),
    "fb_batch_step": (_i, [_vp, _vp, _i, _vp, _vp]),
    "fb_batch_stats": (_i, [_vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "fb_batch_launch_stats": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "fb_batch_set_lanes": (_i, [_vp, _i]),
    "fb_session_set_integration_grid": (_i, [_vp, _i]),
    "fb_batch_submit": (_i, [_vp, _vp, _i, _vp]),
    "fb_batch_collect": (_i, [_vp, _vp]),
    "fb_session_launch_count": (_i, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    "fb_frame_transfer_bytes": (_i, [ctypes.POINTER(Config), ctypes.POINTER(_sz), ctypes.POINTER(_sz)]),
    "fb_download_level": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "fb_download_raw": (_i, [_vp, _i, _vp]),
    "fb_map_get_stats": (_i, [_vp, ctypes.POINTER(MapStats)]),
    "fb_map_download_entries": (_i, [_vp, _vp]),
    "fb_map_download_blocks": (_i, [_vp, _vp, _i, _vp, _vp, _vp]),
    "fb_map_download_visible": (_i, [_vp, _vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]),
    "fb_filter_depth": (_i, [ctypes.POINTER(Image)] * 3 + [_f, _f, _vp]),
    "fb_image_to_intensity": (_i, [ctypes.POINTER(Image)] * 2 + [_vp]),
    "fb_pyrdown_gauss_f32": (_i, [ctypes.POINTER(Image)] * 2 + [_vp]),
    "fb_pyrdown_gauss_u8": (_i, [ctypes.POINTER(Image)] * 2 + [_vp]),
    "fb_compute_vmap": (_i, [ctypes.POINTER(Image)] * 2 + [_f, _f, _f, _f, _f, _vp]),
    "fb_compute_nmap": (_i, [ctypes.POINTER(Image)] * 2 + [_vp]),
    "fb_compute_derivative_image": (_i, [ctypes.POINTER(Image)] * 3 + [_vp]),
    "fb_resize_map": (_i, [ctypes.POINTER(Image)] * 4 + [_vp]),
    "fb_step_scratch_bytes": (_sz, [_i, _i]),
    "fb_track_reduction_grid": (_i, [_i]),
    "fb_create_rendering_blocks": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "fb_map_export_visible": (_i, [_vp, _vp, ctypes.c_uint32, _vp, _vp]),
    "fb_map_export_reference": (_i, [_vp, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _vp, _vp]),
    "fb_icp_step": (_i, [ctypes.POINTER(Image)] * 4 + [_vp] * 6 + [_vp, _sz, _vp, _vp, _vp, _vp]),
    "fb_rgb_step": (_i, [ctypes.POINTER(Image)] * 6 + [_vp] * 7 + [_vp, _sz, _vp, _vp, _vp, _vp]),
    "fb_rgb_step_static": (_i, [ctypes.POINTER(Image)] * 6 + [_vp] * 7 + [_vp, _vp, _vp, _vp]),
    "fb_rgb_step_static_max_pixels": (_sz, []),
    "fb_reset_map": (_i, [_vp]),
    "fb_fuse_map_color": (_i, [_vp] + [ctypes.POINTER(Image)] * 3 + [_vp] * 4 +
                          [ctypes.POINTER(ctypes.c_uint32), _vp]),
    "fb_check_block_visibility": (_i, [_vp, _vp, _vp, _vp, _i, _i, _vp, ctypes.POINTER(ctypes.c_uint32), _vp]),
    "fb_raycast": (_i, [_vp, ctypes.POINTER(Image), ctypes.POINTER(Image), _vp, _vp, _vp, _vp,
                        ctypes.POINTER(ctypes.c_int), _vp]),
}

_LIB = None


class FusionError(RuntimeError):
    def __init__(self, fn, code):
        lib = _LIB
        msg = lib.fb_status_string(code).decode() if lib else str(code)
        extra = lib.fb_last_error().decode() if (lib and code == FB_ECUDA) else ""
        super().__init__(f"{fn}: {msg}" + (f" ({extra})" if extra else ""))
        self.code = code


def load():
    """The loaded library.  Raises if the .so is missing."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m fusion_b200.build` "
                               "(there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def check(fn, code):
    if code != FB_OK:
        raise FusionError(fn, code)
    return code


def exported_symbols():
    return sorted(SIGNATURES)
