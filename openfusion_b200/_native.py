"""ctypes binding of the C-ABI in include/openfusion_b200.h and of_synth.h.

The CUDA library is mandatory: loading fails with an ImportError naming the
missing file, and there is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIBDIR = Path(__file__).resolve().parent / "lib"

c_status = C.c_int32
c_stream = C.c_void_p


class Camera(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("fx", C.c_float), ("fy", C.c_float),
                ("cx", C.c_float), ("cy", C.c_float), ("min_depth_mm", C.c_float),
                ("max_depth_mm", C.c_float)]


class VolumeDesc(C.Structure):
    _fields_ = [("resolution", C.c_int32), ("storage", C.c_int32), ("size_mm", C.c_float),
                ("trunc_mm", C.c_float), ("max_weight", C.c_int32), ("reserved", C.c_int32)]


class FilterParams(C.Structure):
    _fields_ = [("sigma_space_px", C.c_float), ("sigma_range_mm", C.c_float),
                ("radius_px", C.c_int32), ("levels", C.c_int32)]


class RaycastParams(C.Structure):
    _fields_ = [("min_step_vox", C.c_float), ("far_step_frac", C.c_float),
                ("refine_iters", C.c_int32), ("tile", C.c_int32)]


class IcpParams(C.Structure):
    _fields_ = [("levels", C.c_int32), ("iters", C.c_int32 * 4), ("dist_thresh_mm", C.c_float),
                ("normal_thresh", C.c_float), ("stop_rot_rad", C.c_float),
                ("stop_trans_mm", C.c_float), ("judge_max_rms_mm", C.c_float),
                ("judge_min_inlier_frac", C.c_float), ("judge_max_rot_rad", C.c_float),
                ("judge_max_trans_mm", C.c_float), ("warm_levels", C.c_int32)]


class IcpStats(C.Structure):
    _fields_ = [("status", C.c_int32), ("inliers", C.c_int32), ("iterations", C.c_int32),
                ("warm", C.c_int32), ("residual_sq", C.c_double), ("min_pivot", C.c_double)]


class PyramidLayout(C.Structure):
    _fields_ = [("levels", C.c_int32), ("width", C.c_int32 * 4), ("height", C.c_int32 * 4),
                ("depth_offset", C.c_size_t * 4), ("points_offset", C.c_size_t * 4),
                ("total_bytes", C.c_size_t)]


class DepthFilterParams(C.Structure):
    _fields_ = [("steps", C.c_int32), ("null_value", C.c_int32), ("average_passes", C.c_int32),
                ("average_threshold_mm", C.c_float), ("gradient_threshold_mm", C.c_float),
                ("k1", C.c_float), ("k2", C.c_float), ("p1", C.c_float), ("p2", C.c_float)]


class TrackerDesc(C.Structure):
    _fields_ = [("camera", Camera), ("volume", VolumeDesc), ("filter", FilterParams),
                ("raycast", RaycastParams), ("icp", IcpParams),
                ("initial_pose", C.c_double * 16), ("use_graph", C.c_int32),
                ("pose_history", C.c_int32), ("warm_start_weights", C.c_void_p),
                ("depth_filter", DepthFilterParams), ("tune", C.c_int32)]


class TrackerBuffers(C.Structure):
    _fields_ = [("volume", C.c_void_p), ("frame", C.c_void_p), ("model", C.c_void_p),
                ("pose", C.c_void_p), ("depth", C.c_void_p), ("lambda_", C.c_void_p),
                ("stats", C.c_void_p), ("frames", C.c_int64), ("kernels_first", C.c_int32),
                ("kernels_track", C.c_int32)]


class BatchStream(C.Structure):
    _fields_ = [("camera", Camera), ("volume", VolumeDesc), ("initial_pose", C.c_double * 16)]


class BatchTuning(C.Structure):
    _fields_ = [("ray_tile", C.c_int32), ("list_div", C.c_int32), ("icp_clusters", C.c_int32),
                ("tuned", C.c_int32)]


class BatchDesc(C.Structure):
    _fields_ = [("count", C.c_int32), ("streams", C.POINTER(BatchStream)),
                ("filter", FilterParams), ("raycast", RaycastParams), ("icp", IcpParams),
                ("use_graph", C.c_int32), ("tune", C.c_int32), ("tuning", BatchTuning)]


class RecordingInfo(C.Structure):
    _fields_ = [("camera", Camera), ("z_offset_mm", C.c_float), ("frames", C.c_int32),
                ("name", C.c_char * 256), ("date", C.c_char * 64), ("camera_type", C.c_char * 64)]


class SynthPrim(C.Structure):
    _fields_ = [("kind", C.c_int32), ("p", C.c_float * 10)]


class SynthScene(C.Structure):
    _fields_ = [("count", C.c_int32), ("room_half_mm", C.c_float), ("prims", SynthPrim * 64)]


P = C.c_void_p
_SIGS = {
    "of_abi_version": (C.c_int32, []),
    "of_status_string": (C.c_char_p, [c_status]),
    "of_default_params": (None, [C.POINTER(FilterParams), C.POINTER(RaycastParams),
                                 C.POINTER(IcpParams)]),
    "of_camera_level": (c_status, [C.POINTER(Camera), C.c_int32, C.POINTER(Camera)]),
    "of_volume_bytes": (c_status, [C.POINTER(VolumeDesc), C.POINTER(C.c_size_t)]),
    "of_volume_reset": (c_status, [C.POINTER(VolumeDesc), P, c_stream]),
    "of_volume_export": (c_status, [C.POINTER(VolumeDesc), P, P, P, c_stream]),
    "of_volume_import": (c_status, [C.POINTER(VolumeDesc), P, P, P, c_stream]),
    "of_pyramid_layout": (c_status, [C.POINTER(Camera), C.c_int32, C.POINTER(PyramidLayout)]),
    "of_preprocess": (c_status, [C.POINTER(Camera), C.POINTER(FilterParams), P, C.c_int32, P,
                                 c_stream]),
    "of_integrate": (c_status, [C.POINTER(VolumeDesc), P, C.POINTER(Camera), P, C.c_int32, P, P,
                                c_stream]),
    "of_integrate_tiled": (c_status, [C.POINTER(VolumeDesc), P, C.POINTER(Camera), P, C.c_int32,
                                      P, P, P, c_stream]),
    "of_integrate_scratch_bytes": (c_status, [C.POINTER(VolumeDesc), C.POINTER(Camera),
                                              C.POINTER(C.c_size_t)]),
    "of_lambda_bytes": (c_status, [C.POINTER(Camera), C.POINTER(C.c_size_t)]),
    "of_lambda_table": (c_status, [C.POINTER(Camera), P, c_stream]),
    "of_integrate_census": (c_status, [C.POINTER(VolumeDesc), P, C.POINTER(Camera), P, C.c_int32,
                                       P, P, P, c_stream]),
    "of_integrate_visible_census": (c_status, [C.POINTER(VolumeDesc), P, C.POINTER(Camera), P,
                                               C.c_int32, P, P, P, c_stream]),
    "of_raycast": (c_status, [C.POINTER(VolumeDesc), P, C.POINTER(Camera),
                              C.POINTER(RaycastParams), C.c_int32, P, P, P, c_stream]),
    "of_icp_workspace_bytes": (c_status, [C.POINTER(Camera), C.POINTER(C.c_size_t)]),
    "of_icp_track": (c_status, [C.POINTER(Camera), C.POINTER(IcpParams), P, P, P, P, P,
                                c_stream]),
    "of_icp_workspace_hold_barrier": (c_status, [P, C.c_int32, c_stream]),
    "of_icp_track_static": (c_status, [C.POINTER(Camera), C.POINTER(IcpParams), P, P, P, P,
                                       c_stream]),
    "of_icp_system": (c_status, [C.POINTER(Camera), C.POINTER(IcpParams), C.c_int32, P, P, P, P,
                                 P, c_stream]),
    "of_icp_solve_step": (c_status, [P, P, P, c_stream]),
    "of_tracker_create": (c_status, [C.POINTER(TrackerDesc), C.POINTER(C.c_void_p)]),
    "of_tracker_destroy": (c_status, [P]),
    "of_tracker_process": (c_status, [P, P, C.c_int32, c_stream]),
    "of_tracker_flush": (c_status, [P, c_stream]),
    "of_tracker_save": (c_status, [P, C.c_char_p, c_stream]),
    "of_tracker_load": (c_status, [P, C.c_char_p, c_stream]),
    "of_depth_filter_defaults": (None, [C.POINTER(DepthFilterParams)]),
    "of_depth_filter": (c_status, [C.POINTER(Camera), C.POINTER(DepthFilterParams), P, P, P,
                                   c_stream]),
    "of_depth_filter_step": (c_status, [C.POINTER(Camera), C.c_int32,
                                        C.POINTER(DepthFilterParams), P, P, c_stream]),
    "of_depth_to_rgba": (c_status, [C.POINTER(Camera), P, P, c_stream]),
    "of_normals_to_rgba": (c_status, [C.POINTER(Camera), P, P, C.c_float, P, c_stream]),
    "of_mesh_extract": (c_status, [C.POINTER(VolumeDesc), P, P, P, C.c_uint32, P, c_stream]),
    "of_mesh_write_obj": (c_status, [C.c_char_p, P, C.c_uint32]),
    "of_volume_save_raw": (c_status, [C.POINTER(VolumeDesc), P, C.c_char_p, c_stream]),
    "of_recording_read_info": (c_status, [C.c_char_p, C.POINTER(RecordingInfo)]),
    "of_recording_write_info": (c_status, [C.c_char_p, C.POINTER(RecordingInfo)]),
    "of_recording_read_frame": (c_status, [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, P]),
    "of_recording_write_frame": (c_status, [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, P,
                                            C.c_int32, c_stream]),
    "of_reader_open": (c_status, [C.c_char_p, C.c_int32, C.POINTER(C.c_void_p)]),
    "of_reader_info": (c_status, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_int32)]),
    "of_reader_next": (c_status, [P, P, c_stream]),
    "of_reader_close": (c_status, [P]),
    "of_batch_create": (c_status, [C.POINTER(BatchDesc), C.POINTER(C.c_void_p)]),
    "of_batch_destroy": (c_status, [P]),
    "of_batch_process": (c_status, [P, C.POINTER(C.c_void_p), C.c_int32, c_stream]),
    "of_batch_flush": (c_status, [P, c_stream]),
    "of_batch_poses": (c_status, [P, P, P, c_stream]),
    "of_batch_tuning": (c_status, [P, C.POINTER(BatchTuning)]),
    "of_batch_stream_buffers": (c_status, [P, C.c_int32, C.POINTER(TrackerBuffers)]),
    "of_batch_stream_cost": (c_status, [C.POINTER(BatchStream), C.POINTER(IcpParams),
                                        C.POINTER(C.c_double)]),
    "of_batch_shard": (c_status, [P, C.c_int32, C.c_int32, P]),
    "of_tracker_set_prior": (c_status, [P, P]),
    "of_tracker_pose": (c_status, [P, P, P, c_stream]),
    "of_tracker_pose_history": (c_status, [P, P, C.c_int32, c_stream]),
    "of_tracker_buffers": (c_status, [P, C.POINTER(TrackerBuffers)]),
    "of_tracker_tuning": (c_status, [P, P, P]),
    "of_points_to_reference": (c_status, [C.POINTER(Camera), P, P, P, P, c_stream]),
    "of_points_from_reference": (c_status, [C.POINTER(Camera), C.c_int32, P, P, P, c_stream]),
    "of_pose_from_float": (c_status, [P, P, C.c_int32, c_stream]),
    "of_pose_to_float": (c_status, [P, P, P, P, c_stream]),
    "of_cnn_param_count": (c_status, [C.POINTER(C.c_int64)]),
    "of_cnn_workspace_bytes": (c_status, [C.c_int32, C.POINTER(C.c_size_t)]),
    "of_cnn_init": (c_status, [P, P, C.c_uint64, c_stream]),
    "of_cnn_input": (c_status, [P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int64, P, P,
                                c_stream]),
    "of_cnn_forward": (c_status, [P, P, P, C.c_int32, P, P, c_stream]),
    "of_cnn_backward": (c_status, [P, P, P, C.c_int32, P, P, P, P, P, c_stream]),
    "of_cnn_adam": (c_status, [P, P, P, P, P, C.c_int32, C.c_float, c_stream]),
    "of_cnn_load": (c_status, [P, P, c_stream]),
    "of_cnn_predict": (c_status, [P, P, P, P, C.c_int32, C.c_int32, P, P, P, c_stream]),
    "of_cnn_warm_pose": (c_status, [P, P, P, c_stream]),
    "of_icp_track_warm": (c_status, [C.POINTER(Camera), C.POINTER(IcpParams), P, P, P, P, P, P,
                                     c_stream]),
    "of_synth_render_device": (c_status, [P, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_float,
                                          C.c_float, P, C.c_int32, C.c_uint64, C.c_int32,
                                          C.c_float, C.c_float, P, c_stream]),
}

_SYNTH_SIGS = {
    "of_synth_scene": (C.c_int32, [C.c_int32, C.c_uint64, C.c_float, C.POINTER(SynthScene)]),
    "of_synth_trajectory": (C.c_int32, [C.c_int32, C.c_uint64, C.c_float, C.c_int32, P]),
    "of_synth_render": (C.c_int32, [C.POINTER(SynthScene), C.c_int32, C.c_int32, C.c_float,
                                    C.c_float, C.c_float, C.c_float, P, C.c_uint64, C.c_int32,
                                    C.c_float, C.c_float, P, P]),
}

_lib = None
_synth = None


def exported_symbols() -> list[str]:
    """Names the CUDA library must export (every function of the header)."""
    return sorted(_SIGS)


def _load(name: str, sigs: dict) -> C.CDLL:
    path = LIBDIR / name
    if not path.exists():
        raise ImportError(f"{path} is missing: build it with `python -m openfusion_b200.build`")
    lib = C.CDLL(str(path))
    for fn, (res, args) in sigs.items():
        f = getattr(lib, fn)
        f.restype = res
        f.argtypes = args
    return lib


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = _load("libopenfusion_b200.so", _SIGS)
    return _lib


def synth() -> C.CDLL:
    global _synth
    if _synth is None:
        _synth = _load("libof_synth.so", _SYNTH_SIGS)
    return _synth


class OpenFusionError(RuntimeError):
    def __init__(self, fn: str, status: int):
        msg = lib().of_status_string(status).decode()
        super().__init__(f"{fn} failed with status {status}: {msg}")
        self.status = status


def check(fn: str, status: int) -> None:
    if status != 0:
        raise OpenFusionError(fn, status)
