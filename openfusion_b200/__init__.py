"""openfusion_b200 -- a from-scratch sm_100a KinectFusion per-frame path.

Pre-processing (bilateral filter, depth pyramid, vertex/normal maps), TSDF
integration, raycasting and multi-level point-to-plane ICP run as hand-written
CUDA kernels behind the C-ABI of include/openfusion_b200.h; this package is the
Python mirror of the reference's per-frame interfaces over that ABI.
"""
from . import _native
from .api import (CONFIGS, Batch, Config, Reader, c4_configs, copy_pyramid, depth_filter,
                  depth_filter_params,
                  depth_rgba, normals_rgba,
                  extract_mesh, read_recording_frame,
                  save_volume_raw, write_obj,
                  read_recording_info, write_recording, Sequence, Tracker, integrate_scratch, icp_system, icp_track,
                  icp_track_warm,
                  icp_workspace, integrate, integrate_census, integrate_visible_census, lambda_table, level_camera, linear_to_volume,
                  make_scene, make_sequence, make_trajectory, new_pyramid, new_volume,
                  preprocess, pyramid_layout, raycast, raycast_march_samples, render, unpack_depth, unpack_points,
                  volume_bytes, volume_to_linear, shard, stream_cost)

__all__ = [
    "CONFIGS", "Batch", "Config", "Reader", "c4_configs", "copy_pyramid", "depth_filter",
    "depth_filter_params",
    "depth_rgba", "normals_rgba",
    "extract_mesh", "read_recording_frame",
    "save_volume_raw", "write_obj",
    "read_recording_info", "write_recording", "Sequence", "Tracker", "integrate_scratch", "icp_system", "icp_track", "icp_track_warm", "icp_workspace",
    "integrate", "integrate_census", "integrate_visible_census", "lambda_table", "level_camera", "linear_to_volume",
    "make_scene", "make_sequence", "make_trajectory", "new_pyramid", "new_volume", "preprocess",
    "pyramid_layout", "raycast", "raycast_march_samples", "render", "unpack_depth", "unpack_points", "volume_bytes",
    "volume_to_linear", "shard", "stream_cost",
]
