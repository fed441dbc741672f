// openfusion_b200.hpp -- C++ classes shaped like the reference's per-frame
// modules, implemented over the C-ABI of openfusion_b200.h. Code written
// against gilbs10/OpenFusion's VolumeIntegrator / Raycaster / ICP / General /
// CameraHandler::updateCameraData (Source/include/VolumeIntegrator.h:9-17,
// Raycaster.h:6-13, ICP.h:50-70, General.h:6-20, CameraHandler.h:24) keeps its
// call sites; the types below carry the same fields with the same meaning.
//
// Differences a caller must know:
//   - the volume is one buffer of of_volume_bytes() bytes (packed int16 tsdf +
//     uint16 weight per voxel, brick-major, plus brick flags); the
//     `VoxelType*` argument is that buffer and the weight pointer is unused;
//   - modules own their device scratch (allocated in their constructors, as the
//     reference's ICP constructor does, ICP.cpp:26-58);
//   - errors throw openfusion::Error instead of exiting (cutilSafeCall).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

#include "openfusion_b200.h"

namespace openfusion {

struct Error : std::runtime_error {
  of_status_t status;
  Error(const char *what, of_status_t s)
      : std::runtime_error(std::string(what) + ": " + of_status_string(s)), status(s) {}
};

inline void check(of_status_t s, const char *what) {
  if (s != OF_OK) throw Error(what, s);
}

// Intrinsic / CameraParams (Source/include/BasicTypes.h:74-103).
struct Intrinsic {
  float m_fx, m_fy, m_cx, m_cy;
  void Set(float fx = 0, float fy = 0, float cx = 0, float cy = 0) {
    m_fx = fx; m_fy = fy; m_cx = cx; m_cy = cy;
  }
};

struct CameraParams {
  Intrinsic m_intrinsic;
  Intrinsic m_invIntrinsic;
  unsigned m_width;
  unsigned m_height;
  float m_z_offset;
  float m_min_depth;
  float m_max_depth;
  float k1, k2, k3, p1, p2;
  uint16_t depthNullValue;
};

// PointInfo / CameraData (BasicTypes.h:40-49): AoS float3 maps, invalid
// vertex = FLT_MAX, invalid normal = 0.
struct PointInfo {
  float3 *vertex;
  float3 *normal;
};

struct CameraData {
  uint16_t *depth;
  float3 *vertex;
  float3 *normal;
};

typedef void VoxelType;               // the packed volume buffer
typedef unsigned char VoxelWeightType;  // unused (the weight lives in the voxel word)

inline of_camera_t to_camera(const CameraParams &p) {
  of_camera_t c;
  c.width = (int32_t)p.m_width;
  c.height = (int32_t)p.m_height;
  c.fx = p.m_intrinsic.m_fx;
  c.fy = p.m_intrinsic.m_fy;
  c.cx = p.m_intrinsic.m_cx;
  c.cy = p.m_intrinsic.m_cy;
  c.min_depth_mm = p.m_min_depth;
  c.max_depth_mm = p.m_max_depth;
  return c;
}

// Everything the reference fixed at compile time (Constants.h:23-55).
struct Settings {
  of_volume_desc_t volume;
  of_filter_params_t filter;
  of_raycast_params_t raycast;
  of_icp_params_t icp;
  Settings(int32_t resolution = 512, float size_mm = 3000.f, float trunc_mm = 30.f,
           int32_t max_weight = 128) {
    volume.resolution = resolution;
    volume.storage = OF_TSDF_I16;
    volume.size_mm = size_mm;
    volume.trunc_mm = trunc_mm;
    volume.max_weight = max_weight;
    volume.reserved = 0;
    of_default_params(&filter, &raycast, &icp);
  }
};

template <class T>
struct DeviceBuffer {
  T *ptr = nullptr;
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t bytes) {
    if (cudaMalloc((void **)&ptr, bytes) != cudaSuccess) throw Error("cudaMalloc", OF_ERR_OUT_OF_MEMORY);
  }
  ~DeviceBuffer() { if (ptr) cudaFree(ptr); }
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
};

// General (General.h:6-20): volume reset and pose bookkeeping.
class General {
 public:
  explicit General(const Settings &s = Settings()) : m_s(s) {}
  static size_t VolumeBytes(const Settings &s) {
    size_t b = 0;
    check(of_volume_bytes(&s.volume, &b), "of_volume_bytes");
    return b;
  }
  void InitVoxelArray(VoxelType *d_voxel_array, VoxelWeightType * /*unused*/,
                      cudaStream_t stream = 0) {
    check(of_volume_reset(&m_s.volume, d_voxel_array, stream), "of_volume_reset");
  }
  // d_currentTransform (float[16], camera-to-world) -> inverse and camera
  // position (General.cpp:14-40), computed on the device in FP64.
  void UpdateTransforms(float *d_currentTransform, float *d_invCurrentTransform,
                        float3 *d_cameraPosition, float * /*invViewMatrix (UI only)*/,
                        cudaStream_t stream = 0) {
    DeviceBuffer<double> pose(16 * sizeof(double));
    check(of_pose_from_float(d_currentTransform, pose.ptr, 0, stream), "of_pose_from_float");
    check(of_pose_to_float(pose.ptr, nullptr, d_invCurrentTransform, (float *)d_cameraPosition,
                           stream),
          "of_pose_to_float");
    cudaStreamSynchronize(stream);
  }

 private:
  Settings m_s;
};

// VolumeIntegrator (VolumeIntegrator.h:9-17).
class VolumeIntegrator {
 public:
  VolumeIntegrator(CameraParams *cameraParams, const Settings &s = Settings())
      : m_cam(to_camera(*cameraParams)), m_s(s),
        m_lambda(bytes_of(of_lambda_bytes, m_cam)), m_scratch(scratch_bytes(m_s, m_cam)),
        m_pose(16 * sizeof(double)) {
    check(of_lambda_table(&m_cam, m_lambda.ptr, 0), "of_lambda_table");
  }
  // invTransform: world-to-camera float[16] on the device (the reference's
  // d_invCurrentTransform); the camera position is implied by it.
  void Integrate(VoxelType *d_voxel_array, VoxelWeightType * /*unused*/, const float *invTransform,
                 const CameraData &depthMap, const float3 * /*d_cameraPosition*/,
                 cudaStream_t stream = 0) {
    check(of_pose_from_float(invTransform, m_pose.ptr, 1, stream), "of_pose_from_float");
    check(of_integrate_tiled(&m_s.volume, d_voxel_array, &m_cam, depthMap.depth, m_cam.width,
                             m_pose.ptr, m_lambda.ptr, m_scratch.ptr, stream),
          "of_integrate_tiled");
  }

 private:
  static size_t bytes_of(of_status_t (*f)(const of_camera_t *, size_t *), const of_camera_t &c) {
    size_t n = 0;
    check(f(&c, &n), "size query");
    return n;
  }
  static size_t scratch_bytes(const Settings &s, const of_camera_t &c) {
    size_t n = 0;
    check(of_integrate_scratch_bytes(&s.volume, &c, &n), "of_integrate_scratch_bytes");
    return n;
  }
  of_camera_t m_cam;
  Settings m_s;
  DeviceBuffer<float> m_lambda;
  DeviceBuffer<unsigned char> m_scratch;
  DeviceBuffer<double> m_pose;
};

// Raycaster (Raycaster.h:6-13).
class Raycaster {
 public:
  Raycaster(CameraParams *cameraParams, const Settings &s = Settings())
      : m_cam(to_camera(*cameraParams)), m_s(s), m_model(layout_bytes()),
        m_pose(16 * sizeof(double)) {}
  // transform: camera-to-world float[16] on the device. Writes the world
  // vertex/normal maps of `renderedVertexMap` and, if d_output != NULL, the
  // shaded image (Raycaster.cu:221-227). Keeps the model pyramid for ICP.
  void Raycast(unsigned *d_output, float *transform, VoxelType *d_voxel_array,
               const PointInfo &renderedVertexMap, const float3 * /*d_cameraPosition*/,
               bool /*showNormals: shaded output only*/, cudaStream_t stream = 0) {
    check(of_pose_from_float(transform, m_pose.ptr, 0, stream), "of_pose_from_float");
    check(of_raycast(&m_s.volume, d_voxel_array, &m_cam, &m_s.raycast, m_s.icp.levels, m_pose.ptr,
                     m_model.ptr, d_output, stream),
          "of_raycast");
    if (renderedVertexMap.vertex || renderedVertexMap.normal)
      check(of_points_to_reference(&m_cam, m_model.ptr, nullptr, (float *)renderedVertexMap.vertex,
                                   (float *)renderedVertexMap.normal, stream),
            "of_points_to_reference");
  }
  const void *Model() const { return m_model.ptr; }

 private:
  size_t layout_bytes() {
    of_pyramid_layout_t lay;
    check(of_pyramid_layout(&m_cam, m_s.icp.levels, &lay), "of_pyramid_layout");
    return lay.total_bytes;
  }
  of_camera_t m_cam;
  Settings m_s;
  DeviceBuffer<uint8_t> m_model;
  DeviceBuffer<double> m_pose;
};

// ICP (ICP.h:50-70).
class ICP {
 public:
  ICP(dim3 /*gridSize*/, dim3 /*blockSize*/, CameraParams *cameraParams,
      const Settings &s = Settings())
      : m_cam(to_camera(*cameraParams)), m_s(s), m_frame(layout_bytes()), m_model(layout_bytes()),
        m_ws(ws_bytes()), m_pose(16 * sizeof(double)), m_stats(sizeof(of_icp_stats_t)) {
    cudaMemset(m_ws.ptr, 0, ws_bytes());
  }
  // Refines d_currentTransform (float[16] camera-to-world, in/out) of the new
  // depth frame against the rendered model maps (world space).
  void Iterate_ICP(const CameraData &newDepthData, const PointInfo &renderedVertexMap,
                   float *d_currentTransform, cudaStream_t stream = 0) {
    check(of_preprocess(&m_cam, &m_s.filter, newDepthData.depth, m_cam.width, m_frame.ptr, stream),
          "of_preprocess");
    check(of_points_from_reference(&m_cam, m_s.icp.levels, (const float *)renderedVertexMap.vertex,
                                   (const float *)renderedVertexMap.normal, m_model.ptr, stream),
          "of_points_from_reference");
    check(of_pose_from_float(d_currentTransform, m_pose.ptr, 0, stream), "of_pose_from_float");
    check(of_icp_track(&m_cam, &m_s.icp, m_frame.ptr, m_model.ptr, m_pose.ptr, m_ws.ptr,
                       m_stats.ptr, stream),
          "of_icp_track");
    check(of_pose_to_float(m_pose.ptr, d_currentTransform, nullptr, nullptr, stream),
          "of_pose_to_float");
  }
  of_icp_stats_t LastStats(cudaStream_t stream = 0) {
    of_icp_stats_t st;
    cudaMemcpyAsync(&st, m_stats.ptr, sizeof(st), cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    return st;
  }

 private:
  size_t layout_bytes() {
    of_pyramid_layout_t lay;
    check(of_pyramid_layout(&m_cam, m_s.icp.levels, &lay), "of_pyramid_layout");
    return lay.total_bytes;
  }
  size_t ws_bytes() {
    size_t b = 0;
    check(of_icp_workspace_bytes(&m_cam, &b), "of_icp_workspace_bytes");
    return b;
  }
  of_camera_t m_cam;
  Settings m_s;
  DeviceBuffer<uint8_t> m_frame, m_model, m_ws;
  DeviceBuffer<double> m_pose;
  DeviceBuffer<of_icp_stats_t> m_stats;
};

// CameraHandler::updateCameraData (CameraHandler.cu:134-143): the new depth's
// world-space vertex and normal maps at d_currentTransform.
inline void updateCameraData(const CameraParams &params, const CameraData &d_cameraData,
                             const uint16_t *d_newDepth, float *d_currentTransform,
                             const Settings &s = Settings(), cudaStream_t stream = 0) {
  of_camera_t cam = to_camera(params);
  of_pyramid_layout_t lay;
  check(of_pyramid_layout(&cam, 1, &lay), "of_pyramid_layout");
  DeviceBuffer<uint8_t> frame(lay.total_bytes);
  DeviceBuffer<double> pose(16 * sizeof(double));
  of_filter_params_t f = s.filter;
  f.levels = 1;
  const uint16_t *src = d_newDepth ? d_newDepth : d_cameraData.depth;
  if (d_newDepth && d_cameraData.depth && d_newDepth != d_cameraData.depth)
    cudaMemcpyAsync(d_cameraData.depth, d_newDepth, (size_t)cam.width * cam.height * 2,
                    cudaMemcpyDeviceToDevice, stream);
  check(of_preprocess(&cam, &f, src, cam.width, frame.ptr, stream), "of_preprocess");
  check(of_pose_from_float(d_currentTransform, pose.ptr, 0, stream), "of_pose_from_float");
  check(of_points_to_reference(&cam, frame.ptr, pose.ptr, (float *)d_cameraData.vertex,
                               (float *)d_cameraData.normal, stream),
        "of_points_to_reference");
  cudaStreamSynchronize(stream);
}

}  // namespace openfusion
