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
//   - the volume geometry and ICP schedule are a Settings value (the reference
//     fixes them at compile time in Constants.h): SetDefaultSettings() once,
//     then construct the modules as the reference does;
//   - modules own their device scratch (allocated in their constructors, as the
//     reference's ICP constructor does, ICP.cpp:26-58); no per-frame call
//     allocates or synchronises -- every call is ordered on its `stream`
//     argument (default: the legacy default stream, the reference's);
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
  size_t bytes = 0;
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t n) { reset(n); }
  ~DeviceBuffer() { if (ptr) cudaFree(ptr); }
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  // (re)allocates `n` bytes; the contents are undefined afterwards
  void reset(size_t n) {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    if (n && cudaMalloc((void **)&ptr, n) != cudaSuccess) throw Error("cudaMalloc", OF_ERR_OUT_OF_MEMORY);
    bytes = n;
  }
};

// The reference fixes its volume geometry and ICP schedule at compile time
// (Constants.h), so its classes take no settings. Modules constructed without
// a Settings argument (and General::Instance()) use these process-wide
// defaults; set them once before constructing the modules.
inline Settings &DefaultSettings() {
  static Settings s;
  return s;
}
inline void SetDefaultSettings(const Settings &s) { DefaultSettings() = s; }

inline size_t pyramid_bytes(const of_camera_t &cam, int32_t levels) {
  of_pyramid_layout_t lay;
  check(of_pyramid_layout(&cam, levels, &lay), "of_pyramid_layout");
  return lay.total_bytes;
}

// General (General.h:6-20): volume reset and pose bookkeeping. The
// reference's callers reach it through the singleton,
// General::Instance()->InitVoxelArray(...) / ->UpdateTransforms(...)
// (MainApp.cpp:442, 598, 953).
class General {
 public:
  explicit General(const Settings &s = DefaultSettings()) : m_s(s), m_pose(16 * sizeof(double)) {}
  // The process-wide instance (General.cpp:50-58), built with DefaultSettings()
  // on first use.
  static General *Instance() {
    static General instance;
    return &instance;
  }
  static size_t VolumeBytes(const Settings &s = DefaultSettings()) {
    size_t b = 0;
    check(of_volume_bytes(&s.volume, &b), "of_volume_bytes");
    return b;
  }
  void InitVoxelArray(VoxelType *d_voxel_array, VoxelWeightType * /*unused*/,
                      cudaStream_t stream = 0) {
    check(of_volume_reset(&m_s.volume, d_voxel_array, stream), "of_volume_reset");
  }
  // d_currentTransform (float[16], camera-to-world) -> its inverse and the
  // camera position (General.cpp:14-40), in FP64 on the device, ordered on
  // `stream` (the reference copies to the host, inverts with Eigen and
  // synchronises the device). No allocation: the FP64 pose buffer is the
  // instance's.
  void UpdateTransforms(float *d_currentTransform, float *d_invCurrentTransform,
                        float3 *d_cameraPosition, float * /*invViewMatrix (UI only)*/,
                        cudaStream_t stream = 0) {
    check(of_pose_from_float(d_currentTransform, m_pose.ptr, 0, stream), "of_pose_from_float");
    check(of_pose_to_float(m_pose.ptr, nullptr, d_invCurrentTransform, (float *)d_cameraPosition,
                           stream),
          "of_pose_to_float");
  }

 private:
  Settings m_s;
  DeviceBuffer<double> m_pose;
};

// VolumeIntegrator (VolumeIntegrator.h:9-17).
class VolumeIntegrator {
 public:
  VolumeIntegrator(CameraParams *cameraParams, const Settings &s = DefaultSettings())
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
  Raycaster(CameraParams *cameraParams, const Settings &s = DefaultSettings())
      : m_cam(to_camera(*cameraParams)), m_s(s), m_model(pyramid_bytes(m_cam, m_s.icp.levels)),
        m_pose(16 * sizeof(double)) {}
  // transform: camera-to-world float[16] on the device. Writes the world
  // vertex/normal maps of `renderedVertexMap` and, if d_output != NULL, the
  // view (Raycaster.cu:214-228): the shaded grey 0.6 (-d . n) + 0.2, or with
  // showNormals the normal as (n + 1) / 2 with alpha 0. Keeps the model
  // pyramid (Model()).
  void Raycast(unsigned *d_output, float *transform, VoxelType *d_voxel_array,
               const PointInfo &renderedVertexMap, const float3 * /*d_cameraPosition*/,
               bool showNormals, cudaStream_t stream = 0) {
    check(of_pose_from_float(transform, m_pose.ptr, 0, stream), "of_pose_from_float");
    check(of_raycast(&m_s.volume, d_voxel_array, &m_cam, &m_s.raycast, m_s.icp.levels, m_pose.ptr,
                     m_model.ptr, showNormals ? nullptr : d_output, stream),
          "of_raycast");
    if (showNormals && d_output)
      check(of_normals_to_rgba(&m_cam, m_model.ptr, nullptr, 0.f, d_output, stream),
            "of_normals_to_rgba");
    if (renderedVertexMap.vertex || renderedVertexMap.normal)
      check(of_points_to_reference(&m_cam, m_model.ptr, nullptr, (float *)renderedVertexMap.vertex,
                                   (float *)renderedVertexMap.normal, stream),
            "of_points_to_reference");
  }
  const void *Model() const { return m_model.ptr; }

 private:
  of_camera_t m_cam;
  Settings m_s;
  DeviceBuffer<uint8_t> m_model;
  DeviceBuffer<double> m_pose;
};

// ICP (ICP.h:50-70).
class ICP {
 public:
  ICP(dim3 /*gridSize*/, dim3 /*blockSize*/, CameraParams *cameraParams,
      const Settings &s = DefaultSettings())
      : m_cam(to_camera(*cameraParams)), m_s(s), m_ws(ws_bytes()), m_pose(16 * sizeof(double)),
        m_stats(sizeof(of_icp_stats_t)), m_system(32 * sizeof(float)) {
    alloc_maps();
    check(cudaMemset(m_ws.ptr, 0, m_ws.bytes) == cudaSuccess ? OF_OK : OF_ERR_CUDA, "cudaMemset");
  }
  // Refines d_currentTransform (float[16] camera-to-world, in/out) of the new
  // depth frame against the rendered model maps (world space): the
  // coarse-to-fine schedule of Settings::icp on the filtered depth pyramid,
  // all on the device, ordered on `stream`.
  void Iterate_ICP(const CameraData &newDepthData, const PointInfo &renderedVertexMap,
                   float *d_currentTransform, cudaStream_t stream = 0) {
    load_maps(newDepthData, renderedVertexMap, stream);
    check(of_pose_from_float(d_currentTransform, m_pose.ptr, 0, stream), "of_pose_from_float");
    check(of_icp_track(&m_cam, &m_s.icp, m_frame.ptr, m_model.ptr, m_pose.ptr, m_ws.ptr,
                       m_stats.ptr, stream),
          "of_icp_track");
    check(of_pose_to_float(m_pose.ptr, d_currentTransform, nullptr, nullptr, stream),
          "of_pose_to_float");
  }
  // One correspondence pass (ICP.cu:254-262) at the finest level for the
  // ICP's current transform (the last Iterate_ICP result, or LoadTransform's):
  // the 21 upper J^T J entries, 6 J^T r entries, sum r^2 and the inlier count
  // into System() (device float[29]).
  void FindCorresponding(const CameraData &newDepthMap, const PointInfo &currentVertexMap,
                         cudaStream_t stream = 0) {
    load_maps(newDepthMap, currentVertexMap, stream);
    check(of_icp_system(&m_cam, &m_s.icp, 0, m_frame.ptr, m_model.ptr, m_pose.ptr, m_ws.ptr,
                        m_system.ptr, stream),
          "of_icp_system");
  }
  // Solves the last FindCorresponding system and left-multiplies the
  // increment into the current transform (ICP.cu:320-340), FP64 on the device.
  // A singular system leaves the transform unchanged (LastStats().status 1).
  void BuildNewTransformMatrix(cudaStream_t stream = 0) {
    check(of_icp_solve_step(m_system.ptr, m_pose.ptr, m_stats.ptr, stream), "of_icp_solve_step");
  }
  // K and K^-1 as 3x3 row-major host arrays (declared in ICP.h:66, never
  // defined in the reference): fx = |K00|, fy = |K11|, cx = K02, cy = K12;
  // the inverse is implied by K and not read.
  void CopyProjectionMatrix(const float *_kMat, const float * /*_kInvMat*/) {
    m_cam.fx = _kMat[0] < 0 ? -_kMat[0] : _kMat[0];
    m_cam.fy = _kMat[4] < 0 ? -_kMat[4] : _kMat[4];
    m_cam.cx = _kMat[2];
    m_cam.cy = _kMat[5];
  }
  // The image size (declared in ICP.h:68, never defined in the reference);
  // the frame and model pyramids are reallocated for it.
  void CopyWidthAndHeight(const int _width, const int _height) {
    m_cam.width = _width;
    m_cam.height = _height;
    alloc_maps();
  }
  // The current transform, set from / written to a device float[16].
  void LoadTransform(const float *d_T, cudaStream_t stream = 0) {
    check(of_pose_from_float(d_T, m_pose.ptr, 0, stream), "of_pose_from_float");
  }
  void StoreTransform(float *d_T, cudaStream_t stream = 0) const {
    check(of_pose_to_float(m_pose.ptr, d_T, nullptr, nullptr, stream), "of_pose_to_float");
  }
  const float *System() const { return m_system.ptr; }
  of_icp_stats_t LastStats(cudaStream_t stream = 0) {
    of_icp_stats_t st;
    cudaMemcpyAsync(&st, m_stats.ptr, sizeof(st), cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    return st;
  }

 private:
  void alloc_maps() {
    const size_t b = pyramid_bytes(m_cam, m_s.icp.levels);
    m_frame.reset(b);
    m_model.reset(b);
  }
  // the new depth's filtered pyramid and the model's pyramid from the AoS maps
  void load_maps(const CameraData &depth, const PointInfo &model, cudaStream_t stream) {
    check(of_preprocess(&m_cam, &m_s.filter, depth.depth, m_cam.width, m_frame.ptr, stream),
          "of_preprocess");
    check(of_points_from_reference(&m_cam, m_s.icp.levels, (const float *)model.vertex,
                                   (const float *)model.normal, m_model.ptr, stream),
          "of_points_from_reference");
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
  DeviceBuffer<float> m_system;
};

// CameraHandler (CameraHandler.h:10-31) without a camera driver: its static
// updateCameraData (CameraHandler.cu:134-143) converts a new depth frame into
// the world-space vertex and normal maps of a CameraData, as the reference
// does -- raw depth (no filter), vertex = T K^-1 [u v 1] (-depth) inside
// [min, max] depth and FLT_MAX outside (:65-89), normal = the normalised
// cross product of the forward differences, 0 at an invalid neighbour and on
// the last row and column (:91-132) -- optionally with the depth and normal
// RGBA views (:75-78, :128-131). Like the reference's, it reads the camera
// parameters from a static member, set here by the constructor or
// SetCameraParams. Its scratch (one pyramid level and an FP64 pose) is
// allocated once per parameter set; the call is ordered on `stream` and does
// not synchronise.
class CameraHandler {
 public:
  explicit CameraHandler(CameraParams *cameraParams) { SetCameraParams(*cameraParams); }
  CameraParams *GetCameraParams() { return &state().params; }
  static void SetCameraParams(const CameraParams &p) {
    State &st = state();
    st.params = p;
    st.cam = to_camera(p);
    st.frame.reset(pyramid_bytes(st.cam, 1));
    if (!st.pose.ptr) st.pose.reset(16 * sizeof(double));
  }
  static void updateCameraData(dim3 /*gridSize*/, dim3 /*blockSize*/, const CameraData &d_cameraData,
                               uint16_t *d_newDepth, float *d_currentTransform,
                               unsigned *newNormalMap, unsigned *newDepthMap,
                               cudaStream_t stream = 0) {
    State &st = state();
    if (!st.frame.ptr) throw Error("CameraHandler::updateCameraData before SetCameraParams",
                                   OF_ERR_NOT_READY);
    const of_camera_t &cam = st.cam;
    if (d_newDepth && d_newDepth != d_cameraData.depth &&
        cudaMemcpyAsync(d_cameraData.depth, d_newDepth, (size_t)cam.width * cam.height * 2,
                        cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
      throw Error("cudaMemcpyAsync", OF_ERR_CUDA);
    of_filter_params_t raw;
    of_default_params(&raw, nullptr, nullptr);
    raw.radius_px = -1;  // the reference converts the raw depth
    raw.levels = 1;
    check(of_preprocess(&cam, &raw, d_cameraData.depth, cam.width, st.frame.ptr, stream),
          "of_preprocess");
    check(of_pose_from_float(d_currentTransform, st.pose.ptr, 0, stream), "of_pose_from_float");
    check(of_points_to_reference(&cam, st.frame.ptr, st.pose.ptr, (float *)d_cameraData.vertex,
                                 (float *)d_cameraData.normal, stream),
          "of_points_to_reference");
    if (newDepthMap)
      check(of_depth_to_rgba(&cam, d_cameraData.depth, newDepthMap, stream), "of_depth_to_rgba");
    if (newNormalMap)
      check(of_normals_to_rgba(&cam, st.frame.ptr, st.pose.ptr, 1.f, newNormalMap, stream),
            "of_normals_to_rgba");
  }

 private:
  struct State {
    CameraParams params{};
    of_camera_t cam{};
    DeviceBuffer<uint8_t> frame;
    DeviceBuffer<double> pose;
  };
  static State &state() {
    static State s;
    return s;
  }
};

// The free-function form of updateCameraData kept for earlier callers.
inline void updateCameraData(const CameraParams &params, const CameraData &d_cameraData,
                             uint16_t *d_newDepth, float *d_currentTransform,
                             cudaStream_t stream = 0) {
  CameraHandler::SetCameraParams(params);
  CameraHandler::updateCameraData(dim3(), dim3(), d_cameraData, d_newDepth, d_currentTransform,
                                  nullptr, nullptr, stream);
}

}  // namespace openfusion
