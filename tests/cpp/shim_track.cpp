// Drives the reference-shaped C++ classes of include/openfusion_b200.hpp with
// the reference's own call lines, in its per-frame order
// (Source/src/MainApp.cpp:696-723 for the set-up, :786-964 for a frame):
//   m_volumeIntegrator->Integrate(k-1) -> m_raycaster->Raycast(k-1) ->
//   the new depth's upload + CameraHandler::updateCameraData(k) ->
//   icp_module->Iterate_ICP(k) -> General::Instance()->UpdateTransforms,
// on a seeded synthetic sequence rendered up front. Prints one JSON line with
// the largest pose error against the ground truth and the frames/s of the
// frame loop (CUDA events on the legacy default stream around every frame
// after the first two, the host's synchronous depth upload included, as the
// reference's file camera uploads it).
//
//   shim_track [frames] [c1|c2]
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "openfusion_b200.hpp"
#include "of_synth.h"

using namespace openfusion;

static void pose_error(const float *P, const double *G, double *rot, double *trans) {
  double tr = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) tr += (double)P[4 * k + i] * G[4 * k + i];
  double c = std::fmax(-1.0, std::fmin(1.0, (tr - 1.0) / 2.0));
  *rot = std::acos(c);
  double dx = P[3] - G[3], dy = P[7] - G[7], dz = P[11] - G[11];
  *trans = std::sqrt(dx * dx + dy * dy + dz * dz);
}

struct Workload {
  const char *name;
  int W, H;
  float f, cx, cy;
  int resolution;
  float size_mm, trunc_mm;
  int scene_kind, seed;
  float dropout;
};

int main(int argc, char **argv) {
  const int frames = argc > 1 ? std::atoi(argv[1]) : 20;
  const bool full = argc > 2 && std::strcmp(argv[2], "c2") == 0;
  // the small and the full-size workloads of the Python package's CONFIGS
  const Workload w = full ? Workload{"c2_640x480_512^3", 640, 480, 525.f, 319.5f, 239.5f, 512,
                                     3000.f, 30.f, 1, 2000, 0.02f}
                          : Workload{"c1_320x240_128^3", 320, 240, 262.5f, 160.f, 120.f, 128,
                                     2000.f, 60.f, 0, 1000, 0.f};
  const int W = w.W, H = w.H;

  // ---- what the reference's camera and Constants.h provide
  CameraParams params;
  std::memset(&params, 0, sizeof(params));
  params.m_intrinsic.Set(w.f, w.f, w.cx, w.cy);
  params.m_width = W;
  params.m_height = H;
  params.m_min_depth = 300.f;
  params.m_max_depth = 5000.f;
  SetDefaultSettings(Settings(w.resolution, w.size_mm, w.trunc_mm, 128));

  of_synth_scene_t scene;
  of_synth_scene(w.scene_kind, (uint64_t)w.seed, w.size_mm, &scene);
  std::vector<double> gt((size_t)frames * 16);
  of_synth_trajectory(0, (uint64_t)w.seed + 1, w.size_mm, frames, gt.data());
  std::vector<std::vector<uint16_t>> depth_h((size_t)frames, std::vector<uint16_t>((size_t)W * H));
  for (int k = 0; k < frames; ++k)
    of_synth_render(&scene, W, H, w.f, w.f, w.cx, w.cy, gt.data() + 16 * k, (uint64_t)w.seed + 2,
                    k, 1.f, w.dropout, depth_h[k].data(), nullptr);

  // ---- RunApp::initCudaPointers (MainApp.cpp:591-647): the shared buffers
  const dim3 blockSize(16, 16);
  const dim3 gridSize((W + 15) / 16, (H + 15) / 16);
  DeviceBuffer<uint8_t> voxels(General::VolumeBytes());
  VoxelType *d_voxel_array = voxels.ptr;
  VoxelWeightType *d_weight_array = nullptr;  // the weights live in the voxel words
  DeviceBuffer<uint16_t> new_depth((size_t)W * H * 2), depth((size_t)W * H * 2);
  DeviceBuffer<float3> nv((size_t)W * H * sizeof(float3)), nn((size_t)W * H * sizeof(float3));
  DeviceBuffer<float3> mv((size_t)W * H * sizeof(float3)), mn((size_t)W * H * sizeof(float3));
  DeviceBuffer<float> T(16 * sizeof(float)), invT(16 * sizeof(float));
  DeviceBuffer<float3> campos(sizeof(float3));
  DeviceBuffer<unsigned> rgba((size_t)W * H * 4), normal_rgba((size_t)W * H * 4),
      depth_rgba((size_t)W * H * 4);
  uint16_t *d_newDepthMap = new_depth.ptr;
  CameraData newDepthData{depth.ptr, nv.ptr, nn.ptr};
  PointInfo d_renderedVertexMap{mv.ptr, mn.ptr};
  float *d_currentTransform = T.ptr, *d_invCurrentTransform = invT.ptr;
  float3 *d_cameraPosition = campos.ptr;
  unsigned *d_output = rgba.ptr, *newNormalMap = normal_rgba.ptr, *newDepthMap = depth_rgba.ptr;
  const bool showNormalsFlag = false;
  float T0[16];
  for (int i = 0; i < 16; ++i) T0[i] = (float)gt[i];
  cudaMemcpy(d_currentTransform, T0, sizeof(T0), cudaMemcpyHostToDevice);

  // ---- RunApp's constructor (MainApp.cpp:696-723)
  CameraHandler *cameraHandler = new CameraHandler(&params);
  Raycaster *m_raycaster = new Raycaster(cameraHandler->GetCameraParams());
  ICP *icp_module = new ICP(gridSize, blockSize, cameraHandler->GetCameraParams());
  VolumeIntegrator *m_volumeIntegrator = new VolumeIntegrator(cameraHandler->GetCameraParams());
  General::Instance()->InitVoxelArray(d_voxel_array, d_weight_array);
  General::Instance()->UpdateTransforms(d_currentTransform, d_invCurrentTransform, d_cameraPosition,
                                        NULL);
  cudaMemcpy(d_newDepthMap, depth_h[0].data(), (size_t)W * H * 2, cudaMemcpyHostToDevice);
  CameraHandler::updateCameraData(gridSize, blockSize, newDepthData, d_newDepthMap,
                                  d_currentTransform, newNormalMap, newDepthMap);

  double max_rot = 0.0, max_trans = 0.0;
  int bad_status = 0;
  const int warm = frames > 4 ? 2 : 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int k = 1; k < frames; ++k) {
    if (k == 1 + warm) cudaEventRecord(e0, 0);
    // RunApp::display (MainApp.cpp:786-964)
    m_volumeIntegrator->Integrate(d_voxel_array, d_weight_array, d_invCurrentTransform, newDepthData, d_cameraPosition);
    m_raycaster->Raycast(d_output, d_currentTransform, d_voxel_array, d_renderedVertexMap, d_cameraPosition, showNormalsFlag);
    // cameraIteration (CameraHandler.cpp:70-91): the file camera's upload, then
    // updateCameraData
    cudaMemcpy(d_newDepthMap, depth_h[k].data(), (size_t)W * H * 2, cudaMemcpyHostToDevice);
    CameraHandler::updateCameraData(gridSize, blockSize, newDepthData, d_newDepthMap, d_currentTransform, newNormalMap, newDepthMap);
    icp_module->Iterate_ICP(newDepthData, d_renderedVertexMap, d_currentTransform);
    General::Instance()->UpdateTransforms(d_currentTransform, d_invCurrentTransform, d_cameraPosition, NULL);
  }
  cudaEventRecord(e1, 0);
  cudaError_t e = cudaDeviceSynchronize();
  float loop_ms = 0.f;
  cudaEventElapsedTime(&loop_ms, e0, e1);
  const int timed = frames - 1 - warm;

  {
    // a second pass over the same frames from a fresh volume, reading every
    // frame's status and pose back (outside the timed loop) for the errors
    General::Instance()->InitVoxelArray(d_voxel_array, d_weight_array);
    cudaMemcpy(d_currentTransform, T0, sizeof(T0), cudaMemcpyHostToDevice);
    General::Instance()->UpdateTransforms(d_currentTransform, d_invCurrentTransform,
                                          d_cameraPosition, NULL);
    cudaMemcpy(d_newDepthMap, depth_h[0].data(), (size_t)W * H * 2, cudaMemcpyHostToDevice);
    CameraHandler::updateCameraData(gridSize, blockSize, newDepthData, d_newDepthMap,
                                    d_currentTransform, NULL, NULL);
    for (int k = 1; k < frames; ++k) {
      m_volumeIntegrator->Integrate(d_voxel_array, d_weight_array, d_invCurrentTransform, newDepthData, d_cameraPosition);
      m_raycaster->Raycast(d_output, d_currentTransform, d_voxel_array, d_renderedVertexMap, d_cameraPosition, showNormalsFlag);
      cudaMemcpy(d_newDepthMap, depth_h[k].data(), (size_t)W * H * 2, cudaMemcpyHostToDevice);
      CameraHandler::updateCameraData(gridSize, blockSize, newDepthData, d_newDepthMap, d_currentTransform, NULL, NULL);
      icp_module->Iterate_ICP(newDepthData, d_renderedVertexMap, d_currentTransform);
      General::Instance()->UpdateTransforms(d_currentTransform, d_invCurrentTransform, d_cameraPosition, NULL);
      if (icp_module->LastStats().status != 0) ++bad_status;
      float Th[16];
      cudaMemcpy(Th, d_currentTransform, sizeof(Th), cudaMemcpyDeviceToHost);
      double r, t;
      pose_error(Th, gt.data() + 16 * k, &r, &t);
      max_rot = std::fmax(max_rot, r);
      max_trans = std::fmax(max_trans, t);
    }
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  delete m_volumeIntegrator;
  delete icp_module;
  delete m_raycaster;
  delete cameraHandler;
  std::printf("{\"workload\": \"%s\", \"frames\": %d, \"timed_frames\": %d, "
              "\"frames_per_s\": %.6g, \"ms_per_frame\": %.6g, \"max_rot_rad\": %.9g, "
              "\"max_trans_mm\": %.9g, \"bad_status\": %d, \"cuda\": \"%s\"}\n",
              w.name, frames, timed, timed > 0 ? 1e3 * timed / loop_ms : 0.0,
              timed > 0 ? loop_ms / timed : 0.0, max_rot, max_trans, bad_status,
              cudaGetErrorString(e));
  return e == cudaSuccess ? 0 : 1;
}
