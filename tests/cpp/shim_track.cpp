// Drives the reference-shaped C++ classes of include/openfusion_b200.hpp in the
// reference's per-frame order (Source/src/MainApp.cpp:786-964):
// Integrate(k-1) -> Raycast(k-1) -> new depth(k) -> Iterate_ICP(k) ->
// UpdateTransforms, on a seeded synthetic sequence. Prints one JSON line with
// the largest pose error against the ground truth.
#include <cmath>
#include <cstdio>
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

int main(int argc, char **argv) {
  const int frames = argc > 1 ? std::atoi(argv[1]) : 20;
  const int W = 320, H = 240;
  CameraParams p;
  std::memset(&p, 0, sizeof(p));
  p.m_intrinsic.Set(262.5f, 262.5f, 160.f, 120.f);
  p.m_width = W;
  p.m_height = H;
  p.m_min_depth = 300.f;
  p.m_max_depth = 5000.f;
  Settings s(128, 2000.f, 60.f, 128);

  of_synth_scene_t scene;
  of_synth_scene(0, 1000, 2000.f, &scene);
  std::vector<double> gt((size_t)frames * 16);
  of_synth_trajectory(0, 1001, 2000.f, frames, gt.data());
  std::vector<uint16_t> depth_h((size_t)W * H);

  DeviceBuffer<uint8_t> vol(General::VolumeBytes(s));
  DeviceBuffer<uint16_t> depth((size_t)W * H * 2);
  DeviceBuffer<float3> model_v((size_t)W * H * sizeof(float3)), model_n((size_t)W * H * sizeof(float3));
  DeviceBuffer<float> T(16 * sizeof(float)), invT(16 * sizeof(float));
  DeviceBuffer<float3> campos(sizeof(float3));
  DeviceBuffer<unsigned> rgba((size_t)W * H * 4);

  General general(s);
  general.InitVoxelArray(vol.ptr, nullptr);
  VolumeIntegrator integrator(&p, s);
  Raycaster raycaster(&p, s);
  ICP icp(dim3(), dim3(), &p, s);
  CameraData cd{depth.ptr, nullptr, nullptr};
  PointInfo model{model_v.ptr, model_n.ptr};

  float T0[16];
  for (int i = 0; i < 16; ++i) T0[i] = (float)gt[i];
  cudaMemcpy(T.ptr, T0, sizeof(T0), cudaMemcpyHostToDevice);
  general.UpdateTransforms(T.ptr, invT.ptr, campos.ptr, nullptr);
  of_synth_render(&scene, W, H, 262.5f, 262.5f, 160.f, 120.f, gt.data(), 1002, 0, 1.f, 0.f,
                  depth_h.data(), nullptr);
  cudaMemcpy(depth.ptr, depth_h.data(), depth_h.size() * 2, cudaMemcpyHostToDevice);
  double max_rot = 0.0, max_trans = 0.0;
  int bad_status = 0;
  for (int k = 1; k < frames; ++k) {
    integrator.Integrate(vol.ptr, nullptr, invT.ptr, cd, campos.ptr);
    raycaster.Raycast(rgba.ptr, T.ptr, vol.ptr, model, campos.ptr, false);
    of_synth_render(&scene, W, H, 262.5f, 262.5f, 160.f, 120.f, gt.data() + 16 * k, 1002, k, 1.f,
                    0.f, depth_h.data(), nullptr);
    cudaMemcpy(depth.ptr, depth_h.data(), depth_h.size() * 2, cudaMemcpyHostToDevice);
    icp.Iterate_ICP(cd, model, T.ptr);
    general.UpdateTransforms(T.ptr, invT.ptr, campos.ptr, nullptr);
    if (icp.LastStats().status != 0) ++bad_status;
    float Th[16];
    cudaMemcpy(Th, T.ptr, sizeof(Th), cudaMemcpyDeviceToHost);
    double r, t;
    pose_error(Th, gt.data() + 16 * k, &r, &t);
    max_rot = std::fmax(max_rot, r);
    max_trans = std::fmax(max_trans, t);
  }
  cudaError_t e = cudaDeviceSynchronize();
  std::printf("{\"frames\": %d, \"max_rot_rad\": %.9g, \"max_trans_mm\": %.9g, \"bad_status\": %d, "
              "\"cuda\": \"%s\"}\n",
              frames, max_rot, max_trans, bad_status, cudaGetErrorString(e));
  return e == cudaSuccess ? 0 : 1;
}
