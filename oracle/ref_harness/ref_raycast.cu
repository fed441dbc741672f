// Harness around d_raycast (Source/src/Raycaster.cu:97-230) through the
// reference's Raycaster class, on the volume held by ref_volume.cu. Test
// infrastructure.
#include "Raycaster.cu"
#include "ref_common.h"

extern "C" void *ref_volume_device_tsdf(void);

// camera-to-world float[16] + camera position -> world vertex/normal maps
// (float3 W*H, BAD_VERTEX = FLT_MAX) and the shaded RGBA image.
extern "C" int ref_raycast(const ref_cam *c, const float *h_T, const float *h_campos,
                           float *h_vertex, float *h_normal, uint32_t *h_rgba) {
  CameraParams p;
  memset(&p, 0, sizeof(p));
  p.m_intrinsic.Set(c->fx, c->fy, c->cx, c->cy);
  p.m_invIntrinsic.Set(c->ifx, c->ify, c->icx, c->icy);
  p.m_width = c->w;
  p.m_height = c->h;
  p.m_min_depth = c->dmin;
  p.m_max_depth = c->dmax;
  size_t n = (size_t)c->w * c->h;
  PointInfo pi;
  float *dT = nullptr;
  float3 *dpos = nullptr;
  uint32_t *drgba = nullptr;
  REF_TRY(cudaMalloc(&pi.vertex, n * sizeof(float3)));
  REF_TRY(cudaMalloc(&pi.normal, n * sizeof(float3)));
  REF_TRY(cudaMalloc(&dT, 64));
  REF_TRY(cudaMalloc(&dpos, sizeof(float3)));
  REF_TRY(cudaMalloc(&drgba, n * 4));
  REF_TRY(cudaMemset(pi.vertex, 0, n * sizeof(float3)));
  REF_TRY(cudaMemset(pi.normal, 0, n * sizeof(float3)));
  REF_TRY(cudaMemset(drgba, 0, n * 4));
  REF_TRY(cudaMemcpy(dT, h_T, 64, cudaMemcpyHostToDevice));
  REF_TRY(cudaMemcpy(dpos, h_campos, sizeof(float3), cudaMemcpyHostToDevice));
  Raycaster rc(&p);
  rc.Raycast(drgba, dT, (VoxelType *)ref_volume_device_tsdf(), pi, dpos, false);
  REF_TRY(cudaDeviceSynchronize());
  REF_TRY(cudaMemcpy(h_vertex, pi.vertex, n * sizeof(float3), cudaMemcpyDeviceToHost));
  REF_TRY(cudaMemcpy(h_normal, pi.normal, n * sizeof(float3), cudaMemcpyDeviceToHost));
  REF_TRY(cudaMemcpy(h_rgba, drgba, n * 4, cudaMemcpyDeviceToHost));
  cudaFree(pi.vertex); cudaFree(pi.normal); cudaFree(dT); cudaFree(dpos); cudaFree(drgba);
  return 0;
}
