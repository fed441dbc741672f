// Harness around d_convertDepthToWorldVertices / d_convertDepthToWorldNormals
// (Source/src/CameraSupport/CameraHandler.cu:65-132). Test infrastructure.
#include "CameraHandler.cu"
#include "ref_common.h"

static CameraParams to_params(const ref_cam *c) {
  CameraParams p;
  memset(&p, 0, sizeof(p));
  p.m_intrinsic.Set(c->fx, c->fy, c->cx, c->cy);
  p.m_invIntrinsic.Set(c->ifx, c->ify, c->icx, c->icy);
  p.m_width = c->w;
  p.m_height = c->h;
  p.m_min_depth = c->dmin;
  p.m_max_depth = c->dmax;
  return p;
}

// depth (uint16 W*H) + camera-to-world pose (float[16]) -> world vertex and
// normal maps (float3 W*H), with the reference's launch shape.
extern "C" int ref_convert(const ref_cam *c, const uint16_t *h_depth, const float *h_T,
                           float *h_vertex, float *h_normal) {
  CameraParams p = to_params(c);
  size_t n = (size_t)c->w * c->h;
  CameraData d;
  uint16_t *dd = nullptr;
  float *dT = nullptr;
  REF_TRY(cudaMalloc(&dd, n * 2));
  REF_TRY(cudaMalloc(&d.vertex, n * sizeof(float3)));
  REF_TRY(cudaMalloc(&d.normal, n * sizeof(float3)));
  REF_TRY(cudaMalloc(&dT, 16 * sizeof(float)));
  d.depth = dd;
  REF_TRY(cudaMemcpy(dd, h_depth, n * 2, cudaMemcpyHostToDevice));
  REF_TRY(cudaMemcpy(dT, h_T, 64, cudaMemcpyHostToDevice));
  dim3 grid(iDivUp(c->w, blockSize.x), iDivUp(c->h, blockSize.y));
  d_convertDepthToWorldVertices<<<grid, blockSize>>>(d, nullptr, dT, nullptr, p);
  REF_TRY(cudaDeviceSynchronize());
  d_convertDepthToWorldNormals<<<grid, blockSize>>>(d, nullptr, p);
  REF_TRY(cudaDeviceSynchronize());
  REF_TRY(cudaMemcpy(h_vertex, d.vertex, n * sizeof(float3), cudaMemcpyDeviceToHost));
  REF_TRY(cudaMemcpy(h_normal, d.normal, n * sizeof(float3), cudaMemcpyDeviceToHost));
  cudaFree(dd); cudaFree(d.vertex); cudaFree(d.normal); cudaFree(dT);
  return 0;
}

// CameraHandler::m_params is a private static set by the CameraHandler
// constructor (CameraHandler.cpp:121), which probes camera hardware; the
// harness sets it directly. An explicit template instantiation may name a
// private member, which yields its address here.
template <typename Tag, typename Tag::type M>
struct ref_member_address {
  friend typename Tag::type ref_get(Tag) { return M; }
};
struct ref_params_tag {
  typedef CameraParams *type;
  friend type ref_get(ref_params_tag);
};
template struct ref_member_address<ref_params_tag, &CameraHandler::m_params>;

extern "C" void ref_set_camera_params(const ref_cam *c) { *ref_get(ref_params_tag()) = to_params(c); }
