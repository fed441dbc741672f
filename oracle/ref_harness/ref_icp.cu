// Harness around d_find_corresponding (Source/src/ICP.cu:116-251) and the host
// routine Cpu_buildNewTransformMatrix (ICP.cu:266-321). Test infrastructure.
//
// The kernel is launched with 32x16 = 512-thread blocks: its shared-memory
// tree is written for CORRESPONDENCE_BLOCK = 512 threads (Constants.h:10-11)
// while ICP::FindCorresponding launches 256 (ICP.cu:257), which makes the tree
// read slots no thread wrote. With 512 threads every slot is written.
#include <new>
#include <vector>

#include "ref_common.h"
#include "utilities.h"
#include "CudaUtilities.cuh"
// ICP's members are private by default; the harness reaches the host routine
// Cpu_buildNewTransformMatrix by reading the class as a struct.
#define class struct
#include "ICP.cu"
#undef class

// One correspondence pass. Inputs: new frame depth (uint16) and its world
// vertex/normal maps at the current estimate, the model's world maps, the
// world-to-camera float[16] of the current estimate. Outputs the per-block
// 36 + 6 floats (upper AtA entries are the written ones) and their sum over
// blocks in float, block by block as ICP.cpp:128-135 does.
extern "C" int ref_find_corresponding(const ref_cam *c, const uint16_t *h_depth,
                                      const float *h_new_vertex, const float *h_new_normal,
                                      const float *h_model_vertex, const float *h_model_normal,
                                      const float *h_invT, float *h_AtA_sum, float *h_Atb_sum,
                                      int *blocks_out) {
  CameraParams p;
  memset(&p, 0, sizeof(p));
  p.m_intrinsic.Set(c->fx, c->fy, c->cx, c->cy);
  p.m_invIntrinsic.Set(c->ifx, c->ify, c->icx, c->icy);
  p.m_width = c->w;
  p.m_height = c->h;
  p.m_min_depth = c->dmin;
  p.m_max_depth = c->dmax;
  size_t n = (size_t)c->w * c->h;
  dim3 block(32, 16);
  dim3 grid(iDivUp(c->w, 32), iDivUp(c->h, 16));
  int nblocks = grid.x * grid.y;
  CameraData nd;
  PointInfo model;
  float *AtA = nullptr, *Atb = nullptr, *inv = nullptr;
  REF_TRY(cudaMalloc(&nd.depth, n * 2));
  REF_TRY(cudaMalloc(&nd.vertex, n * sizeof(float3)));
  REF_TRY(cudaMalloc(&nd.normal, n * sizeof(float3)));
  REF_TRY(cudaMalloc(&model.vertex, n * sizeof(float3)));
  REF_TRY(cudaMalloc(&model.normal, n * sizeof(float3)));
  REF_TRY(cudaMalloc(&AtA, (size_t)nblocks * 36 * 4));
  REF_TRY(cudaMalloc(&Atb, (size_t)nblocks * 6 * 4));
  REF_TRY(cudaMalloc(&inv, 64));
  REF_TRY(cudaMemset(AtA, 0, (size_t)nblocks * 36 * 4));
  REF_TRY(cudaMemcpy(nd.depth, h_depth, n * 2, cudaMemcpyHostToDevice));
  REF_TRY(cudaMemcpy(nd.vertex, h_new_vertex, n * 12, cudaMemcpyHostToDevice));
  REF_TRY(cudaMemcpy(nd.normal, h_new_normal, n * 12, cudaMemcpyHostToDevice));
  REF_TRY(cudaMemcpy(model.vertex, h_model_vertex, n * 12, cudaMemcpyHostToDevice));
  REF_TRY(cudaMemcpy(model.normal, h_model_normal, n * 12, cudaMemcpyHostToDevice));
  REF_TRY(cudaMemcpy(inv, h_invT, 64, cudaMemcpyHostToDevice));
  d_find_corresponding<<<grid, block>>>(nd, model, nullptr, nullptr, AtA, Atb, inv, nullptr, p);
  REF_TRY(cudaDeviceSynchronize());
  std::vector<float> a((size_t)nblocks * 36), b((size_t)nblocks * 6);
  REF_TRY(cudaMemcpy(a.data(), AtA, a.size() * 4, cudaMemcpyDeviceToHost));
  REF_TRY(cudaMemcpy(b.data(), Atb, b.size() * 4, cudaMemcpyDeviceToHost));
  for (int j = 0; j < 36; ++j) h_AtA_sum[j] = 0.f;
  for (int j = 0; j < 6; ++j) h_Atb_sum[j] = 0.f;
  for (int i = 0; i < nblocks; ++i) {
    for (int j = 0; j < 36; ++j) h_AtA_sum[j] += a[(size_t)i * 36 + j];
    for (int j = 0; j < 6; ++j) h_Atb_sum[j] += b[(size_t)i * 6 + j];
  }
  *blocks_out = nblocks;
  cudaFree(nd.depth); cudaFree(nd.vertex); cudaFree(nd.normal); cudaFree(model.vertex);
  cudaFree(model.normal); cudaFree(AtA); cudaFree(Atb); cudaFree(inv);
  return 0;
}

// ICP::Cpu_buildNewTransformMatrix (host code): xOpt[6] -> newTransform and
// the accumulated increment, both float[16] in/out. The routine touches no
// member of the object, so it runs on uninitialised storage (the ICP
// constructor would allocate device memory).
extern "C" void ref_build_transform(float *xOpt, float *newTransform, float *fullIncrement) {
  alignas(ICP) static unsigned char storage[sizeof(ICP)];
  reinterpret_cast<ICP *>(storage)->Cpu_buildNewTransformMatrix(xOpt, newTransform, fullIncrement);
}
