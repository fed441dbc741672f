// Headless replay of RunApp::display (Source/src/MainApp.cpp:786-964) with the
// reference's own classes and kernels, for timing the reference rebuilt for
// sm_100a: Integrate -> Raycast -> new depth (H2D + updateCameraData) ->
// 15 ICP iterations with the host solve -> General::UpdateTransforms.
// Test infrastructure.
//
// ICP::Iterate_ICP (ICP.cpp:84-182) is restated below step by step with one
// change: its correspondence kernel runs with 512-thread blocks instead of
// ICP::FindCorresponding's 256 (ICP.cu:257), because the kernel's reduction
// tree is written for 512 (Constants.h:10-11) and reads unwritten shared
// memory otherwise; the host sums then cover those blocks.
#include <Eigen/Core>  // before the cutil headers: their min/max macros break Eigen
#include <Eigen/Dense>

#include <chrono>
#include <cmath>
#include <fstream>
#include <iostream>
#include <math.h>
#include <vector>

#include "ref_common.h"
#include "cutil_inline.h"
#include "cutil_math.h"
#include "utilities.h"
#include "CudaUtilities.cuh"
// General's and ICP's members are private by default; this TU reads those
// classes as structs to reach their buffers (system headers come first).
#define class struct
#include "General.cpp"
#include "ICP.cpp"
#undef class
#include "CameraHandler.h"
#include "Raycaster.h"
#include "VolumeIntegrator.h"

// the reference's correspondence kernel, defined in ICP.cu (ref_icp.cu)
__global__ void d_find_corresponding(const CameraData newDepthData, const PointInfo currentVertexMap,
                                     float *A, float *b, float *AtA, float *Atb,
                                     const float *const invLastTransform,
                                     const float *const newTransform, const CameraParams cameraParams);
extern "C" void *ref_volume_device_tsdf(void);
extern "C" int ref_volume_init(void);
extern "C" void ref_set_camera_params(const ref_cam *c);
void *ref_volume_device_weight(void);

namespace {
struct Pipeline {
  CameraParams p;
  dim3 grid;
  CameraData nd;           // newDepthData
  PointInfo model;         // d_renderedVertexMap
  uint16_t *d_new = nullptr;
  float *dT = nullptr, *dInvT = nullptr;
  float3 *dPos = nullptr;
  unsigned *rgba = nullptr;
  ICP *icp = nullptr;
  VolumeIntegrator *vi = nullptr;
  Raycaster *rc = nullptr;
  int frames = 0;
};
Pipeline *g_pl = nullptr;

// ICP::Iterate_ICP (ICP.cpp:84-182) with 512-thread correspondence blocks.
void iterate_icp(Pipeline &P) {
  ICP &icp = *P.icp;
  Eigen::Matrix4f ident;
  ident.setIdentity();
  cutilSafeCall(cudaMemcpy(icp.incrementalTransform, ident.data(), 64, cudaMemcpyHostToDevice));
  cutilSafeCall(cudaMemcpy(icp.newTransform, P.dT, 64, cudaMemcpyDeviceToDevice));
  cutilSafeCall(cudaMemcpy(icp.bestTransform, icp.newTransform, 64, cudaMemcpyDeviceToDevice));
  dim3 block(32, 16);
  dim3 grid(iDivUp(P.p.m_width, 32), iDivUp(P.p.m_height, 16));
  const int nblocks = grid.x * grid.y;
  int it = 0;
  do {
    ++it;
    cutilSafeCall(cudaMemcpy(icp.invLastTransform_host, icp.newTransform, 64, cudaMemcpyDeviceToHost));
    cudaDeviceSynchronize();
    Eigen::Map<Eigen::Matrix<float, 4, 4, Eigen::RowMajor> > inv(icp.invLastTransform_host);
    inv = inv.inverse();
    cutilSafeCall(cudaMemcpy(icp.invLastTransform, icp.invLastTransform_host, 64, cudaMemcpyHostToDevice));
    cudaDeviceSynchronize();
    d_find_corresponding<<<grid, block>>>(P.nd, P.model, icp.d_A_Matrix, icp.d_b_Matrix, icp.AtA,
                                          icp.Atb, icp.invLastTransform, icp.newTransform, P.p);
    cutilSafeCall(cudaDeviceSynchronize());
    icp.ClearHostMatrices();
    cutilSafeCall(cudaMemcpy(icp.AtA_host, icp.AtA, NUM_VARS * NUM_VARS * nblocks * 4, cudaMemcpyDeviceToHost));
    cutilSafeCall(cudaMemcpy(icp.Atb_host, icp.Atb, NUM_VARS * nblocks * 4, cudaMemcpyDeviceToHost));
    for (int i = 0; i < nblocks; ++i) {
      for (int j = 0; j < NUM_VARS * NUM_VARS; ++j) icp.AtA_sum[j] += icp.AtA_host[i * NUM_VARS * NUM_VARS + j];
      for (int j = 0; j < NUM_VARS; ++j) icp.Atb_sum[j] += icp.Atb_host[i * NUM_VARS + j];
    }
    for (int i = 0; i < NUM_VARS; ++i)
      for (int j = 0; j < i; ++j) icp.AtA_sum[i * NUM_VARS + j] = icp.AtA_sum[j * NUM_VARS + i];
    Eigen::Matrix<float, NUM_VARS, NUM_VARS, Eigen::RowMajor> A;
    Eigen::Matrix<float, NUM_VARS, 1> b;
    for (int i = 0; i < NUM_VARS; ++i) {
      b(i) = icp.Atb_sum[i];
      for (int j = 0; j < NUM_VARS; ++j) A(i, j) = icp.AtA_sum[i * NUM_VARS + j];
    }
    float det = A.determinant();
    if (std::isnan(det) || det == 0.f || fabs(det) < _EPSILON_) {
      cutilSafeCall(cudaMemcpy(icp.newTransform, P.dT, 64, cudaMemcpyDeviceToDevice));
      break;
    }
    Eigen::Matrix<float, NUM_VARS, 1> x = A.llt().solve(b).cast<float>();
    for (int i = 0; i < 3; ++i) icp.xOpt_host[i] = -x(i);
    for (int i = 3; i < 6; ++i) icp.xOpt_host[i] = x(i);
    cutilSafeCall(cudaMemcpy(icp.xOpt, icp.xOpt_host, NUM_VARS * 4, cudaMemcpyHostToDevice));
    icp.BuildNewTransformMatrix();
    CameraHandler::updateCameraData(P.grid, blockSize, P.nd, NULL, icp.newTransform, NULL, NULL);
    cutilSafeCall(cudaDeviceSynchronize());
  } while (it < icp.m_maxIterations);
  cutilSafeCall(cudaMemcpy(P.dT, icp.newTransform, 64, cudaMemcpyDeviceToDevice));
}
}  // namespace

extern "C" int ref_pipeline_create(const ref_cam *c, const float *pose0) {
  if (g_pl) return -1;
  ref_set_camera_params(c);
  REF_TRY((cudaError_t)ref_volume_init());
  Pipeline *P = new Pipeline();
  memset(&P->p, 0, sizeof(P->p));
  P->p.m_intrinsic.Set(c->fx, c->fy, c->cx, c->cy);
  P->p.m_invIntrinsic.Set(c->ifx, c->ify, c->icx, c->icy);
  P->p.m_width = c->w;
  P->p.m_height = c->h;
  P->p.m_min_depth = c->dmin;
  P->p.m_max_depth = c->dmax;
  P->grid = dim3(iDivUp(c->w, blockSize.x), iDivUp(c->h, blockSize.y));
  size_t n = (size_t)c->w * c->h;
  REF_TRY(cudaMalloc(&P->nd.depth, n * 2));
  REF_TRY(cudaMalloc(&P->nd.vertex, n * sizeof(float3)));
  REF_TRY(cudaMalloc(&P->nd.normal, n * sizeof(float3)));
  REF_TRY(cudaMalloc(&P->model.vertex, n * sizeof(float3)));
  REF_TRY(cudaMalloc(&P->model.normal, n * sizeof(float3)));
  REF_TRY(cudaMemset(P->model.vertex, 0, n * sizeof(float3)));
  REF_TRY(cudaMemset(P->model.normal, 0, n * sizeof(float3)));
  REF_TRY(cudaMalloc(&P->d_new, n * 2));
  REF_TRY(cudaMalloc(&P->dT, 64));
  REF_TRY(cudaMalloc(&P->dInvT, 64));
  REF_TRY(cudaMalloc(&P->dPos, sizeof(float3)));
  REF_TRY(cudaMalloc(&P->rgba, n * 4));
  REF_TRY(cudaMemcpy(P->dT, pose0, 64, cudaMemcpyHostToDevice));
  P->icp = new ICP(P->grid, blockSize, &P->p);
  P->vi = new VolumeIntegrator(&P->p);
  P->rc = new Raycaster(&P->p);
  General::Instance()->UpdateTransforms(P->dT, P->dInvT, P->dPos, NULL);
  g_pl = P;
  return 0;
}

// One display() iteration with `depth` as the camera's next frame; the first
// call only loads and converts it (RunApp's constructor runs cameraIteration
// before the loop, MainApp.cpp:720-723). Returns the pose after the frame and
// the wall time of the frame in ms.
extern "C" int ref_pipeline_frame(const uint16_t *depth, float *pose_out, double *ms_out) {
  Pipeline &P = *g_pl;
  size_t n = (size_t)P.p.m_width * P.p.m_height;
  auto t0 = std::chrono::steady_clock::now();
  if (P.frames > 0) {
    cudaDeviceSynchronize();
    P.vi->Integrate((VoxelType *)ref_volume_device_tsdf(), (VoxelWeightType *)ref_volume_device_weight(),
                    P.dInvT, P.nd, P.dPos);
    cudaDeviceSynchronize();
    P.rc->Raycast(P.rgba, P.dT, (VoxelType *)ref_volume_device_tsdf(), P.model, P.dPos, false);
  }
  // cameraIteration: the file camera's H2D copy, then updateCameraData
  cutilSafeCall(cudaMemcpy(P.d_new, depth, n * 2, cudaMemcpyHostToDevice));
  CameraHandler::updateCameraData(P.grid, blockSize, P.nd, P.d_new, P.dT, NULL, NULL);
  if (P.frames > 0) {
    cudaDeviceSynchronize();
    iterate_icp(P);
    General::Instance()->UpdateTransforms(P.dT, P.dInvT, P.dPos, NULL);
    cudaDeviceSynchronize();
  }
  auto t1 = std::chrono::steady_clock::now();
  *ms_out = std::chrono::duration<double, std::milli>(t1 - t0).count();
  REF_TRY(cudaMemcpy(pose_out, P.dT, 64, cudaMemcpyDeviceToHost));
  P.frames += 1;
  return (int)cudaGetLastError();
}
