// Harness around the camera-side depth filters d_MedianFilter,
// d_GradientFilter, d_AverageFilter and d_undistort
// (Source/src/CameraSupport/CameraAbstract.cu:9-229). Test infrastructure.
#include "CameraAbstract.cu"
#include "ref_common.h"

// kind 0 = median 5x5, 1 = Prewitt gradient, 2 = 8-neighbour average; one
// launch with the reference's block shape, host in / out
extern "C" int ref_depth_filter(int kind, int w, int h, int null_value, const uint16_t *h_in,
                                uint16_t *h_out) {
  const size_t bytes = (size_t)w * h * sizeof(uint16_t);
  uint16_t *din = nullptr, *dout = nullptr;
  REF_TRY(cudaMalloc(&din, bytes));
  REF_TRY(cudaMalloc(&dout, bytes));
  REF_TRY(cudaMemcpy(din, h_in, bytes, cudaMemcpyHostToDevice));
  REF_TRY(cudaMemset(dout, 0, bytes));
  dim3 grid(iDivUp(w, blockSize.x), iDivUp(h, blockSize.y));
  if (kind == 0) d_MedianFilter<<<grid, blockSize>>>(din, dout, w, h, (CAMERA_DEPTH_TYPE)null_value);
  else if (kind == 1) d_GradientFilter<<<grid, blockSize>>>(din, dout, w, h);
  else d_AverageFilter<<<grid, blockSize>>>(din, dout, w, h, (CAMERA_DEPTH_TYPE)null_value);
  REF_TRY(cudaDeviceSynchronize());
  REF_TRY(cudaMemcpy(h_out, dout, bytes, cudaMemcpyDeviceToHost));
  cudaFree(din);
  cudaFree(dout);
  return 0;
}

// d_undistort on a raw frame; the output starts as `fill` (pixels the kernel
// does not write keep it)
extern "C" int ref_undistort(const ref_cam *c, float k1, float k2, float p1, float p2,
                             const uint16_t *h_in, uint16_t *h_out, uint16_t fill) {
  CameraParams p;
  memset(&p, 0, sizeof(p));
  p.m_intrinsic.Set(c->fx, c->fy, c->cx, c->cy);
  p.m_width = c->w;
  p.m_height = c->h;
  p.k1 = k1; p.k2 = k2; p.p1 = p1; p.p2 = p2;
  const size_t n = (size_t)c->w * c->h, bytes = n * sizeof(uint16_t);
  uint16_t *din = nullptr, *dout = nullptr;
  REF_TRY(cudaMalloc(&din, bytes));
  REF_TRY(cudaMalloc(&dout, bytes));
  REF_TRY(cudaMemcpy(din, h_in, bytes, cudaMemcpyHostToDevice));
  for (size_t i = 0; i < n; ++i) h_out[i] = fill;
  REF_TRY(cudaMemcpy(dout, h_out, bytes, cudaMemcpyHostToDevice));
  dim3 grid(iDivUp(c->w, blockSize.x), iDivUp(c->h, blockSize.y));
  d_undistort<<<grid, blockSize>>>(p, din, dout);
  REF_TRY(cudaDeviceSynchronize());
  REF_TRY(cudaMemcpy(h_out, dout, bytes, cudaMemcpyDeviceToHost));
  cudaFree(din);
  cudaFree(dout);
  return 0;
}
