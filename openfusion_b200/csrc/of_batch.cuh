// of_batch.cuh -- internal interface of the batched stages: many independent
// depth streams (each its own camera, volume, pose and buffers) processed by
// one launch per stage.
//
// Every batched launch is a flat grid over all streams' blocks: block b
// belongs to job j with first[j] <= b < first[j + 1] and runs the same body as
// the single-stream kernel with the local block index b - first[j], so a
// batched stage writes, per stream, exactly what the single-stream stage
// writes. Each stage file owns its job table (built once on the host, kept in
// device memory) behind an opaque handle.
#pragma once

#include "of_common.cuh"

namespace of {

// One stream of a batch as the stage launchers see it (device pointers).
struct BatchStream {
  of_camera_t cam;
  of_volume_desc_t vol_desc;
  void *volume;
  const float *lambda;
  void *scratch;  // of_integrate_tiled scratch
  void *frame;    // frame pyramid (of_pyramid_layout)
  void *model;    // model pyramid
  const uint16_t *depth[2];  // depth frames by parity (frame k in depth[k & 1])
  double *pose;
  of_icp_stats_t *stats;
};

struct BatchParams {
  of_filter_params_t filter;
  of_raycast_params_t raycast;
  of_icp_params_t icp;
};

// Tuning knobs of the batched stages. None changes a result: they choose tile
// shapes and block counts only.
struct BatchKnobs {
  int ray_tile;        // raycast block shape: 0 = 16x16, 1 = 32x8, 2 = 8x32, 3 = 32x4,
                       // 4 = 16x8, 5 = 8x16, 6 = 8x8
  int list_div;        // integrate: blocks per stream = ceil(bricks / list_div), capped
  int icp_clusters;    // batched ICP: resident clusters of the persistent grid
};

// Job j's block range in a flat batched grid: first[j] <= b < first[j + 1].
__device__ __forceinline__ int batch_job(const int *__restrict__ first, int n, int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(first + mid) <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Host: copies a job table and its block prefix to the device.
template <class Job>
of_status_t upload_jobs(const Job *jobs, const int *first, int n, Job **d_jobs, int **d_first) {
  *d_jobs = nullptr;
  *d_first = nullptr;
  cudaError_t e = cudaMalloc(d_jobs, sizeof(Job) * (size_t)(n > 0 ? n : 1));
  if (e == cudaSuccess) e = cudaMalloc(d_first, sizeof(int) * (size_t)(n + 1));
  if (e == cudaSuccess) e = cudaMemcpy(*d_jobs, jobs, sizeof(Job) * (size_t)n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(*d_first, first, sizeof(int) * (size_t)(n + 1), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    if (*d_jobs) cudaFree(*d_jobs);
    if (*d_first) cudaFree(*d_first);
    *d_jobs = nullptr;
    *d_first = nullptr;
    return of_set_cuda_error(e);
  }
  return OF_OK;
}

struct PreprocessBatch;
of_status_t preprocess_batch_create(const BatchStream *s, int n, const BatchParams &p,
                                    PreprocessBatch **out);
of_status_t preprocess_batch_launch(const PreprocessBatch *b, int parity, cudaStream_t st);
void preprocess_batch_destroy(PreprocessBatch *b);

struct IntegrateBatch;
of_status_t integrate_batch_create(const BatchStream *s, int n, IntegrateBatch **out);
of_status_t integrate_batch_launch(const IntegrateBatch *b, int parity, const BatchKnobs &k,
                                   cudaStream_t st);
void integrate_batch_destroy(IntegrateBatch *b);

struct RaycastBatch;
of_status_t raycast_batch_create(const BatchStream *s, int n, const BatchParams &p,
                                 RaycastBatch **out);
of_status_t raycast_batch_launch(const RaycastBatch *b, const BatchKnobs &k, cudaStream_t st);
void raycast_batch_destroy(RaycastBatch *b);

struct IcpBatch;
of_status_t icp_batch_create(const BatchStream *s, int n, const BatchParams &p, IcpBatch **out);
of_status_t icp_batch_launch(const IcpBatch *b, const BatchKnobs &k, cudaStream_t st);
void icp_batch_destroy(IcpBatch *b);
int icp_batch_max_clusters();

}  // namespace of
