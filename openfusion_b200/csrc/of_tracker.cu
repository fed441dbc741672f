// of_tracker.cu -- the whole per-frame pipeline, owned state and CUDA graphs.
//
// Replaces RunApp::display (Source/src/MainApp.cpp:786-964) without its host
// round trips: frame k is pre-processed, tracked against the model raycast
// after frame k-1, fused at the tracked pose and raycast at that pose for
// frame k+1. The reference's order (integrate(k-1) -> raycast(k-1) ->
// convert(k) -> ICP(k) -> UpdateTransforms) is the same sequence rotated by
// one stage. The state the reference allocates in RunApp::initCudaPointers
// (MainApp.cpp:591-647) lives here; the per-frame launch sequence is captured
// once as a CUDA graph and replayed.
#include "of_common.cuh"

#include <new>
#include <string.h>

using namespace of;

bool of_camera_valid(const of_camera_t *c);
bool of_volume_valid(const of_volume_desc_t *d);
size_t of_icp_workspace_size();
of_status_t of_icp_launch(const of_camera_t *cam, const of_icp_params_t *ip, const void *d_frame,
                          const void *d_model, double *pose, void *d_ws, of_icp_stats_t *stats,
                          cudaStream_t s, const double *d_warm);
of_status_t of_icp_set_prior(void *d_workspace, const double *prior_host, cudaStream_t s);

struct of_tracker {
  of_tracker_desc_t desc;
  of_pyramid_layout_t lay;
  cudaStream_t cap;
  // the warm-start CNN runs on a branch beside pre-processing (fork / join)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  void *volume = nullptr;
  void *frame = nullptr;
  void *model = nullptr;
  void *icp_ws = nullptr;
  double *pose = nullptr;
  double *hist = nullptr;
  unsigned long long *hist_count = nullptr;
  uint16_t *depth = nullptr;
  float *lambda = nullptr;
  void *scratch = nullptr;
  of_icp_stats_t *stats = nullptr;
  // learned warm start (desc.warm_start_weights != NULL)
  bool warm = false;
  float *cnn_master = nullptr;
  uint16_t *cnn_params = nullptr;
  void *cnn_ws = nullptr;
  uint16_t *cnn_in = nullptr;
  float *cnn_cells = nullptr;
  float *cnn_out = nullptr;
  double *warm_pose = nullptr;
  uint16_t *prev_depth = nullptr;
  int hist_cap = 1024;
  int64_t frames = 0;
  int kernels_first = 0;
  int kernels_track = 0;
  cudaGraphExec_t g_first = nullptr;
  cudaGraphExec_t g_track = nullptr;
};

namespace {

__global__ void k_record_pose(const double *pose, double *hist, unsigned long long *count,
                              int cap) {
  if (threadIdx.x != 0) return;
  unsigned long long c = *count;
  double *dst = hist + (size_t)(c % (unsigned long long)cap) * 16;
  for (int i = 0; i < 16; ++i) dst[i] = pose[i];
  *count = c + 1;
}

of_status_t enqueue_frame(of_tracker *t, bool track, cudaStream_t s) {
  const of_tracker_desc_t &d = t->desc;
  of_status_t st;
  if (track) {
    if (t->warm) {
      // the CNN's motion estimate between the previous and this depth frame,
      // on a branch that runs beside pre-processing and joins before ICP
      OF_CUDA_TRY(cudaEventRecord(t->ev_fork, s));
      OF_CUDA_TRY(cudaStreamWaitEvent(t->side, t->ev_fork, 0));
      st = of_cnn_predict(t->cnn_params, t->cnn_master, t->prev_depth, t->depth, d.camera.width,
                          d.camera.height, t->pose, t->cnn_out, t->warm_pose, t->side);
      OF_CUDA_TRY(cudaEventRecord(t->ev_join, t->side));
      if (st != OF_OK) {
        cudaStreamWaitEvent(s, t->ev_join, 0);
        return st;
      }
    }
    st = of_preprocess(&d.camera, &d.filter, t->depth, d.camera.width, t->frame, s);
    if (t->warm) OF_CUDA_TRY(cudaStreamWaitEvent(s, t->ev_join, 0));
    if (st != OF_OK) return st;
    st = of_icp_launch(&d.camera, &d.icp, t->frame, t->model, t->pose, t->icp_ws, t->stats, s,
                       t->warm ? t->warm_pose : nullptr);
    if (st != OF_OK) return st;
  }
  st = of_integrate_tiled(&d.volume, t->volume, &d.camera, t->depth, d.camera.width, t->pose,
                          t->lambda, t->scratch, s);
  if (st != OF_OK) return st;
  st = of_raycast(&d.volume, t->volume, &d.camera, &d.raycast, d.icp.levels, t->pose, t->model,
                  nullptr, s);
  if (st != OF_OK) return st;
  k_record_pose<<<1, 32, 0, s>>>(t->pose, t->hist, t->hist_count, t->hist_cap);
  st = of_launch_status();
  if (st == OF_OK && t->warm)  // the next frame's pair
    OF_CUDA_TRY(cudaMemcpyAsync(t->prev_depth, t->depth,
                                (size_t)d.camera.width * d.camera.height * sizeof(uint16_t),
                                cudaMemcpyDeviceToDevice, s));
  return st;
}

int count_kernel_nodes(cudaGraph_t g) {
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return 0;
  cudaGraphNode_t *nodes = new cudaGraphNode_t[n];
  int k = 0;
  if (cudaGraphGetNodes(g, nodes, &n) == cudaSuccess)
    for (size_t i = 0; i < n; ++i) {
      cudaGraphNodeType ty;
      if (cudaGraphNodeGetType(nodes[i], &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++k;
    }
  delete[] nodes;
  return k;
}

of_status_t capture(of_tracker *t, bool track, cudaGraphExec_t *out) {
  cudaGraph_t g = nullptr;
  OF_CUDA_TRY(cudaStreamBeginCapture(t->cap, cudaStreamCaptureModeThreadLocal));
  of_status_t st = enqueue_frame(t, track, t->cap);
  cudaError_t e = cudaStreamEndCapture(t->cap, &g);
  if (st != OF_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) return of_set_cuda_error(e);
  (track ? t->kernels_track : t->kernels_first) = count_kernel_nodes(g);
  e = cudaGraphInstantiateWithFlags(out, g, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return of_set_cuda_error(e);
  return OF_OK;
}

void release(of_tracker *t) {
  if (t->g_first) cudaGraphExecDestroy(t->g_first);
  if (t->g_track) cudaGraphExecDestroy(t->g_track);
  void *bufs[] = {t->volume, t->frame, t->model, t->icp_ws, t->pose, t->hist, t->hist_count,
                  t->depth, t->lambda, t->scratch, t->stats, t->cnn_master, t->cnn_params,
                  t->cnn_ws, t->cnn_in, t->cnn_cells, t->cnn_out, t->warm_pose, t->prev_depth};
  for (void *b : bufs)
    if (b) cudaFree(b);
  if (t->cap) cudaStreamDestroy(t->cap);
  if (t->side) cudaStreamDestroy(t->side);
  if (t->ev_fork) cudaEventDestroy(t->ev_fork);
  if (t->ev_join) cudaEventDestroy(t->ev_join);
  delete t;
}

}  // namespace

extern "C" of_status_t of_tracker_create(const of_tracker_desc_t *desc, of_tracker_t *out) {
  if (!desc || !out || !of_camera_valid(&desc->camera) || !of_volume_valid(&desc->volume))
    return OF_ERR_INVALID_ARGUMENT;
  if (desc->filter.levels != desc->icp.levels || desc->icp.levels < 1 ||
      desc->icp.levels > kMaxLevels || desc->pose_history < 0)
    return OF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  of_tracker *t = new (std::nothrow) of_tracker();
  if (!t) return OF_ERR_OUT_OF_MEMORY;
  t->desc = *desc;
  t->hist_cap = desc->pose_history > 0 ? desc->pose_history : 1024;
  of_status_t st = of_pyramid_layout(&desc->camera, desc->icp.levels, &t->lay);
  if (st != OF_OK) { release(t); return st; }
  cudaError_t e = cudaStreamCreateWithFlags(&t->cap, cudaStreamNonBlocking);
  if (e == cudaSuccess && desc->warm_start_weights) {
    // the CNN branch at the greatest priority: its cluster of whole SMs is
    // placed before pre-processing blocks fill them (kept in the graphs by
    // cudaGraphInstantiateFlagUseNodePriority)
    int least = 0, greatest = 0;
    e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&t->side, cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_join, cudaEventDisableTiming);
  }
  if (e != cudaSuccess) { release(t); return of_set_cuda_error(e); }
  size_t vol_bytes = 0, lam_bytes = 0, scratch_bytes = 0;
  of_volume_bytes(&desc->volume, &vol_bytes);
  of_lambda_bytes(&desc->camera, &lam_bytes);
  of_integrate_scratch_bytes(&desc->volume, &desc->camera, &scratch_bytes);
  size_t px = (size_t)desc->camera.width * desc->camera.height;
  int64_t np = 0;
  size_t cnn_ws = 0;
  t->warm = desc->warm_start_weights != nullptr;
  if (t->warm) {
    const int w = desc->camera.width, h = desc->camera.height;
    if (w % 80 || h % 60 || w / 80 != h / 60) { release(t); return OF_ERR_INVALID_ARGUMENT; }
    of_cnn_param_count(&np);
    of_cnn_workspace_bytes(1, &cnn_ws);
  }
  struct { void **p; size_t n; } allocs[] = {
      {&t->volume, vol_bytes},
      {&t->frame, t->lay.total_bytes},
      {&t->model, t->lay.total_bytes},
      {&t->icp_ws, of_icp_workspace_size()},
      {(void **)&t->pose, 16 * sizeof(double)},
      {(void **)&t->hist, (size_t)t->hist_cap * 16 * sizeof(double)},
      {(void **)&t->hist_count, sizeof(unsigned long long)},
      {(void **)&t->depth, px * sizeof(uint16_t)},
      {(void **)&t->lambda, lam_bytes},
      {&t->scratch, scratch_bytes},
      {(void **)&t->stats, sizeof(of_icp_stats_t)},
      {(void **)&t->cnn_master, (size_t)np * sizeof(float)},
      {(void **)&t->cnn_params, (size_t)np * sizeof(uint16_t)},
      {&t->cnn_ws, cnn_ws},
      {(void **)&t->cnn_in, t->warm ? 2 * 60 * 80 * sizeof(uint16_t) : 0},
      {(void **)&t->cnn_cells, t->warm ? 2 * 60 * 80 * sizeof(float) : 0},
      {(void **)&t->cnn_out, t->warm ? 6 * sizeof(float) : 0},
      {(void **)&t->warm_pose, t->warm ? 16 * sizeof(double) : 0},
      {(void **)&t->prev_depth, t->warm ? px * sizeof(uint16_t) : 0},
  };
  for (auto &a : allocs) {
    if (a.n == 0) continue;
    e = cudaMalloc(a.p, a.n);
    if (e != cudaSuccess) {
      cudaGetLastError();
      release(t);
      return e == cudaErrorMemoryAllocation ? OF_ERR_OUT_OF_MEMORY : of_set_cuda_error(e);
    }
  }
  cudaStream_t s = t->cap;
  bool ok = cudaMemsetAsync(t->icp_ws, 0, of_icp_workspace_size(), s) == cudaSuccess &&
            cudaMemsetAsync(t->hist_count, 0, sizeof(unsigned long long), s) == cudaSuccess &&
            cudaMemsetAsync(t->stats, 0, sizeof(of_icp_stats_t), s) == cudaSuccess &&
            cudaMemsetAsync(t->model, 0, t->lay.total_bytes, s) == cudaSuccess &&
            cudaMemsetAsync(t->frame, 0, t->lay.total_bytes, s) == cudaSuccess &&
            cudaMemcpyAsync(t->pose, desc->initial_pose, 16 * sizeof(double),
                            cudaMemcpyHostToDevice, s) == cudaSuccess;
  if (ok && t->warm)
    ok = cudaMemcpyAsync(t->cnn_master, desc->warm_start_weights, (size_t)np * sizeof(float),
                         cudaMemcpyHostToDevice, s) == cudaSuccess &&
         of_cnn_load(t->cnn_master, t->cnn_params, s) == OF_OK;
  if (!ok) { release(t); return of_set_cuda_error(cudaGetLastError()); }
  st = of_volume_reset(&desc->volume, t->volume, s);
  if (st == OF_OK) st = of_lambda_table(&desc->camera, t->lambda, s);
  if (st == OF_OK && cudaStreamSynchronize(s) != cudaSuccess) st = of_set_cuda_error(cudaGetLastError());
  if (st == OF_OK && desc->use_graph) {
    st = capture(t, false, &t->g_first);
    if (st == OF_OK) st = capture(t, true, &t->g_track);
  }
  if (st != OF_OK) { release(t); return st; }
  *out = t;
  return OF_OK;
}

extern "C" of_status_t of_tracker_destroy(of_tracker_t t) {
  if (!t) return OF_ERR_INVALID_ARGUMENT;
  cudaDeviceSynchronize();
  release(t);
  return OF_OK;
}

extern "C" of_status_t of_tracker_process(of_tracker_t t, const uint16_t *depth, int32_t on_host,
                                          of_stream_t stream) {
  if (!t || !depth) return OF_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  size_t bytes = (size_t)t->desc.camera.width * t->desc.camera.height * sizeof(uint16_t);
  if (on_host) {
    OF_CUDA_TRY(cudaMemcpyAsync(t->depth, depth, bytes, cudaMemcpyHostToDevice, s));
  } else if (depth != t->depth) {
    OF_CUDA_TRY(cudaMemcpyAsync(t->depth, depth, bytes, cudaMemcpyDeviceToDevice, s));
  }
  bool track = t->frames > 0;
  if (t->desc.use_graph) {
    OF_CUDA_TRY(cudaGraphLaunch(track ? t->g_track : t->g_first, s));
  } else {
    of_status_t st = enqueue_frame(t, track, s);
    if (st != OF_OK) return st;
  }
  t->frames += 1;
  return OF_OK;
}

extern "C" of_status_t of_tracker_set_prior(of_tracker_t t, const double *delta) {
  if (!t) return OF_ERR_INVALID_ARGUMENT;
  of_status_t st = of_icp_set_prior(t->icp_ws, delta, t->cap);
  if (st != OF_OK) return st;
  OF_CUDA_TRY(cudaStreamSynchronize(t->cap));
  return OF_OK;
}

extern "C" of_status_t of_tracker_pose(of_tracker_t t, double *pose, of_icp_stats_t *stats,
                                       of_stream_t stream) {
  if (!t || !pose) return OF_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  OF_CUDA_TRY(cudaMemcpyAsync(pose, t->pose, 16 * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (stats)
    OF_CUDA_TRY(cudaMemcpyAsync(stats, t->stats, sizeof(of_icp_stats_t), cudaMemcpyDeviceToHost, s));
  return OF_OK;
}

extern "C" of_status_t of_tracker_pose_history(of_tracker_t t, double *poses, int32_t count,
                                               of_stream_t stream) {
  if (!t || !poses || count < 0 || count > t->hist_cap || count > t->frames)
    return OF_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  OF_CUDA_TRY(cudaStreamSynchronize(s));
  int64_t first = t->frames - count;
  for (int32_t i = 0; i < count; ++i) {
    int64_t slot = (first + i) % t->hist_cap;
    OF_CUDA_TRY(cudaMemcpy(poses + 16 * (size_t)i, t->hist + 16 * (size_t)slot,
                           16 * sizeof(double), cudaMemcpyDeviceToHost));
  }
  return OF_OK;
}

extern "C" of_status_t of_tracker_buffers(of_tracker_t t, of_tracker_buffers_t *out) {
  if (!t || !out) return OF_ERR_INVALID_ARGUMENT;
  out->volume = t->volume;
  out->frame = t->frame;
  out->model = t->model;
  out->pose = t->pose;
  out->depth = t->depth;
  out->lambda = t->lambda;
  out->stats = t->stats;
  out->frames = t->frames;
  out->kernels_first = t->kernels_first;
  out->kernels_track = t->kernels_track;
  return OF_OK;
}
