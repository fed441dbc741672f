// of_tracker.cu -- the whole per-frame pipeline, owned state and CUDA graphs.
//
// Replaces RunApp::display (Source/src/MainApp.cpp:786-964) without its host
// round trips and in its order: the step that receives depth frame k fuses
// frame k-1 at its tracked pose and raycasts the model there
// (integrate(k-1) -> raycast(k-1)), pre-processes frame k, and tracks frame k
// against that model (convert(k) -> ICP(k)). Pre-processing (and the
// warm-start CNN) depend only on the new depth frame, so they run on graph
// branches beside integrate -> raycast and join before ICP; the last frame is
// fused by the next step or by of_tracker_flush. The depth input is double
// buffered (frame k-1 is fused while frame k is pre-processed). The state the
// reference allocates in RunApp::initCudaPointers (MainApp.cpp:591-647) lives
// here; each step's launch sequence is captured once as a CUDA graph (one per
// depth-buffer parity) and replayed.
#include "of_common.cuh"

#include <algorithm>
#include <new>
#include <stdio.h>
#include <string.h>
#include <vector>

using namespace of;

bool of_camera_valid(const of_camera_t *c);
bool of_volume_valid(const of_volume_desc_t *d);
size_t of_icp_workspace_size();
of_status_t of_icp_launch(const of_camera_t *cam, const of_icp_params_t *ip, const void *d_frame,
                          const void *d_model, double *pose, void *d_ws, of_icp_stats_t *stats,
                          cudaStream_t s, const double *d_warm, double *d_hist,
                          unsigned long long *d_hist_count, int hist_cap);
of_status_t of_icp_set_prior(void *d_workspace, const double *prior_host, cudaStream_t s);
of_status_t of_icp_begin_launch(double *pose, void *d_ws, of_icp_stats_t *stats,
                                const double *d_warm, cudaStream_t s);
of_status_t of_icp_fused_launch(const of_camera_t *cam, const of_icp_params_t *ip,
                                const void *d_frame, const void *d_model, double *pose, void *d_ws,
                                of_icp_stats_t *stats, cudaStream_t s, double *d_hist,
                                unsigned long long *d_hist_count, int hist_cap);


struct of_tracker {
  of_tracker_desc_t desc;
  of_pyramid_layout_t lay;
  cudaStream_t cap;
  // branches of a step: pre-processing at the least stream priority, and the
  // warm-start CNN at the greatest (its cluster of whole SMs is placed before
  // other blocks fill them); the capture stream `cap` carries the critical
  // path between them (kept in the graphs by cudaGraphInstantiateFlagUseNodePriority)
  cudaStream_t pre = nullptr, side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_pre = nullptr, ev_cnn = nullptr, ev_up = nullptr;
  void *volume = nullptr;
  void *frame = nullptr;
  void *model = nullptr;
  void *icp_ws = nullptr;
  double *pose = nullptr;
  double *hist = nullptr;
  unsigned long long *hist_count = nullptr;
  uint16_t *depth[2] = {nullptr, nullptr};  // frame k in depth[k & 1]
  uint16_t *filter_scratch = nullptr;       // camera-side filters (desc.depth_filter)
  float *lambda = nullptr;
  void *scratch = nullptr;
  of_icp_stats_t *stats = nullptr;
  // learned warm start (desc.warm_start_weights != NULL)
  bool warm = false;
  float *cnn_master = nullptr;
  uint16_t *cnn_params = nullptr;
  float *cnn_out = nullptr;
  double *warm_pose = nullptr;
  int hist_cap = 1024;
  int64_t frames = 0;
  bool last_fused = false;  // of_tracker_flush fused the last frame already
  int kernels_first = 0;
  int kernels_track = 0;
  bool tuned = false;  // desc.tune: the online tuning has run
  cudaGraphExec_t g_first = nullptr;
  cudaGraphExec_t g_track[2] = {nullptr, nullptr};
  // The step graphs upload a host frame themselves, at the head of the
  // pre-processing branch (beside the fusion of the previous frame): a memcpy
  // node captured from `stage` and pointed at the caller's pinned buffer at
  // every launch, or disabled when the frame is already on the device. The
  // graphs they were instantiated from stay alive for those node handles.
  cudaGraph_t g_track_src[2] = {nullptr, nullptr};
  cudaGraphNode_t up_node[2] = {nullptr, nullptr};
  uint16_t *stage = nullptr;  // pinned placeholder source of the captured upload
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

// the camera-side filters of the new frame, in place (none when steps = 0)
of_status_t enqueue_filters(of_tracker *t, int cur, cudaStream_t s) {
  if (t->desc.depth_filter.steps == 0) return OF_OK;
  return of_depth_filter(&t->desc.camera, &t->desc.depth_filter, t->depth[cur], t->depth[cur],
                         t->filter_scratch, s);
}

// Frame 0 of a tracker: its pose is the initial pose (fused by the next step).
of_status_t enqueue_first(of_tracker *t, cudaStream_t s) {
  of_status_t st = enqueue_filters(t, 0, s);
  if (st != OF_OK) return st;
  k_record_pose<<<1, 32, 0, s>>>(t->pose, t->hist, t->hist_count, t->hist_cap);
  return of_launch_status();
}

// fuse the frame in `depth` at the current pose and raycast the model there
of_status_t enqueue_fuse(of_tracker *t, const uint16_t *depth, cudaStream_t s) {
  const of_tracker_desc_t &d = t->desc;
  of_status_t st = of_integrate_tiled(&d.volume, t->volume, &d.camera, depth, d.camera.width,
                                      t->pose, t->lambda, t->scratch, s);
  if (st != OF_OK) return st;
  return of_raycast(&d.volume, t->volume, &d.camera, &d.raycast, d.icp.levels, t->pose, t->model,
                    nullptr, s);
}

// The step of frame k >= 1 (depth[cur]): integrate(k-1) -> raycast(k-1) on
// `s`, beside pre-process(k) and the CNN(k-1, k) on their branches, each
// branch closed by the frame's ICP start (the begin kernel, which reads only
// the previous pose: after the CNN when it predicts the warm start, else
// after pre-processing); ICP(k) after the join. `fuse` = false when
// of_tracker_flush fused frame k-1.
// `upload` (may be null): a pinned host frame that the pre-processing branch
// copies into depth[cur] before anything reads it (the camera-side filters
// follow on that branch, and the CNN branch waits for both).
of_status_t enqueue_track(of_tracker *t, int cur, bool fuse, cudaStream_t s,
                          const uint16_t *upload = nullptr) {
  const of_tracker_desc_t &d = t->desc;
  const uint16_t *now = t->depth[cur], *before = t->depth[cur ^ 1];
  OF_CUDA_TRY(cudaEventRecord(t->ev_fork, s));  // nothing has forked before this
  // From the fork on, a failed call is remembered rather than returned at
  // once, so that every branch that forked also joins `s` before the error is
  // returned (a capture must end joined).
  cudaError_t first = cudaSuccess;
  auto ok = [&first](cudaError_t e) {
    if (e != cudaSuccess && first == cudaSuccess) first = e;
    return e == cudaSuccess;
  };
  const bool pre_forked = ok(cudaStreamWaitEvent(t->pre, t->ev_fork, 0));
  of_status_t st = OF_OK, sp = OF_OK, sb = OF_OK, sflt = OF_OK;
  bool up_recorded = false;
  if (pre_forked) {
    const size_t bytes = (size_t)d.camera.width * d.camera.height * sizeof(uint16_t);
    if (upload)
      ok(cudaMemcpyAsync(t->depth[cur], upload, bytes, cudaMemcpyHostToDevice, t->pre));
    sflt = enqueue_filters(t, cur, t->pre);
    up_recorded = t->warm && ok(cudaEventRecord(t->ev_up, t->pre));
  }
  const bool side_forked = up_recorded && ok(cudaStreamWaitEvent(t->side, t->ev_up, 0));
  bool cnn_recorded = false, pre_recorded = false;
  if (side_forked) {
    st = of_cnn_predict(t->cnn_params, t->cnn_master, before, now, d.camera.width,
                        d.camera.height, t->pose, t->cnn_out, t->warm_pose, t->side);
    if (st == OF_OK) sb = of_icp_begin_launch(t->pose, t->icp_ws, t->stats, t->warm_pose, t->side);
    cnn_recorded = ok(cudaEventRecord(t->ev_cnn, t->side));
  }
  if (pre_forked) {
    if (sflt == OF_OK) sp = of_preprocess(&d.camera, &d.filter, now, d.camera.width, t->frame, t->pre);
    if (sp == OF_OK && !t->warm)
      sb = of_icp_begin_launch(t->pose, t->icp_ws, t->stats, nullptr, t->pre);
    pre_recorded = ok(cudaEventRecord(t->ev_pre, t->pre));
  }
  of_status_t sf = fuse ? enqueue_fuse(t, before, s) : OF_OK;
  if (pre_recorded) ok(cudaStreamWaitEvent(s, t->ev_pre, 0));
  if (cnn_recorded) ok(cudaStreamWaitEvent(s, t->ev_cnn, 0));
  if (first != cudaSuccess) return of_set_cuda_error(first);
  if (sflt != OF_OK) return sflt;
  if (st != OF_OK) return st;
  if (sp != OF_OK) return sp;
  if (sb != OF_OK) return sb;
  if (sf != OF_OK) return sf;
  // the ICP kernel appends the frame's pose to the history itself
  return of_icp_fused_launch(&d.camera, &d.icp, t->frame, t->model, t->pose, t->icp_ws, t->stats,
                             s, t->hist, t->hist_count, t->hist_cap);
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

// the graph's memcpy node whose source is `src` (the captured upload)
cudaGraphNode_t find_upload(cudaGraph_t g, const void *src) {
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return nullptr;
  cudaGraphNode_t *nodes = new cudaGraphNode_t[n];
  cudaGraphNode_t found = nullptr;
  if (cudaGraphGetNodes(g, nodes, &n) == cudaSuccess)
    for (size_t i = 0; i < n && !found; ++i) {
      cudaGraphNodeType ty;
      cudaMemcpy3DParms p = {};
      if (cudaGraphNodeGetType(nodes[i], &ty) == cudaSuccess && ty == cudaGraphNodeTypeMemcpy &&
          cudaGraphMemcpyNodeGetParams(nodes[i], &p) == cudaSuccess && p.srcPtr.ptr == src)
        found = nodes[i];
    }
  delete[] nodes;
  return found;
}

// graph of frame 0 (cur < 0) or of a tracking step with depth[cur]; a step
// graph keeps its source graph and its upload node (of_tracker_process points
// the node at each host frame)
of_status_t capture(of_tracker *t, int cur, cudaGraphExec_t *out) {
  cudaGraph_t g = nullptr;
  OF_CUDA_TRY(cudaStreamBeginCapture(t->cap, cudaStreamCaptureModeThreadLocal));
  of_status_t st =
      cur < 0 ? enqueue_first(t, t->cap) : enqueue_track(t, cur, true, t->cap, t->stage);
  cudaError_t e = cudaStreamEndCapture(t->cap, &g);
  if (st != OF_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) return of_set_cuda_error(e);
  (cur >= 0 ? t->kernels_track : t->kernels_first) = count_kernel_nodes(g);
  if (*out) cudaGraphExecDestroy(*out);
  *out = nullptr;
  e = cudaGraphInstantiateWithFlags(out, g, cudaGraphInstantiateFlagUseNodePriority);
  if (e != cudaSuccess || cur < 0) {
    cudaGraphDestroy(g);
    return e != cudaSuccess ? of_set_cuda_error(e) : OF_OK;
  }
  if (t->g_track_src[cur]) cudaGraphDestroy(t->g_track_src[cur]);
  t->g_track_src[cur] = g;
  t->up_node[cur] = find_upload(g, t->stage);
  return t->up_node[cur] ? OF_OK : OF_ERR_CUDA;
}

// The online tuning (desc.tune): every raycast block shape kTuneReps times,
// the shapes interleaved (round r times every shape once), on the volume as
// this step left it, at the tracked pose, into a scratch pyramid (the
// tracker's model is left alone); CUDA events on `s`. The shape with the
// least median time wins (the shapes' times lie within a few percent of each
// other, so one run each picks by noise). Then the step graphs are captured
// with the winner.
constexpr int kTuneTiles = 7;  // every shape of of_raycast_params_t.tile
constexpr int kTuneReps = 5;
of_status_t tune_shapes(of_tracker *t, cudaStream_t s) {
  void *tmp = nullptr;
  cudaEvent_t ev[2 * kTuneTiles * kTuneReps] = {};
  of_status_t st = OF_OK;
  cudaError_t e = cudaMalloc(&tmp, t->lay.total_bytes);
  for (int i = 0; e == cudaSuccess && i < 2 * kTuneTiles * kTuneReps; ++i) e = cudaEventCreate(&ev[i]);
  for (int r = 0; r < kTuneReps && e == cudaSuccess && st == OF_OK; ++r)
    for (int c = 0; c < kTuneTiles && e == cudaSuccess && st == OF_OK; ++c) {
      const int i = 2 * (c * kTuneReps + r);
      of_raycast_params_t rp = t->desc.raycast;
      rp.tile = c;
      e = cudaEventRecord(ev[i], s);
      if (e == cudaSuccess)
        st = of_raycast(&t->desc.volume, t->volume, &t->desc.camera, &rp, t->desc.icp.levels,
                        t->pose, tmp, nullptr, s);
      if (e == cudaSuccess && st == OF_OK) e = cudaEventRecord(ev[i + 1], s);
    }
  if (e == cudaSuccess && st == OF_OK) e = cudaStreamSynchronize(s);
  int best = t->desc.raycast.tile;
  float best_ms = 1e30f;
  for (int c = 0; c < kTuneTiles && e == cudaSuccess && st == OF_OK; ++c) {
    float ms[kTuneReps];
    for (int r = 0; r < kTuneReps && e == cudaSuccess; ++r) {
      const int i = 2 * (c * kTuneReps + r);
      e = cudaEventElapsedTime(&ms[r], ev[i], ev[i + 1]);
    }
    if (e != cudaSuccess) break;
    std::sort(ms, ms + kTuneReps);
    const float med = ms[kTuneReps / 2];
    if (med < best_ms) { best_ms = med; best = c; }
  }
  for (cudaEvent_t x : ev)
    if (x) cudaEventDestroy(x);
  if (tmp) cudaFree(tmp);
  if (st != OF_OK) return st;
  if (e != cudaSuccess) return of_set_cuda_error(e);
  t->desc.raycast.tile = best;
  t->tuned = true;
  if (t->desc.use_graph) {
    st = capture(t, 0, &t->g_track[0]);
    if (st == OF_OK) st = capture(t, 1, &t->g_track[1]);
  }
  return st;
}

void release(of_tracker *t) {
  if (t->g_first) cudaGraphExecDestroy(t->g_first);
  for (cudaGraphExec_t g : t->g_track)
    if (g) cudaGraphExecDestroy(g);
  for (cudaGraph_t g : t->g_track_src)
    if (g) cudaGraphDestroy(g);
  if (t->stage) cudaFreeHost(t->stage);
  void *bufs[] = {t->volume, t->frame, t->model, t->icp_ws, t->pose, t->hist, t->hist_count,
                  t->depth[0], t->depth[1], t->filter_scratch, t->lambda, t->scratch, t->stats, t->cnn_master,
                  t->cnn_params, t->cnn_out, t->warm_pose};
  for (void *b : bufs)
    if (b) cudaFree(b);
  for (cudaStream_t q : {t->cap, t->pre, t->side})
    if (q) cudaStreamDestroy(q);
  for (cudaEvent_t ev : {t->ev_fork, t->ev_pre, t->ev_cnn, t->ev_up})
    if (ev) cudaEventDestroy(ev);
  delete t;
}

}  // namespace

extern "C" of_status_t of_tracker_create(const of_tracker_desc_t *desc, of_tracker_t *out) {
  if (!desc || !out || !of_camera_valid(&desc->camera) || !of_volume_valid(&desc->volume))
    return OF_ERR_INVALID_ARGUMENT;
  if (desc->filter.levels != desc->icp.levels || desc->icp.levels < 1 ||
      desc->icp.levels > kMaxLevels || desc->pose_history < 0 || desc->tune < 0)
    return OF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  of_tracker *t = new (std::nothrow) of_tracker();
  if (!t) return OF_ERR_OUT_OF_MEMORY;
  t->desc = *desc;
  t->hist_cap = desc->pose_history > 0 ? desc->pose_history : 1024;
  of_status_t st = of_pyramid_layout(&desc->camera, desc->icp.levels, &t->lay);
  if (st != OF_OK) { release(t); return st; }
  // Stream priorities, kept in the step graphs as node priorities: the
  // critical path (fusion -> raycast -> ICP) above the pre-processing branch,
  // whose blocks fill the SMs that it leaves (measured on B200 at 640x480 /
  // 512^3: 2696 -> 2797 frames/s over 300 steps), and the warm-start CNN
  // branch above both.
  int least = 0, greatest = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  if (e == cudaSuccess)
    e = cudaStreamCreateWithPriority(&t->cap, cudaStreamNonBlocking, (least + greatest) / 2);
  if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&t->pre, cudaStreamNonBlocking, least);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_pre, cudaEventDisableTiming);
  if (e == cudaSuccess && desc->warm_start_weights) {
    e = cudaStreamCreateWithPriority(&t->side, cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_cnn, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_up, cudaEventDisableTiming);
  }
  if (e == cudaSuccess && desc->use_graph)
    e = cudaMallocHost((void **)&t->stage, (size_t)desc->camera.width * desc->camera.height *
                                               sizeof(uint16_t));
  if (e != cudaSuccess) { release(t); return of_set_cuda_error(e); }
  size_t vol_bytes = 0, lam_bytes = 0, scratch_bytes = 0;
  of_volume_bytes(&desc->volume, &vol_bytes);
  of_lambda_bytes(&desc->camera, &lam_bytes);
  of_integrate_scratch_bytes(&desc->volume, &desc->camera, &scratch_bytes);
  size_t px = (size_t)desc->camera.width * desc->camera.height;
  int64_t np = 0;
  t->warm = desc->warm_start_weights != nullptr;
  if (t->warm) {
    const int w = desc->camera.width, h = desc->camera.height;
    if (w % 80 || h % 60 || w / 80 != h / 60) { release(t); return OF_ERR_INVALID_ARGUMENT; }
    of_cnn_param_count(&np);
  }
  struct { void **p; size_t n; } allocs[] = {
      {&t->volume, vol_bytes},
      {&t->frame, t->lay.total_bytes},
      {&t->model, t->lay.total_bytes},
      {&t->icp_ws, of_icp_workspace_size()},
      {(void **)&t->pose, 16 * sizeof(double)},
      {(void **)&t->hist, (size_t)t->hist_cap * 16 * sizeof(double)},
      {(void **)&t->hist_count, sizeof(unsigned long long)},
      {(void **)&t->depth[0], px * sizeof(uint16_t)},
      {(void **)&t->depth[1], px * sizeof(uint16_t)},
      {(void **)&t->filter_scratch, desc->depth_filter.steps ? px * sizeof(uint16_t) : 0},
      {(void **)&t->lambda, lam_bytes},
      {&t->scratch, scratch_bytes},
      {(void **)&t->stats, sizeof(of_icp_stats_t)},
      {(void **)&t->cnn_master, (size_t)np * sizeof(float)},
      {(void **)&t->cnn_params, (size_t)np * sizeof(uint16_t)},
      {(void **)&t->cnn_out, t->warm ? 6 * sizeof(float) : 0},
      {(void **)&t->warm_pose, t->warm ? 16 * sizeof(double) : 0},
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
  // with online tuning the step graphs are captured once the shapes are chosen
  if (st == OF_OK && desc->use_graph) {
    st = capture(t, -1, &t->g_first);
    if (st == OF_OK && desc->tune == 0) st = capture(t, 0, &t->g_track[0]);
    if (st == OF_OK && desc->tune == 0) st = capture(t, 1, &t->g_track[1]);
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
  OF_RANGE("of_tracker_process");
  if (!t || !depth) return OF_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  const int cur = (int)(t->frames & 1);
  size_t bytes = (size_t)t->desc.camera.width * t->desc.camera.height * sizeof(uint16_t);
  const bool track = t->frames > 0;
  const bool graphs = t->desc.use_graph && (t->desc.tune == 0 || t->tuned);
  // A step graph uploads a pinned host frame itself, beside the fusion of the
  // previous frame; any other frame is copied before the step, as the eager
  // path does.
  bool in_graph = false;
  if (graphs && track && !t->last_fused && t->up_node[cur]) {
    cudaPointerAttributes a;
    if (on_host && cudaPointerGetAttributes(&a, depth) == cudaSuccess &&
        a.type == cudaMemoryTypeHost)
      in_graph = cudaGraphExecMemcpyNodeSetParams1D(t->g_track[cur], t->up_node[cur],
                                                    t->depth[cur], depth, bytes,
                                                    cudaMemcpyHostToDevice) == cudaSuccess;
    cudaGetLastError();  // a refused update falls back to the copy below
    OF_CUDA_TRY(cudaGraphNodeSetEnabled(t->g_track[cur], t->up_node[cur], in_graph ? 1 : 0));
  }
  if (!in_graph) {
    if (on_host) {
      OF_CUDA_TRY(cudaMemcpyAsync(t->depth[cur], depth, bytes, cudaMemcpyHostToDevice, s));
    } else if (depth != t->depth[cur]) {
      OF_CUDA_TRY(cudaMemcpyAsync(t->depth[cur], depth, bytes, cudaMemcpyDeviceToDevice, s));
    }
  }
  if (t->desc.use_graph && !track) {
    OF_CUDA_TRY(cudaGraphLaunch(t->g_first, s));
  } else if (graphs && !t->last_fused) {
    OF_CUDA_TRY(cudaGraphLaunch(t->g_track[cur], s));
  } else {
    of_status_t st = track ? enqueue_track(t, cur, !t->last_fused, s) : enqueue_first(t, s);
    if (st != OF_OK) return st;
  }
  t->last_fused = false;
  t->frames += 1;
  if (track && t->desc.tune > 0 && !t->tuned && t->frames > t->desc.tune) {
    of_status_t st = tune_shapes(t, s);
    if (st != OF_OK) return st;
  }
  return OF_OK;
}

extern "C" of_status_t of_tracker_flush(of_tracker_t t, of_stream_t stream) {
  if (!t) return OF_ERR_INVALID_ARGUMENT;
  if (t->frames == 0 || t->last_fused) return OF_OK;
  of_status_t st = enqueue_fuse(t, t->depth[(t->frames - 1) & 1], (cudaStream_t)stream);
  if (st != OF_OK) return st;
  t->last_fused = true;
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

extern "C" of_status_t of_tracker_tuning(of_tracker_t t, int32_t *ray_tile, int32_t *tuned) {
  if (!t || !ray_tile || !tuned) return OF_ERR_INVALID_ARGUMENT;
  *ray_tile = t->desc.raycast.tile;
  *tuned = t->tuned ? 1 : 0;
  return OF_OK;
}

extern "C" of_status_t of_tracker_buffers(of_tracker_t t, of_tracker_buffers_t *out) {
  if (!t || !out) return OF_ERR_INVALID_ARGUMENT;
  out->volume = t->volume;
  out->frame = t->frame;
  out->model = t->model;
  out->pose = t->pose;
  out->depth = t->frames > 0 ? t->depth[(t->frames - 1) & 1] : t->depth[0];
  out->lambda = t->lambda;
  out->stats = t->stats;
  out->frames = t->frames;
  out->kernels_first = t->kernels_first;
  out->kernels_track = t->kernels_track;
  return OF_OK;
}

// ---------------------------------------------------------- checkpoints --
//
// A tracker's state as one file: a header (what the state belongs to and the
// scalars), then the pose history, the last depth frame (the next step fuses
// it) and the whole volume buffer (voxel words and the brick bytes). The
// frame and model pyramids are not saved: the next step recomputes both.
// The reference saves the raw float volume only (SavedVolume.raw,
// Source/src/MainApp.cpp:259-268) and the pose on a key press (:430-451).

namespace {

struct CheckpointHeader {
  char magic[8];  // "OFCKPT1\0"
  int32_t abi_version;
  int32_t width, height;
  int32_t resolution, storage;
  float size_mm, trunc_mm;
  int32_t max_weight;
  int32_t last_fused;
  int64_t frames;
  int32_t hist_cap;
  int32_t pad;
  uint64_t hist_count;
  uint64_t volume_bytes;
  double pose[16];
};

const char kCheckpointMagic[8] = {'O', 'F', 'C', 'K', 'P', 'T', '1', 0};

of_status_t write_all(FILE *f, const void *p, size_t n) {
  return fwrite(p, 1, n, f) == n ? OF_OK : OF_ERR_IO;
}
of_status_t read_all(FILE *f, void *p, size_t n) {
  return fread(p, 1, n, f) == n ? OF_OK : OF_ERR_IO;
}

}  // namespace

extern "C" of_status_t of_tracker_save(of_tracker_t t, const char *path, of_stream_t stream) {
  if (!t || !path) return OF_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  OF_CUDA_TRY(cudaStreamSynchronize(s));
  const of_tracker_desc_t &d = t->desc;
  size_t vol_bytes = 0;
  of_volume_bytes(&d.volume, &vol_bytes);
  const size_t px = (size_t)d.camera.width * d.camera.height;
  CheckpointHeader h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, kCheckpointMagic, 8);
  h.abi_version = OF_ABI_VERSION;
  h.width = d.camera.width;
  h.height = d.camera.height;
  h.resolution = d.volume.resolution;
  h.storage = d.volume.storage;
  h.size_mm = d.volume.size_mm;
  h.trunc_mm = d.volume.trunc_mm;
  h.max_weight = d.volume.max_weight;
  h.last_fused = t->last_fused ? 1 : 0;
  h.frames = t->frames;
  h.hist_cap = t->hist_cap;
  h.volume_bytes = vol_bytes;
  std::vector<double> hist((size_t)t->hist_cap * 16);
  std::vector<uint16_t> depth(px);
  std::vector<char> vol(vol_bytes);
  OF_CUDA_TRY(cudaMemcpy(h.pose, t->pose, sizeof(h.pose), cudaMemcpyDeviceToHost));
  OF_CUDA_TRY(cudaMemcpy(&h.hist_count, t->hist_count, sizeof(h.hist_count), cudaMemcpyDeviceToHost));
  OF_CUDA_TRY(cudaMemcpy(hist.data(), t->hist, hist.size() * sizeof(double), cudaMemcpyDeviceToHost));
  if (t->frames > 0)
    OF_CUDA_TRY(cudaMemcpy(depth.data(), t->depth[(t->frames - 1) & 1], px * sizeof(uint16_t),
                           cudaMemcpyDeviceToHost));
  OF_CUDA_TRY(cudaMemcpy(vol.data(), t->volume, vol_bytes, cudaMemcpyDeviceToHost));
  FILE *f = fopen(path, "wb");
  if (!f) return OF_ERR_IO;
  of_status_t st = write_all(f, &h, sizeof(h));
  if (st == OF_OK) st = write_all(f, hist.data(), hist.size() * sizeof(double));
  if (st == OF_OK) st = write_all(f, depth.data(), px * sizeof(uint16_t));
  if (st == OF_OK) st = write_all(f, vol.data(), vol_bytes);
  if (fclose(f) != 0 && st == OF_OK) st = OF_ERR_IO;
  return st;
}

extern "C" of_status_t of_tracker_load(of_tracker_t t, const char *path, of_stream_t stream) {
  if (!t || !path) return OF_ERR_INVALID_ARGUMENT;
  const of_tracker_desc_t &d = t->desc;
  FILE *f = fopen(path, "rb");
  if (!f) return OF_ERR_IO;
  CheckpointHeader h;
  of_status_t st = read_all(f, &h, sizeof(h));
  size_t vol_bytes = 0;
  of_volume_bytes(&d.volume, &vol_bytes);
  const size_t px = (size_t)d.camera.width * d.camera.height;
  if (st == OF_OK &&
      (memcmp(h.magic, kCheckpointMagic, 8) != 0 || h.abi_version != OF_ABI_VERSION ||
       h.width != d.camera.width || h.height != d.camera.height ||
       h.resolution != d.volume.resolution || h.storage != d.volume.storage ||
       h.size_mm != d.volume.size_mm || h.trunc_mm != d.volume.trunc_mm ||
       h.max_weight != d.volume.max_weight || h.volume_bytes != vol_bytes ||
       h.hist_cap != t->hist_cap || h.frames < 0))
    st = OF_ERR_INVALID_ARGUMENT;  // a checkpoint of another configuration
  std::vector<double> hist;
  std::vector<uint16_t> depth;
  std::vector<char> vol;
  if (st == OF_OK) {
    hist.resize((size_t)t->hist_cap * 16);
    depth.resize(px);
    vol.resize(vol_bytes);
    st = read_all(f, hist.data(), hist.size() * sizeof(double));
    if (st == OF_OK) st = read_all(f, depth.data(), px * sizeof(uint16_t));
    if (st == OF_OK) st = read_all(f, vol.data(), vol_bytes);
  }
  fclose(f);
  if (st != OF_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  OF_CUDA_TRY(cudaStreamSynchronize(s));
  OF_CUDA_TRY(cudaMemcpy(t->pose, h.pose, sizeof(h.pose), cudaMemcpyHostToDevice));
  OF_CUDA_TRY(cudaMemcpy(t->hist_count, &h.hist_count, sizeof(h.hist_count), cudaMemcpyHostToDevice));
  OF_CUDA_TRY(cudaMemcpy(t->hist, hist.data(), hist.size() * sizeof(double), cudaMemcpyHostToDevice));
  if (h.frames > 0)
    OF_CUDA_TRY(cudaMemcpy(t->depth[(h.frames - 1) & 1], depth.data(), px * sizeof(uint16_t),
                           cudaMemcpyHostToDevice));
  OF_CUDA_TRY(cudaMemcpy(t->volume, vol.data(), vol_bytes, cudaMemcpyHostToDevice));
  t->frames = h.frames;
  t->last_fused = h.last_fused != 0;
  return OF_OK;
}

