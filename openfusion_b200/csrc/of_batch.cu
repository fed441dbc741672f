// of_batch.cu -- many independent depth streams (each its own camera, volume
// and trajectory) tracked and fused together: one launch per stage for all
// streams, one CUDA graph per step.
//
// A step has the tracker's order (of_tracker.cu; the reference's
// RunApp::display, Source/src/MainApp.cpp:786-964): every stream's previous
// frame is fused and its model raycast (batched integrate, then batched
// raycast) while every stream's new frame is pre-processed (batched filter,
// pyramid and vertex/normal maps) on a graph branch; then one persistent
// cluster launch tracks every stream (of_icp.cu). Per stream the filter,
// pyramid, maps, integration and raycast write exactly what the
// single-stream stages write; the batched ICP sums in another order.
//
// Tuning: the knobs (raycast block shape, integration blocks per stream, ICP
// clusters) change no result, so they are chosen online: the first steps run
// eagerly, each with one candidate of one knob, timed with CUDA events
// (coordinate descent, two steps per candidate, the faster of the two kept), and
// the step graphs are captured with the winners.
#include "of_batch.cuh"

#include <new>
#include <string.h>
#include <vector>

using namespace of;

bool of_camera_valid(const of_camera_t *c);
bool of_volume_valid(const of_volume_desc_t *d);

namespace {

constexpr int kTuneReps = 2;

struct Knob {
  int *value;
  std::vector<int> candidates;
  int ev0;  // its stage runs between events ev_t[ev0] and ev_t[ev0 + 1]
};

}  // namespace

struct of_batch {
  of_batch_desc_t desc;
  std::vector<of_batch_stream_t> streams;
  std::vector<BatchStream> bs;
  void *arena = nullptr;
  PreprocessBatch *pre = nullptr;
  IntegrateBatch *integ = nullptr;
  RaycastBatch *ray = nullptr;
  IcpBatch *icp = nullptr;
  cudaStream_t cap = nullptr, side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_pre = nullptr;
  // stage timing while tuning: before/after integrate, after raycast, after
  // the join, after ICP
  cudaEvent_t ev_t[5] = {};
  BatchKnobs knobs{};
  bool tuned = false;
  // online tuning state
  std::vector<Knob> plan;
  int tune_knob = 0, tune_cand = 0, tune_rep = 0;
  std::vector<float> tune_ms;
  std::vector<float> best_ms;
  int64_t frames = 0;
  bool last_fused = false;
  int kernels_step = 0;
  cudaGraphExec_t g_step[2] = {nullptr, nullptr};
};

namespace {

void release(of_batch *b) {
  for (cudaGraphExec_t g : b->g_step)
    if (g) cudaGraphExecDestroy(g);
  preprocess_batch_destroy(b->pre);
  integrate_batch_destroy(b->integ);
  raycast_batch_destroy(b->ray);
  icp_batch_destroy(b->icp);
  if (b->arena) cudaFree(b->arena);
  for (cudaStream_t q : {b->cap, b->side})
    if (q) cudaStreamDestroy(q);
  for (cudaEvent_t e : {b->ev_fork, b->ev_pre, b->ev_t[0], b->ev_t[1], b->ev_t[2], b->ev_t[3],
                        b->ev_t[4]})
    if (e) cudaEventDestroy(e);
  delete b;
}

// fuse every stream's frame in depth[parity] at its pose, raycast the models
of_status_t enqueue_fuse(of_batch *b, int parity, cudaStream_t s, bool timed) {
  if (timed) OF_CUDA_TRY(cudaEventRecord(b->ev_t[0], s));
  of_status_t st = integrate_batch_launch(b->integ, parity, b->knobs, s);
  if (st != OF_OK) return st;
  if (timed) OF_CUDA_TRY(cudaEventRecord(b->ev_t[1], s));
  st = raycast_batch_launch(b->ray, b->knobs, s);
  if (st != OF_OK) return st;
  if (timed) OF_CUDA_TRY(cudaEventRecord(b->ev_t[2], s));
  return OF_OK;
}

// step of frames k >= 1 (depth[cur]): fuse k-1 and raycast beside
// pre-processing k, then ICP k
of_status_t enqueue_step(of_batch *b, int cur, bool fuse, cudaStream_t s, bool timed) {
  OF_CUDA_TRY(cudaEventRecord(b->ev_fork, s));
  OF_CUDA_TRY(cudaStreamWaitEvent(b->side, b->ev_fork, 0));
  of_status_t sp = preprocess_batch_launch(b->pre, cur, b->side);
  OF_CUDA_TRY(cudaEventRecord(b->ev_pre, b->side));
  of_status_t sf = fuse ? enqueue_fuse(b, cur ^ 1, s, timed) : OF_OK;
  OF_CUDA_TRY(cudaStreamWaitEvent(s, b->ev_pre, 0));
  if (sp != OF_OK) return sp;
  if (sf != OF_OK) return sf;
  if (timed) OF_CUDA_TRY(cudaEventRecord(b->ev_t[3], s));
  of_status_t st = icp_batch_launch(b->icp, b->knobs, s);
  if (st != OF_OK) return st;
  if (timed) OF_CUDA_TRY(cudaEventRecord(b->ev_t[4], s));
  return OF_OK;
}

int count_kernels(cudaGraph_t g) {
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return 0;
  std::vector<cudaGraphNode_t> nodes(n);
  int k = 0;
  if (cudaGraphGetNodes(g, nodes.data(), &n) == cudaSuccess)
    for (size_t i = 0; i < n; ++i) {
      cudaGraphNodeType ty;
      if (cudaGraphNodeGetType(nodes[i], &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++k;
    }
  return k;
}

of_status_t capture(of_batch *b, int cur, cudaGraphExec_t *out) {
  cudaGraph_t g = nullptr;
  OF_CUDA_TRY(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
  of_status_t st = enqueue_step(b, cur, true, b->cap, false);
  cudaError_t e = cudaStreamEndCapture(b->cap, &g);
  if (st != OF_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) return of_set_cuda_error(e);
  b->kernels_step = count_kernels(g);
  e = cudaGraphInstantiateWithFlags(out, g, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return of_set_cuda_error(e);
  return OF_OK;
}

of_status_t capture_graphs(of_batch *b) {
  for (int c = 0; c < 2; ++c) {
    if (b->g_step[c]) {
      cudaGraphExecDestroy(b->g_step[c]);
      b->g_step[c] = nullptr;
    }
    of_status_t st = capture(b, c, &b->g_step[c]);
    if (st != OF_OK) return st;
  }
  return OF_OK;
}

// After a timed step: record the tuned stage's time for the current candidate
// and move to the next candidate / knob; captures the graphs when done.
of_status_t tune_advance(of_batch *b) {
  OF_CUDA_TRY(cudaEventSynchronize(b->ev_t[4]));
  Knob &K = b->plan[b->tune_knob];
  float ms = 0.f;
  OF_CUDA_TRY(cudaEventElapsedTime(&ms, b->ev_t[K.ev0], b->ev_t[K.ev0 + 1]));
  b->tune_ms.push_back(ms);
  if (++b->tune_rep < kTuneReps) return OF_OK;
  // the candidate's time: the smaller of its repetitions
  float m = b->tune_ms[0];
  for (float x : b->tune_ms) m = x < m ? x : m;
  b->tune_ms.clear();
  b->tune_rep = 0;
  b->best_ms.push_back(m);
  if (++b->tune_cand < (int)K.candidates.size()) {
    *K.value = K.candidates[b->tune_cand];
    return OF_OK;
  }
  int best = 0;
  for (int i = 1; i < (int)b->best_ms.size(); ++i)
    if (b->best_ms[i] < b->best_ms[best]) best = i;
  *K.value = K.candidates[best];
  b->best_ms.clear();
  b->tune_cand = 0;
  if (++b->tune_knob < (int)b->plan.size()) {
    Knob &N = b->plan[b->tune_knob];
    *N.value = N.candidates[0];
    return OF_OK;
  }
  b->tuned = true;
  return b->desc.use_graph ? capture_graphs(b) : OF_OK;
}

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" of_status_t of_batch_create(const of_batch_desc_t *desc, of_batch_t *out) {
  if (!desc || !out || desc->count < 1 || !desc->streams) return OF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  const int n = desc->count;
  if (desc->filter.levels != desc->icp.levels || desc->icp.levels < 1 ||
      desc->icp.levels > kMaxLevels)
    return OF_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < n; ++i)
    if (!of_camera_valid(&desc->streams[i].camera) || !of_volume_valid(&desc->streams[i].volume) ||
        desc->streams[i].volume.storage != desc->streams[0].volume.storage)
      return OF_ERR_INVALID_ARGUMENT;
  of_batch *b = new (std::nothrow) of_batch();
  if (!b) return OF_ERR_OUT_OF_MEMORY;
  b->desc = *desc;
  b->streams.assign(desc->streams, desc->streams + n);
  b->desc.streams = b->streams.data();
  // the critical path above the pre-processing branch (as in a tracker step;
  // the graphs keep the priorities as node priorities)
  int least = 0, greatest = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  if (e == cudaSuccess)
    e = cudaStreamCreateWithPriority(&b->cap, cudaStreamNonBlocking, (least + greatest) / 2);
  if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&b->side, cudaStreamNonBlocking, least);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_pre, cudaEventDisableTiming);
  for (int i = 0; i < 5 && e == cudaSuccess; ++i) e = cudaEventCreate(&b->ev_t[i]);
  if (e != cudaSuccess) { release(b); return of_set_cuda_error(e); }
  // one arena: per stream volume, lambda table, integration scratch, frame
  // and model pyramids, two depth buffers, pose, ICP statistics
  struct Off { size_t vol, lam, scratch, frame, model, depth0, depth1, pose, stats; };
  std::vector<Off> off(n);
  size_t total = 0;
  for (int i = 0; i < n; ++i) {
    const of_batch_stream_t &S = b->streams[i];
    size_t vb = 0, lb = 0, sb = 0;
    of_volume_bytes(&S.volume, &vb);
    of_lambda_bytes(&S.camera, &lb);
    of_integrate_scratch_bytes(&S.volume, &S.camera, &sb);
    of_pyramid_layout_t lay;
    of_status_t st = of_pyramid_layout(&S.camera, desc->icp.levels, &lay);
    if (st != OF_OK) { release(b); return st; }
    const size_t px = (size_t)S.camera.width * S.camera.height * sizeof(uint16_t);
    Off &o = off[i];
    o.vol = total; total = a256(total + vb);
    o.lam = total; total = a256(total + lb);
    o.scratch = total; total = a256(total + sb);
    o.frame = total; total = a256(total + lay.total_bytes);
    o.model = total; total = a256(total + lay.total_bytes);
    o.depth0 = total; total = a256(total + px);
    o.depth1 = total; total = a256(total + px);
    o.pose = total; total = a256(total + 16 * sizeof(double));
    o.stats = total; total = a256(total + sizeof(of_icp_stats_t));
  }
  e = cudaMalloc(&b->arena, total);
  if (e != cudaSuccess) {
    cudaGetLastError();
    release(b);
    return e == cudaErrorMemoryAllocation ? OF_ERR_OUT_OF_MEMORY : of_set_cuda_error(e);
  }
  char *base = (char *)b->arena;
  b->bs.resize(n);
  cudaStream_t s = b->cap;
  of_status_t st = OF_OK;
  for (int i = 0; i < n && st == OF_OK; ++i) {
    const of_batch_stream_t &S = b->streams[i];
    BatchStream &B = b->bs[i];
    B.cam = S.camera;
    B.vol_desc = S.volume;
    B.volume = base + off[i].vol;
    B.lambda = (const float *)(base + off[i].lam);
    B.scratch = base + off[i].scratch;
    B.frame = base + off[i].frame;
    B.model = base + off[i].model;
    B.depth[0] = (const uint16_t *)(base + off[i].depth0);
    B.depth[1] = (const uint16_t *)(base + off[i].depth1);
    B.pose = (double *)(base + off[i].pose);
    B.stats = (of_icp_stats_t *)(base + off[i].stats);
    st = of_volume_reset(&S.volume, B.volume, s);
    if (st == OF_OK) st = of_lambda_table(&S.camera, (float *)B.lambda, s);
    of_pyramid_layout_t lay;
    if (st == OF_OK) st = of_pyramid_layout(&S.camera, desc->icp.levels, &lay);
    if (st == OF_OK &&
        (cudaMemsetAsync(B.frame, 0, lay.total_bytes, s) != cudaSuccess ||
         cudaMemsetAsync(B.model, 0, lay.total_bytes, s) != cudaSuccess ||
         cudaMemsetAsync(B.stats, 0, sizeof(of_icp_stats_t), s) != cudaSuccess ||
         cudaMemcpyAsync(B.pose, S.initial_pose, 16 * sizeof(double), cudaMemcpyHostToDevice, s) !=
             cudaSuccess))
      st = of_set_cuda_error(cudaGetLastError());
  }
  BatchParams P;
  P.filter = desc->filter;
  P.raycast = desc->raycast;
  P.icp = desc->icp;
  if (st == OF_OK) st = preprocess_batch_create(b->bs.data(), n, P, &b->pre);
  if (st == OF_OK) st = integrate_batch_create(b->bs.data(), n, &b->integ);
  if (st == OF_OK) st = raycast_batch_create(b->bs.data(), n, P, &b->ray);
  if (st == OF_OK) st = icp_batch_create(b->bs.data(), n, P, &b->icp);
  if (st == OF_OK && cudaStreamSynchronize(s) != cudaSuccess) st = of_set_cuda_error(cudaGetLastError());
  if (st != OF_OK) { release(b); return st; }
  // knobs: given, or tuned online over the first steps
  const int maxc = icp_batch_max_clusters();
  b->knobs.ray_tile = desc->tuning.ray_tile;
  b->knobs.list_div = desc->tuning.list_div;
  b->knobs.icp_clusters = desc->tuning.icp_clusters;
  if (desc->tune) {
    b->plan.push_back({&b->knobs.list_div, {0, 1, 2, 3, 4}, 0});
    b->plan.push_back({&b->knobs.ray_tile, {0, 1, 2, 3, 4, 5, 6}, 1});
    std::vector<int> cl;
    for (int c : {maxc / 4, maxc / 2, maxc})
      if (c >= 1 && (cl.empty() || cl.back() != c)) cl.push_back(c);
    b->plan.push_back({&b->knobs.icp_clusters, cl, 3});
    *b->plan[0].value = b->plan[0].candidates[0];
  } else {
    b->tuned = true;
    if (desc->use_graph) st = capture_graphs(b);
    if (st != OF_OK) { release(b); return st; }
  }
  *out = b;
  return OF_OK;
}

extern "C" of_status_t of_batch_destroy(of_batch_t b) {
  if (!b) return OF_ERR_INVALID_ARGUMENT;
  cudaDeviceSynchronize();
  release(b);
  return OF_OK;
}

extern "C" of_status_t of_batch_process(of_batch_t b, const uint16_t *const *depth,
                                        int32_t depth_is_host, of_stream_t stream) {
  OF_RANGE("of_batch_process");
  if (!b || !depth) return OF_ERR_INVALID_ARGUMENT;
  const int n = b->desc.count;
  for (int i = 0; i < n; ++i)
    if (!depth[i]) return OF_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  const int cur = (int)(b->frames & 1);
  for (int i = 0; i < n; ++i) {
    const size_t bytes = (size_t)b->bs[i].cam.width * b->bs[i].cam.height * sizeof(uint16_t);
    uint16_t *dst = (uint16_t *)b->bs[i].depth[cur];
    if (depth[i] != dst)
      OF_CUDA_TRY(cudaMemcpyAsync(dst, depth[i], bytes,
                                  depth_is_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
  }
  if (b->frames > 0) {
    const bool fuse = !b->last_fused;
    if (b->tuned && b->desc.use_graph && fuse) {
      OF_CUDA_TRY(cudaGraphLaunch(b->g_step[cur], s));
    } else {
      // tuning steps need the ICP time too, so they run with every stage
      const bool timing = !b->tuned && fuse;
      of_status_t st = enqueue_step(b, cur, fuse, s, timing);
      if (st != OF_OK) return st;
      if (timing) {
        st = tune_advance(b);
        if (st != OF_OK) return st;
      }
    }
  }
  b->last_fused = false;
  b->frames += 1;
  return OF_OK;
}

extern "C" of_status_t of_batch_flush(of_batch_t b, of_stream_t stream) {
  if (!b) return OF_ERR_INVALID_ARGUMENT;
  if (b->frames == 0 || b->last_fused) return OF_OK;
  of_status_t st = enqueue_fuse(b, (int)((b->frames - 1) & 1), (cudaStream_t)stream, false);
  if (st != OF_OK) return st;
  b->last_fused = true;
  return OF_OK;
}

extern "C" of_status_t of_batch_poses(of_batch_t b, double *poses, of_icp_stats_t *stats,
                                      of_stream_t stream) {
  if (!b || !poses) return OF_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  for (int i = 0; i < b->desc.count; ++i) {
    OF_CUDA_TRY(cudaMemcpyAsync(poses + 16 * (size_t)i, b->bs[i].pose, 16 * sizeof(double),
                                cudaMemcpyDeviceToHost, s));
    if (stats)
      OF_CUDA_TRY(cudaMemcpyAsync(stats + i, b->bs[i].stats, sizeof(of_icp_stats_t),
                                  cudaMemcpyDeviceToHost, s));
  }
  return OF_OK;
}

extern "C" of_status_t of_batch_tuning(of_batch_t b, of_batch_tuning_t *out) {
  if (!b || !out) return OF_ERR_INVALID_ARGUMENT;
  out->ray_tile = b->knobs.ray_tile;
  out->list_div = b->knobs.list_div;
  out->icp_clusters = b->knobs.icp_clusters;
  out->tuned = b->tuned && b->desc.tune ? 1 : 0;
  return OF_OK;
}

extern "C" of_status_t of_batch_stream_buffers(of_batch_t b, int32_t i, of_tracker_buffers_t *out) {
  if (!b || !out || i < 0 || i >= b->desc.count) return OF_ERR_INVALID_ARGUMENT;
  const BatchStream &B = b->bs[i];
  out->volume = B.volume;
  out->frame = B.frame;
  out->model = B.model;
  out->pose = B.pose;
  out->depth = (uint16_t *)B.depth[b->frames > 0 ? (b->frames - 1) & 1 : 0];
  out->lambda = (float *)B.lambda;
  out->stats = B.stats;
  out->frames = b->frames;
  out->kernels_first = 0;
  out->kernels_track = b->kernels_step;
  return OF_OK;
}

// Host-side planning (no device work) ----------------------------------------

extern "C" of_status_t of_batch_stream_cost(const of_batch_stream_t *s, const of_icp_params_t *icp,
                                            double *cost) {
  if (!s || !icp || !cost || icp->levels < 1 || icp->levels > kMaxLevels)
    return OF_ERR_INVALID_ARGUMENT;
  // per frame: the voxels integration may visit plus every ICP iteration's
  // pixels of its level, plus the raycast's pixels (units of one voxel visit)
  const double n = (double)s->volume.resolution;
  double c = n * n * n / 8.0;
  for (int l = 0; l < icp->levels; ++l) {
    const of_camera_t cl = camera_level(s->camera, l);
    c += (double)cl.width * cl.height * (icp->iters[l] + (l == 0 ? 8.0 : 0.0));
  }
  *cost = c;
  return OF_OK;
}

extern "C" of_status_t of_batch_shard(const double *cost, int32_t count, int32_t ranks,
                                      int32_t *rank_of_stream) {
  if (!cost || !rank_of_stream || count < 0 || ranks < 1) return OF_ERR_INVALID_ARGUMENT;
  // longest processing time first: each stream, heaviest first (ties by
  // index), goes to the least loaded rank (ties by rank)
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  for (int i = 1; i < count; ++i)
    for (int k = i; k > 0 && (cost[order[k]] > cost[order[k - 1]] ||
                              (cost[order[k]] == cost[order[k - 1]] && order[k] < order[k - 1]));
         --k) {
      const int t = order[k]; order[k] = order[k - 1]; order[k - 1] = t;
    }
  std::vector<double> load(ranks, 0.0);
  for (int i : order) {
    int r = 0;
    for (int q = 1; q < ranks; ++q)
      if (load[q] < load[r]) r = q;
    rank_of_stream[i] = r;
    load[r] += cost[i];
  }
  return OF_OK;
}
