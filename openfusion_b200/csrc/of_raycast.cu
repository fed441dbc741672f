// of_raycast.cu -- surface prediction by ray marching the TSDF: the
// single-stream launch (of_raycast), the batched one and the model pyramid.
// The per-ray method (the reference's d_raycast, Source/src/Raycaster.cu:97-230,
// with the KinectFusion refinement it left commented out) is in of_raycast.cuh.
#include "of_raycast.cuh"

bool of_camera_valid(const of_camera_t *c);
bool of_volume_valid(const of_volume_desc_t *d);

namespace {

template <int STORAGE>
__global__ void __launch_bounds__(256) k_raycast(const uint32_t *__restrict__ vol,
                                                 of_volume_desc_t desc, Cam cam,
                                                 of_raycast_params_t rp,
                                                 const double *__restrict__ pose,
                                                 float4 *__restrict__ pts, uint32_t *rgba,
                                                 ModelLevels coarse) {
  raycast_tile<STORAGE>(vol, desc, cam, rp, pose, pts, rgba, blockIdx.x, blockIdx.y, &coarse);
}

// Model level l -> l+1 by subsampling pixel (2x, 2y): model points are used
// by ICP only through their world positions, so the subset fixes nothing
// about the model pixels' intrinsics.
__global__ void k_model_down(const float4 *__restrict__ src, int sw, float4 *__restrict__ dst,
                             int dw, int dh) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= dw || y >= dh) return;
  size_t sp = (size_t)(2 * y) * sw + 2 * x;
  size_t dp = (size_t)y * dw + x;
  dst[2 * dp] = src[2 * sp];
  dst[2 * dp + 1] = src[2 * sp + 1];
}

// ---------------------------------------------------------------- batched --
struct RayJob {
  const uint32_t *vol;
  of_volume_desc_t desc;
  Cam cam;
  const double *pose;
  float4 *pts;
};
// level l >= 1 of a model pyramid from level 0: pixel (2^l x, 2^l y), the
// value k_model_down's chain of subsamplings gives
struct DownJob {
  const float4 *src;
  float4 *dst;
  int sw, dw, dh, step, gx;
};

// block shapes of the raycast (a tuning knob; every ray is the same)
constexpr int kRayTiles = 7;
constexpr int kRayTileX[kRayTiles] = {16, 32, 8, 32, 16, 8, 8};
constexpr int kRayTileY[kRayTiles] = {16, 8, 32, 4, 8, 16, 8};

template <int STORAGE>
__global__ void __launch_bounds__(256) k_raycast_batch(const RayJob *__restrict__ jobs,
                                                       const int *__restrict__ first, int n,
                                                       of_raycast_params_t rp) {
  const int j = batch_job(first, n, blockIdx.x);
  const RayJob &J = jobs[j];
  const int b = blockIdx.x - __ldg(first + j);
  const int gx = (J.cam.w + (int)blockDim.x - 1) / (int)blockDim.x;
  raycast_tile<STORAGE>(J.vol, J.desc, J.cam, rp, J.pose, J.pts, nullptr, b % gx, b / gx);
}

__global__ void k_model_down_batch(const DownJob *__restrict__ jobs, const int *__restrict__ first,
                                   int n) {
  const int j = batch_job(first, n, blockIdx.x);
  const DownJob &J = jobs[j];
  const int b = blockIdx.x - __ldg(first + j);
  const int x = (b % J.gx) * blockDim.x + threadIdx.x;
  const int y = (b / J.gx) * blockDim.y + threadIdx.y;
  if (x >= J.dw || y >= J.dh) return;
  const size_t sp = (size_t)(J.step * y) * J.sw + (size_t)J.step * x;
  const size_t dp = (size_t)y * J.dw + x;
  J.dst[2 * dp] = J.src[2 * sp];
  J.dst[2 * dp + 1] = J.src[2 * sp + 1];
}

}  // namespace

namespace of {

struct RaycastBatch {
  int n = 0, storage = OF_TSDF_I16;
  of_raycast_params_t rp{};
  RayJob *jobs = nullptr;
  int *first[kRayTiles] = {}, blocks[kRayTiles] = {};
  DownJob *down = nullptr;
  int *down_first = nullptr, down_jobs = 0, down_blocks = 0;
};

void raycast_batch_destroy(RaycastBatch *b) {
  if (!b) return;
  cudaFree(b->jobs);
  for (int t = 0; t < kRayTiles; ++t) cudaFree(b->first[t]);
  cudaFree(b->down);
  cudaFree(b->down_first);
  delete b;
}

of_status_t raycast_batch_create(const BatchStream *s, int n, const BatchParams &p,
                                 RaycastBatch **out) {
  const of_raycast_params_t &rp = p.raycast;
  const int levels = p.icp.levels;
  if (n < 1 || levels < 1 || levels > kMaxLevels || rp.min_step_vox <= 0.f ||
      rp.far_step_frac < 0.f || rp.refine_iters < 0 || rp.refine_iters > 16)
    return OF_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < n; ++i)
    if (s[i].vol_desc.storage != s[0].vol_desc.storage) return OF_ERR_INVALID_ARGUMENT;
  RaycastBatch *b = new RaycastBatch();
  b->n = n;
  b->storage = s[0].vol_desc.storage;
  b->rp = rp;
  RayJob *jobs = new RayJob[n];
  DownJob *down = new DownJob[(size_t)n * kMaxLevels];
  int *first = new int[(size_t)n * kMaxLevels + 1];
  of_status_t st = OF_OK;
  for (int i = 0; i < n && st == OF_OK; ++i) {
    of_pyramid_layout_t lay;
    st = of_pyramid_layout(&s[i].cam, levels, &lay);
    jobs[i] = {(const uint32_t *)s[i].volume, s[i].vol_desc, make_cam(s[i].cam), s[i].pose,
               (float4 *)((char *)s[i].model + lay.points_offset[0])};
  }
  for (int t = 0; t < kRayTiles && st == OF_OK; ++t) {
    first[0] = 0;
    for (int i = 0; i < n; ++i)
      first[i + 1] = first[i] + ((s[i].cam.width + kRayTileX[t] - 1) / kRayTileX[t]) *
                                    ((s[i].cam.height + kRayTileY[t] - 1) / kRayTileY[t]);
    b->blocks[t] = first[n];
    RayJob *tmp = nullptr;
    st = upload_jobs(jobs, first, n, t == 0 ? &b->jobs : &tmp, &b->first[t]);
    if (tmp) cudaFree(tmp);
  }
  if (st == OF_OK) {
    int k = 0;
    first[0] = 0;
    for (int i = 0; i < n; ++i) {
      of_pyramid_layout_t lay;
      of_pyramid_layout(&s[i].cam, levels, &lay);
      char *base = (char *)s[i].model;
      for (int l = 1; l < levels; ++l, ++k) {
        down[k] = {(const float4 *)(base + lay.points_offset[0]), (float4 *)(base + lay.points_offset[l]),
                   lay.width[0], lay.width[l], lay.height[l], 1 << l, (lay.width[l] + 31) / 32};
        first[k + 1] = first[k] + down[k].gx * ((lay.height[l] + 7) / 8);
      }
    }
    b->down_jobs = k;
    b->down_blocks = first[k];
    if (k > 0) st = upload_jobs(down, first, k, &b->down, &b->down_first);
  }
  delete[] jobs;
  delete[] down;
  delete[] first;
  if (st != OF_OK) {
    raycast_batch_destroy(b);
    return st;
  }
  *out = b;
  return OF_OK;
}

of_status_t raycast_batch_launch(const RaycastBatch *b, const BatchKnobs &k, cudaStream_t s) {
  const int t = k.ray_tile < 0 ? 0 : k.ray_tile % kRayTiles;
  const dim3 blk(kRayTileX[t], kRayTileY[t]);
  if (b->storage == OF_TSDF_I16)
    k_raycast_batch<OF_TSDF_I16><<<b->blocks[t], blk, 0, s>>>(b->jobs, b->first[t], b->n, b->rp);
  else
    k_raycast_batch<OF_TSDF_F16><<<b->blocks[t], blk, 0, s>>>(b->jobs, b->first[t], b->n, b->rp);
  if (b->down_jobs > 0)
    k_model_down_batch<<<b->down_blocks, dim3(32, 8), 0, s>>>(b->down, b->down_first, b->down_jobs);
  return of_launch_status();
}

}  // namespace of

of_status_t of_model_pyramid(const of_camera_t *cam, int levels, void *d_model, cudaStream_t s) {
  of_pyramid_layout_t lay;
  of_status_t st = of_pyramid_layout(cam, levels, &lay);
  if (st != OF_OK) return st;
  char *base = (char *)d_model;
  for (int l = 1; l < levels; ++l) {
    dim3 blk(32, 8);
    dim3 grid((lay.width[l] + 31) / 32, (lay.height[l] + 7) / 8);
    k_model_down<<<grid, blk, 0, s>>>((const float4 *)(base + lay.points_offset[l - 1]),
                                      lay.width[l - 1], (float4 *)(base + lay.points_offset[l]),
                                      lay.width[l], lay.height[l]);
  }
  return of_launch_status();
}

extern "C" of_status_t of_raycast(const of_volume_desc_t *d, const void *vol,
                                  const of_camera_t *cam, const of_raycast_params_t *rp,
                                  int32_t levels, const double *pose, void *d_model,
                                  uint32_t *rgba, of_stream_t stream) {
  OF_RANGE("of_raycast");
  if (!of_volume_valid(d) || !of_camera_valid(cam) || !rp || !vol || !pose || !d_model)
    return OF_ERR_INVALID_ARGUMENT;
  if (levels < 1 || levels > kMaxLevels || rp->min_step_vox <= 0.f || rp->far_step_frac < 0.f ||
      rp->refine_iters < 0 || rp->refine_iters > 16 || rp->tile < 0 || rp->tile >= kRayTiles)
    return OF_ERR_INVALID_ARGUMENT;
  of_pyramid_layout_t lay;
  of_status_t st = of_pyramid_layout(cam, levels, &lay);
  if (st != OF_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const int tx = kRayTileX[rp->tile], ty = kRayTileY[rp->tile];
  dim3 blk(tx, ty);
  dim3 grid((cam->width + tx - 1) / tx, (cam->height + ty - 1) / ty);
  Cam c = make_cam(*cam);
  float4 *pts = (float4 *)((char *)d_model + lay.points_offset[0]);
  ModelLevels coarse;
  memset(&coarse, 0, sizeof(coarse));
  coarse.levels = levels;
  for (int l = 0; l < levels; ++l) {
    coarse.pts[l] = (float4 *)((char *)d_model + lay.points_offset[l]);
    coarse.w[l] = lay.width[l];
  }
  if (d->storage == OF_TSDF_I16)
    k_raycast<OF_TSDF_I16><<<grid, blk, 0, s>>>((const uint32_t *)vol, *d, c, *rp, pose, pts, rgba,
                                                coarse);
  else
    k_raycast<OF_TSDF_F16><<<grid, blk, 0, s>>>((const uint32_t *)vol, *d, c, *rp, pose, pts, rgba,
                                                coarse);
  return of_launch_status();
}
