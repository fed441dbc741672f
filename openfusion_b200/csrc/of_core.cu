// of_core.cu -- status codes, parameter defaults, layouts and volume
// maintenance (reset / export / import), the per-pixel ray-length table and
// the pose adapters of the C-ABI.
#include "of_common.cuh"

#include <string.h>

using namespace of;

static thread_local cudaError_t g_last_cuda_error = cudaSuccess;

of_status_t of_set_cuda_error(cudaError_t e) {
  g_last_cuda_error = e;
  return OF_ERR_CUDA;
}

of_status_t of_launch_status() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return of_set_cuda_error(e);
  return OF_OK;
}

extern "C" int32_t of_abi_version(void) { return OF_ABI_VERSION; }

extern "C" const char *of_status_string(of_status_t s) {
  switch (s) {
    case OF_OK: return "ok";
    case OF_ERR_INVALID_ARGUMENT: return "invalid argument";
    case OF_ERR_CUDA: return cudaGetErrorString(g_last_cuda_error);
    case OF_ERR_OUT_OF_MEMORY: return "out of device memory";
    case OF_ERR_NOT_READY: return "not ready";
    case OF_ERR_TOO_LARGE: return "size beyond the entry point's fixed maximum";
    case OF_ERR_IO: return "file could not be opened, read or written";
    case OF_END_OF_SEQUENCE: return "end of the recorded sequence";
    default: return "unknown status";
  }
}

extern "C" void of_default_params(of_filter_params_t *f, of_raycast_params_t *r,
                                  of_icp_params_t *i) {
  if (f) {
    f->sigma_space_px = 4.5f;
    f->sigma_range_mm = 30.0f;
    f->radius_px = 0;
    f->levels = 3;
  }
  if (r) {
    r->min_step_vox = 0.75f;
    r->far_step_frac = 0.8f;
    r->refine_iters = 3;
    r->tile = 0;
  }
  if (i) {
    i->levels = 3;
    i->iters[0] = 10; i->iters[1] = 5; i->iters[2] = 4; i->iters[3] = 0;
    i->dist_thresh_mm = 25.0f;
    i->normal_thresh = 0.65f;
    i->stop_rot_rad = 0.0f;
    i->stop_trans_mm = 0.0f;
    i->judge_max_rms_mm = 10.0f;
    i->judge_min_inlier_frac = 0.3f;
    i->judge_max_rot_rad = 0.05f;
    i->judge_max_trans_mm = 50.0f;
    i->warm_levels = 0;
  }
}

static bool camera_ok(const of_camera_t *c) {
  return c && c->width >= 8 && c->height >= 8 && c->width <= 8192 && c->height <= 8192 &&
         c->fx > 0.f && c->fy > 0.f && c->min_depth_mm >= 0.f &&
         c->max_depth_mm > c->min_depth_mm;
}

bool of_camera_valid(const of_camera_t *c) { return camera_ok(c); }

bool of_volume_valid(const of_volume_desc_t *d) {
  return d && d->resolution >= 8 && d->resolution <= 1024 && (d->resolution % 8) == 0 &&
         (d->storage == OF_TSDF_I16 || d->storage == OF_TSDF_F16) && d->size_mm > 0.f &&
         d->trunc_mm > 0.f && d->max_weight >= 1 && d->max_weight <= 65535;
}

extern "C" of_status_t of_camera_level(const of_camera_t *cam, int32_t level, of_camera_t *out) {
  if (!camera_ok(cam) || !out || level < 0 || level >= kMaxLevels) return OF_ERR_INVALID_ARGUMENT;
  *out = camera_level(*cam, level);
  return OF_OK;
}

extern "C" of_status_t of_pyramid_layout(const of_camera_t *cam, int32_t levels,
                                         of_pyramid_layout_t *out) {
  if (!camera_ok(cam) || !out || levels < 1 || levels > kMaxLevels) return OF_ERR_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  out->levels = levels;
  size_t off = 0;
  for (int l = 0; l < levels; ++l) {
    of_camera_t c = camera_level(*cam, l);
    out->width[l] = c.width;
    out->height[l] = c.height;
    size_t px = (size_t)c.width * c.height;
    out->depth_offset[l] = off;
    off = align256(off + px * sizeof(float));
    out->points_offset[l] = off;
    off = align256(off + px * 2 * sizeof(float4));
  }
  out->total_bytes = off;
  return OF_OK;
}

// ------------------------------------------------------------------ volume --

extern "C" of_status_t of_volume_bytes(const of_volume_desc_t *d, size_t *bytes) {
  if (!of_volume_valid(d) || !bytes) return OF_ERR_INVALID_ARGUMENT;
  size_t n = (size_t)d->resolution;
  size_t nb = n / kBrick, ns = (size_t)super_count((int)n);
  // voxel words, brick flags, super-brick flags, saturated-brick bytes
  *bytes = n * n * n * sizeof(uint32_t) + align256(nb * nb * nb) + align256(ns * ns * ns) +
           align256(nb * nb * nb);
  return OF_OK;
}

// Every voxel word := value (the +1 bit pattern with weight 0).
__global__ void k_volume_fill(uint4 *__restrict__ words, size_t n4, uint32_t value) {
  const uint4 v = make_uint4(value, value, value, value);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4;
       i += (size_t)gridDim.x * blockDim.x)
    words[i] = v;
}

extern "C" of_status_t of_volume_reset(const of_volume_desc_t *d, void *vol, of_stream_t s) {
  size_t bytes;
  if (of_volume_bytes(d, &bytes) != OF_OK || !vol) return OF_ERR_INVALID_ARGUMENT;
  // weight 0 everywhere: every voxel reads as +trunc (General.cu:27-50). The
  // stored tsdf of an unobserved voxel is the +1 pattern, so readers need no
  // weight test; every brick and super-brick flag cleared.
  const size_t n = (size_t)d->resolution, words = n * n * n;
  const uint32_t one = d->storage == OF_TSDF_I16 ? VoxelCodec<OF_TSDF_I16>::kOneBits
                                                 : VoxelCodec<OF_TSDF_F16>::kOneBits;
  k_volume_fill<<<kSmCount * 8, 256, 0, (cudaStream_t)s>>>((uint4 *)vol, words / 4, one);
  of_status_t st = of_launch_status();
  if (st != OF_OK) return st;
  OF_CUDA_TRY(cudaMemsetAsync(brick_flags(vol, (int)n), 0, bytes - words * sizeof(uint32_t),
                              (cudaStream_t)s));
  return OF_OK;
}

template <int STORAGE>
__global__ void k_volume_export(const uint32_t *__restrict__ vol, VolGeom g, float *tsdf,
                                uint16_t *weight) {
  size_t n = (size_t)g.n;
  size_t total = n * n * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    int k = (int)(idx % n);
    int j = (int)((idx / n) % n);
    int i = (int)(idx / (n * n));
    uint32_t w = vol[vox_index(g.nb, i, j, k)];
    if (tsdf) tsdf[idx] = vox_value<STORAGE>(w) * g.trunc;
    if (weight) weight[idx] = (uint16_t)(w >> 16);
  }
}

template <int STORAGE>
__global__ void k_volume_import(uint32_t *__restrict__ vol, VolGeom g, const float *tsdf,
                                const uint16_t *weight) {
  size_t n = (size_t)g.n;
  size_t total = n * n * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    int k = (int)(idx % n);
    int j = (int)((idx / n) % n);
    int i = (int)(idx / (n * n));
    uint32_t wt = weight ? weight[idx] : 1u;
    // an unobserved voxel keeps the +1 pattern (as after a reset)
    float t = (tsdf && wt) ? tsdf[idx] * g.inv_trunc : 1.0f;
    vol[vox_index(g.nb, i, j, k)] = VoxelCodec<STORAGE>::pack(t, wt);
  }
}

extern "C" of_status_t of_volume_export(const of_volume_desc_t *d, const void *vol, float *tsdf,
                                        uint16_t *weight, of_stream_t s) {
  if (!of_volume_valid(d) || !vol) return OF_ERR_INVALID_ARGUMENT;
  VolGeom g = make_geom(*d);
  int blocks = kSmCount * 8;
  if (d->storage == OF_TSDF_I16)
    k_volume_export<OF_TSDF_I16><<<blocks, 256, 0, (cudaStream_t)s>>>((const uint32_t *)vol, g,
                                                                     tsdf, weight);
  else
    k_volume_export<OF_TSDF_F16><<<blocks, 256, 0, (cudaStream_t)s>>>((const uint32_t *)vol, g,
                                                                     tsdf, weight);
  return of_launch_status();
}

extern "C" of_status_t of_volume_import(const of_volume_desc_t *d, void *vol, const float *tsdf,
                                        const uint16_t *weight, of_stream_t s) {
  if (!of_volume_valid(d) || !vol) return OF_ERR_INVALID_ARGUMENT;
  VolGeom g = make_geom(*d);
  int blocks = kSmCount * 8;
  if (d->storage == OF_TSDF_I16)
    k_volume_import<OF_TSDF_I16><<<blocks, 256, 0, (cudaStream_t)s>>>((uint32_t *)vol, g, tsdf,
                                                                     weight);
  else
    k_volume_import<OF_TSDF_F16><<<blocks, 256, 0, (cudaStream_t)s>>>((uint32_t *)vol, g, tsdf,
                                                                     weight);
  of_status_t st = of_launch_status();
  if (st != OF_OK) return st;
  // imported content is unknown: mark every brick (and super-brick) as near
  // a surface
  size_t n = (size_t)d->resolution, nb = n / kBrick, ns = (size_t)super_count((int)n);
  OF_CUDA_TRY(cudaMemsetAsync(brick_flags(vol, (int)n), 1, nb * nb * nb, (cudaStream_t)s));
  OF_CUDA_TRY(cudaMemsetAsync(super_flags(vol, (int)n), 1, ns * ns * ns, (cudaStream_t)s));
  OF_CUDA_TRY(cudaMemsetAsync(saturated_flags(vol, (int)n), 0, nb * nb * nb, (cudaStream_t)s));
  return OF_OK;
}

// ------------------------------------------------------- ray-length table --

__global__ void k_lambda_table(of_camera_t c, float2 *lam) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= c.width * c.height) return;
  int u = idx % c.width, v = idx / c.width;
  double a = ((double)u - (double)c.cx) / (double)c.fx;
  double b = ((double)v - (double)c.cy) / (double)c.fy;
  double l = sqrt(1.0 + a * a + b * b);
  float hi = (float)l;
  lam[idx] = make_float2(hi, (float)(l - (double)hi));
}

extern "C" of_status_t of_lambda_bytes(const of_camera_t *cam, size_t *bytes) {
  if (!camera_ok(cam) || !bytes) return OF_ERR_INVALID_ARGUMENT;
  *bytes = (size_t)cam->width * cam->height * sizeof(float2);
  return OF_OK;
}

extern "C" of_status_t of_lambda_table(const of_camera_t *cam, float *d_lambda, of_stream_t s) {
  if (!camera_ok(cam) || !d_lambda) return OF_ERR_INVALID_ARGUMENT;
  int n = cam->width * cam->height;
  k_lambda_table<<<(n + 255) / 256, 256, 0, (cudaStream_t)s>>>(*cam, (float2 *)d_lambda);
  return of_launch_status();
}

// ------------------------------------------------------------ pose adapters --

__global__ void k_pose_from_float(const float *pf, double *pd, int invert) {
  if (threadIdx.x != 0) return;
  double m[16];
  for (int i = 0; i < 16; ++i) m[i] = (double)pf[i];
  if (!invert) {
    for (int i = 0; i < 16; ++i) pd[i] = m[i];
    return;
  }
  for (int i = 0; i < 3; ++i) {
    double acc = 0.0;
    for (int j = 0; j < 3; ++j) {
      pd[4 * i + j] = m[4 * j + i];
      acc -= m[4 * j + i] * m[4 * j + 3];
    }
    pd[4 * i + 3] = acc;
  }
  pd[12] = pd[13] = pd[14] = 0.0;
  pd[15] = 1.0;
}

__global__ void k_pose_to_float(const double *pd, float *pf, float *inv, float *campos) {
  if (threadIdx.x != 0) return;
  if (pf)
    for (int i = 0; i < 16; ++i) pf[i] = (float)pd[i];
  if (inv) {
    // rigid inverse [R^T, -R^T t] (General.cpp:27-37 inverts with Eigen)
    for (int i = 0; i < 3; ++i) {
      double acc = 0.0;
      for (int j = 0; j < 3; ++j) {
        inv[4 * i + j] = (float)pd[4 * j + i];
        acc -= pd[4 * j + i] * pd[4 * j + 3];
      }
      inv[4 * i + 3] = (float)acc;
    }
    inv[12] = inv[13] = inv[14] = 0.f;
    inv[15] = 1.f;
  }
  if (campos) {
    // d_updateTransforms (General.cu:57-62)
    campos[0] = (float)pd[3];
    campos[1] = (float)pd[7];
    campos[2] = (float)pd[11];
  }
}

extern "C" of_status_t of_pose_from_float(const float *pf, double *pd, int32_t invert,
                                          of_stream_t s) {
  if (!pf || !pd) return OF_ERR_INVALID_ARGUMENT;
  k_pose_from_float<<<1, 32, 0, (cudaStream_t)s>>>(pf, pd, invert);
  return of_launch_status();
}

extern "C" of_status_t of_pose_to_float(const double *pd, float *pf, float *inv, float *campos,
                                        of_stream_t s) {
  if (!pd) return OF_ERR_INVALID_ARGUMENT;
  k_pose_to_float<<<1, 32, 0, (cudaStream_t)s>>>(pd, pf, inv, campos);
  return of_launch_status();
}
