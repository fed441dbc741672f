// of_preprocess.cu -- depth pre-processing: bilateral filter (Tomasi &
// Manduchi 1998, as used by KinectFusion, Newcombe et al. ISMAR 2011 s3.2),
// guarded 2x2 depth pyramid and per-level camera-space vertex/normal maps.
//
// The vertex map follows d_convertDepthToWorldVertices
// (Source/src/CameraSupport/CameraHandler.cu:65-89) in camera space, and the
// normal map follows d_convertDepthToWorldNormals (CameraHandler.cu:91-132):
// n = normalize((v(x+1,y) - v) x (v(x,y+1) - v)), invalid on the last
// row/column, where a neighbour is invalid, or where the cross product is zero.
// The world transform the reference applies at every ICP iteration
// (ICP.cpp:174) is applied on the fly inside the ICP kernel instead.
#include "of_batch.cuh"

using namespace of;

bool of_camera_valid(const of_camera_t *c);

namespace {

constexpr int kTileX = 32;
constexpr int kTileY = 8;
constexpr int kMaxRadius = 16;

__device__ __forceinline__ bool depth_valid(float d, float dmin, float dmax) {
  return d > 0.f && d >= dmin && d <= dmax;
}

// Bilateral filter of the raw uint16 depth. Invalid centre -> 0; invalid
// neighbours get weight 0. Weight = 2^-(r^2 ks + delta^2 kr) with
// ks = log2(e)/(2 sigma_s^2), kr = log2(e)/(2 sigma_r^2).
__global__ void __launch_bounds__(256) k_bilateral(const uint16_t *__restrict__ depth, int pitch,
                                                   int w, int h, float dmin, float dmax, int R,
                                                   float ks, float kr, float *__restrict__ out) {
  extern __shared__ float tile[];
  const int tw = kTileX + 2 * R;
  const int th = kTileY + 2 * R;
  const int x0 = blockIdx.x * kTileX - R;
  const int y0 = blockIdx.y * kTileY - R;
  for (int i = threadIdx.x; i < tw * th; i += blockDim.x) {
    int tx = i % tw, ty = i / tw;
    int gx = x0 + tx, gy = y0 + ty;
    float d = 0.f;
    if (gx >= 0 && gx < w && gy >= 0 && gy < h) {
      d = (float)__ldg(depth + (size_t)gy * pitch + gx);
      if (!depth_valid(d, dmin, dmax)) d = 0.f;
    }
    tile[i] = d;
  }
  __syncthreads();
  const int lx = threadIdx.x % kTileX, ly = threadIdx.x / kTileX;
  const int x = blockIdx.x * kTileX + lx, y = blockIdx.y * kTileY + ly;
  if (x >= w || y >= h) return;
  const float c = tile[(ly + R) * tw + lx + R];
  float result = 0.f;
  if (c > 0.f) {
    float sw = 0.f, sd = 0.f;
    for (int dy = -R; dy <= R; ++dy) {
      const float *row = tile + (ly + R + dy) * tw + lx + R;
      const float ry = (float)(dy * dy) * ks;
      for (int dx = -R; dx <= R; ++dx) {
        float q = row[dx];
        float del = q - c;
        float e = fmaf(del * del, kr, fmaf((float)(dx * dx), ks, ry));
        float wt = q > 0.f ? exp2f(-e) : 0.f;
        sw += wt;
        sd = fmaf(wt, q, sd);
      }
    }
    result = sd / sw;
  }
  out[(size_t)y * w + x] = result;
}

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Same filter with the radius fixed at compile time (taps fully unrolled).
// Invalid depths are stored as -1e30 in the tile: their squared range
// difference overflows to +inf and their weight 2^-inf is exactly 0, so no
// per-tap select is needed. One ex2 per tap.
// (tile (bx, by) of the image; the kernels below pass their block index)
template <int R, bool UNROLL_ROWS>
__device__ __forceinline__ void bilateral_tile(const uint16_t *__restrict__ depth, int pitch,
                                               int w, int h, float dmin, float dmax, float ks,
                                               float kr, float *__restrict__ out, int bx, int by) {
  constexpr int TW = kTileX + 2 * R;
  constexpr int TH = kTileY + 2 * R;
  __shared__ float tile[TH * TW];
  const int x0 = bx * kTileX - R;
  const int y0 = by * kTileY - R;
  for (int i = threadIdx.x; i < TW * TH; i += blockDim.x) {
    int tx = i % TW, ty = i / TW;
    int gx = x0 + tx, gy = y0 + ty;
    float d = -1e30f;
    if (gx >= 0 && gx < w && gy >= 0 && gy < h) {
      float v = (float)__ldg(depth + (size_t)gy * pitch + gx);
      if (depth_valid(v, dmin, dmax)) d = v;
    }
    tile[i] = d;
  }
  __syncthreads();
  const int lx = threadIdx.x % kTileX, ly = threadIdx.x / kTileX;
  const int x = bx * kTileX + lx, y = by * kTileY + ly;
  if (x >= w || y >= h) return;
  const float *ctr = tile + (ly + R) * TW + lx + R;
  const float c = *ctr;
  float result = 0.f;
  if (c > 0.f) {
    const float nkr = -kr;
    float sw = 0.f, sd = 0.f;
    // single-stream filter: rows not unrolled (32 registers a thread, see
    // filter_footprint); the batched one unrolls them (the same sums)
    auto row = [&](int dy) {
      const float ry = -(float)(dy * dy) * ks;
#pragma unroll
      for (int dx = -R; dx <= R; ++dx) {
        float q = ctr[dy * TW + dx];
        float del = q - c;
        float e = fmaf(del * nkr, del, fmaf(-(float)(dx * dx), ks, ry));
        float wt = ex2_approx(e);
        sw += wt;
        sd = fmaf(wt, q, sd);
      }
    };
    if (UNROLL_ROWS) {
#pragma unroll
      for (int dy = -R; dy <= R; ++dy) row(dy);
    } else {
#pragma unroll 1
      for (int dy = -R; dy <= R; ++dy) row(dy);
    }
    result = sd / sw;
  }
  out[(size_t)y * w + x] = result;
}

template <int R>
__global__ void __launch_bounds__(256) k_bilateral_r(const uint16_t *__restrict__ depth, int pitch,
                                                     int w, int h, float dmin, float dmax,
                                                     float ks, float kr, float *__restrict__ out) {
  bilateral_tile<R, false>(depth, pitch, w, h, dmin, dmax, ks, kr, out, blockIdx.x, blockIdx.y);
}

// No filter: the raw depth as float, invalid -> 0 (the reference converts the
// raw depth, CameraHandler.cu:65-89).
__device__ __forceinline__ void depth_raw_tile(const uint16_t *__restrict__ depth, int pitch,
                                               int w, int h, float dmin, float dmax,
                                               float *__restrict__ out, int bx, int by) {
  int x = bx * blockDim.x + threadIdx.x;
  int y = by * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  float d = (float)depth[(size_t)y * pitch + x];
  out[(size_t)y * w + x] = depth_valid(d, dmin, dmax) ? d : 0.f;
}
__global__ void k_depth_raw(const uint16_t *__restrict__ depth, int pitch, int w, int h,
                            float dmin, float dmax, float *__restrict__ out) {
  depth_raw_tile(depth, pitch, w, h, dmin, dmax, out, blockIdx.x, blockIdx.y);
}

// Level l -> l+1: pixel (x, y) averages the valid pixels of the 2x2 block
// {2x, 2x+1} x {2y, 2y+1} that lie within 3 sigma_r of the block's first
// valid pixel (row-major order); 0 if the block has none.
__device__ __forceinline__ void pyr_down_tile(const float *__restrict__ src, int sw, int sh,
                                              float *__restrict__ dst, int dw, int dh, float guard,
                                              int bx, int by) {
  int x = bx * blockDim.x + threadIdx.x;
  int y = by * blockDim.y + threadIdx.y;
  if (x >= dw || y >= dh) return;
  float ref = 0.f, sum = 0.f;
  int cnt = 0;
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      int sx = 2 * x + i, sy = 2 * y + j;
      if (sx < sw && sy < sh) {
        float d = src[(size_t)sy * sw + sx];
        if (d > 0.f) {
          if (cnt == 0) ref = d;
          if (fabsf(d - ref) <= guard) {
            sum += d;
            ++cnt;
          }
        }
      }
    }
  dst[(size_t)y * dw + x] = cnt ? sum / (float)cnt : 0.f;
}
__global__ void k_pyr_down(const float *__restrict__ src, int sw, int sh, float *__restrict__ dst,
                           int dw, int dh, float guard) {
  pyr_down_tile(src, sw, sh, dst, dw, dh, guard, blockIdx.x, blockIdx.y);
}

// Camera-space vertex and normal of every pixel of one level. Differences
// of neighbouring vertices are formed from depth differences (no
// cancellation between large coordinates).
__device__ __forceinline__ void vertex_normal_tile(const float *__restrict__ depth, int w, int h,
                                                   float cx, float cy, float ifx, float ify,
                                                   float4 *__restrict__ pts, int bx, int by) {
  int x = bx * blockDim.x + threadIdx.x;
  int y = by * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  size_t p = (size_t)y * w + x;
  float d = depth[p];
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 n = make_float4(0.f, 0.f, 0.f, 0.f);
  if (d > 0.f) {
    float ax = (float)x - cx, ay = (float)y - cy;
    v = make_float4(-d * ax * ifx, -d * ay * ify, -d, 1.f);
    if (x + 1 < w && y + 1 < h) {
      float d10 = depth[p + 1];
      float d01 = depth[p + w];
      if (d10 > 0.f && d01 > 0.f) {
        float e10 = d10 - d, e01 = d01 - d;
        float3 a = make_float3(-ifx * fmaf(e10, ax, d10), -ify * ay * e10, -e10);
        float3 b = make_float3(-ifx * ax * e01, -ify * fmaf(e01, ay, d01), -e01);
        float3 c = make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
        float l2 = c.x * c.x + c.y * c.y + c.z * c.z;
        if (l2 > 0.f) {
          float il = rsqrtf(l2);
          il = il * (1.5f - 0.5f * l2 * il * il);  // one Newton step on rsqrt
          n = make_float4(c.x * il, c.y * il, c.z * il, 1.f);
        }
      }
    }
  }
  pts[2 * p] = v;
  pts[2 * p + 1] = n;
}
__global__ void k_vertex_normal(const float *__restrict__ depth, int w, int h, float cx, float cy,
                                float ifx, float ify, float4 *__restrict__ pts) {
  vertex_normal_tile(depth, w, h, cx, cy, ifx, ify, pts, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------- batched --
// Jobs of the batched launches (one per stream, or per stream and level);
// gx = tiles per image row.
struct FilterJob {
  const uint16_t *depth[2];
  int pitch, w, h, gx;
  float dmin, dmax;
  float *out;
};
struct PyrJob {
  const float *src;
  float *dst;
  int sw, sh, dw, dh, gx;
};
struct VnJob {
  const float *depth;
  float4 *pts;
  int w, h, gx;
  float cx, cy, ifx, ify;
};

template <int R>
__global__ void __launch_bounds__(256) k_bilateral_batch(const FilterJob *__restrict__ jobs,
                                                         const int *__restrict__ first, int n,
                                                         int parity, float ks, float kr) {
  const int j = batch_job(first, n, blockIdx.x);
  const FilterJob &J = jobs[j];
  const int b = blockIdx.x - __ldg(first + j);
  bilateral_tile<R, true>(J.depth[parity], J.pitch, J.w, J.h, J.dmin, J.dmax, ks, kr, J.out, b % J.gx,
                    b / J.gx);
}
// The single-stream filter runs on the step graph's pre-processing branch, at
// the lower stream priority, beside the integration and the raycast. A block of it that
// sits on an SM holds registers and threads that their blocks then wait for,
// so the filter keeps a small footprint: 32 registers a thread and at most
// kFilterBlocksPerSm blocks per SM, set by a reservation of dynamic shared
// memory that the kernel leaves unused. Measured at C2 (300 frames, alternating
// runs on one B200): fully unrolled rows (128 registers, two blocks filling
// the register file) 2956 / 2903-2916 frames/s (value / e2e); 32 registers
// and two blocks per SM 3008 / 2941-2946; three per SM 2964-2967; one per SM
// gained `value` but lost `e2e` (the branch then took 108 us); 32 registers
// with no cap (eight per SM) lost 3 %. The filtered depth is the same bits.
// (The batched filter keeps the unrolled rows and no cap: capped the same way
// it lost 5 % of the 64-stream batch's frames/s.)
constexpr int kFilterBlocksPerSm = 2;
template <typename Kernel>
cudaError_t filter_footprint(Kernel *k, size_t *dyn) {
  int dev = 0, smem_sm = 0, reserved = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
  cudaFuncAttributes fa = {};
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, (const void *)k);
  if (e != cudaSuccess) return e;
  long d = (long)smem_sm / kFilterBlocksPerSm - (long)fa.sharedSizeBytes - reserved;
  if (d < 0) d = 0;
  *dyn = (size_t)d;
  // (set on every call: the attribute belongs to the current context)
  return cudaFuncSetAttribute((const void *)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d);
}

__global__ void k_depth_raw_batch(const FilterJob *__restrict__ jobs, const int *__restrict__ first,
                                  int n, int parity) {
  const int j = batch_job(first, n, blockIdx.x);
  const FilterJob &J = jobs[j];
  const int b = blockIdx.x - __ldg(first + j);
  depth_raw_tile(J.depth[parity], J.pitch, J.w, J.h, J.dmin, J.dmax, J.out, b % J.gx, b / J.gx);
}
__global__ void k_pyr_down_batch(const PyrJob *__restrict__ jobs, const int *__restrict__ first,
                                 int n, float guard) {
  const int j = batch_job(first, n, blockIdx.x);
  const PyrJob &J = jobs[j];
  const int b = blockIdx.x - __ldg(first + j);
  pyr_down_tile(J.src, J.sw, J.sh, J.dst, J.dw, J.dh, guard, b % J.gx, b / J.gx);
}
__global__ void k_vertex_normal_batch(const VnJob *__restrict__ jobs, const int *__restrict__ first,
                                      int n) {
  const int j = batch_job(first, n, blockIdx.x);
  const VnJob &J = jobs[j];
  const int b = blockIdx.x - __ldg(first + j);
  vertex_normal_tile(J.depth, J.w, J.h, J.cx, J.cy, J.ifx, J.ify, J.pts, b % J.gx, b / J.gx);
}

int filter_radius(const of_filter_params_t *fp) {
  return fp->radius_px > 0 ? fp->radius_px : (int)ceilf(2.0f * fp->sigma_space_px);
}

}  // namespace

namespace of {

// Level-0 filter of every stream in one launch, then one launch per pyramid
// level, then the vertex/normal maps of every (stream, level) in one launch.
struct PreprocessBatch {
  int n = 0, levels = 0, radius = 0;
  float ks = 0.f, kr = 0.f, guard = 0.f;
  FilterJob *filter = nullptr;
  int *filter_first = nullptr, filter_blocks = 0;
  PyrJob *pyr[kMaxLevels] = {};
  int *pyr_first[kMaxLevels] = {}, pyr_blocks[kMaxLevels] = {};
  VnJob *vn = nullptr;
  int *vn_first = nullptr, vn_jobs = 0, vn_blocks = 0;
};

void preprocess_batch_destroy(PreprocessBatch *b) {
  if (!b) return;
  cudaFree(b->filter);
  cudaFree(b->filter_first);
  for (int l = 0; l < kMaxLevels; ++l) {
    cudaFree(b->pyr[l]);
    cudaFree(b->pyr_first[l]);
  }
  cudaFree(b->vn);
  cudaFree(b->vn_first);
  delete b;
}

of_status_t preprocess_batch_create(const BatchStream *s, int n, const BatchParams &p,
                                    PreprocessBatch **out) {
  const of_filter_params_t *fp = &p.filter;
  if (n < 1 || fp->levels < 1 || fp->levels > kMaxLevels || fp->sigma_space_px <= 0.f ||
      fp->sigma_range_mm <= 0.f || fp->radius_px < -1)
    return OF_ERR_INVALID_ARGUMENT;
  const int R = filter_radius(fp);
  const bool raw = fp->radius_px == -1;
  if (!raw && !(R >= 3 && R <= 10) && R != 12) return OF_ERR_INVALID_ARGUMENT;
  PreprocessBatch *b = new PreprocessBatch();
  b->n = n;
  b->levels = fp->levels;
  b->radius = raw ? -1 : R;
  const double log2e = 1.4426950408889634;
  b->ks = (float)(log2e / (2.0 * (double)fp->sigma_space_px * fp->sigma_space_px));
  b->kr = (float)(log2e / (2.0 * (double)fp->sigma_range_mm * fp->sigma_range_mm));
  b->guard = 3.0f * fp->sigma_range_mm;
  FilterJob *fj = new FilterJob[n];
  PyrJob *pj = new PyrJob[n];
  VnJob *vj = new VnJob[(size_t)n * fp->levels];
  int *first = new int[(size_t)n * fp->levels + 1];
  of_status_t st = OF_OK;
  // level-0 filter (32x8 tiles either way)
  first[0] = 0;
  for (int i = 0; i < n && st == OF_OK; ++i) {
    of_pyramid_layout_t lay;
    st = of_pyramid_layout(&s[i].cam, fp->levels, &lay);
    const int w = s[i].cam.width, h = s[i].cam.height;
    fj[i] = {{s[i].depth[0], s[i].depth[1]}, w, w, h, (w + kTileX - 1) / kTileX,
             s[i].cam.min_depth_mm, s[i].cam.max_depth_mm,
             (float *)((char *)s[i].frame + lay.depth_offset[0])};
    first[i + 1] = first[i] + fj[i].gx * ((h + kTileY - 1) / kTileY);
  }
  if (st == OF_OK) {
    b->filter_blocks = first[n];
    st = upload_jobs(fj, first, n, &b->filter, &b->filter_first);
  }
  for (int l = 1; l < fp->levels && st == OF_OK; ++l) {
    first[0] = 0;
    for (int i = 0; i < n; ++i) {
      of_pyramid_layout_t lay;
      of_pyramid_layout(&s[i].cam, fp->levels, &lay);
      char *base = (char *)s[i].frame;
      pj[i] = {(const float *)(base + lay.depth_offset[l - 1]), (float *)(base + lay.depth_offset[l]),
               lay.width[l - 1], lay.height[l - 1], lay.width[l], lay.height[l],
               (lay.width[l] + 31) / 32};
      first[i + 1] = first[i] + pj[i].gx * ((lay.height[l] + 7) / 8);
    }
    b->pyr_blocks[l] = first[n];
    st = upload_jobs(pj, first, n, &b->pyr[l], &b->pyr_first[l]);
  }
  if (st == OF_OK) {
    int k = 0;
    first[0] = 0;
    for (int i = 0; i < n; ++i) {
      of_pyramid_layout_t lay;
      of_pyramid_layout(&s[i].cam, fp->levels, &lay);
      char *base = (char *)s[i].frame;
      for (int l = 0; l < fp->levels; ++l, ++k) {
        const of_camera_t c = camera_level(s[i].cam, l);
        vj[k] = {(const float *)(base + lay.depth_offset[l]), (float4 *)(base + lay.points_offset[l]),
                 c.width, c.height, (c.width + 31) / 32, c.cx, c.cy,
                 (float)(1.0 / (double)c.fx), (float)(1.0 / (double)c.fy)};
        first[k + 1] = first[k] + vj[k].gx * ((c.height + 7) / 8);
      }
    }
    b->vn_jobs = k;
    b->vn_blocks = first[k];
    st = upload_jobs(vj, first, k, &b->vn, &b->vn_first);
  }
  delete[] fj;
  delete[] pj;
  delete[] vj;
  delete[] first;
  if (st != OF_OK) {
    preprocess_batch_destroy(b);
    return st;
  }
  *out = b;
  return OF_OK;
}

of_status_t preprocess_batch_launch(const PreprocessBatch *b, int parity, cudaStream_t s) {
  if (b->radius < 0) {
    k_depth_raw_batch<<<b->filter_blocks, dim3(32, 8), 0, s>>>(b->filter, b->filter_first, b->n,
                                                               parity);
  } else {
#define OF_BILATERAL_BATCH(RR)                                                          \
  case RR:                                                                              \
    k_bilateral_batch<RR><<<b->filter_blocks, kTileX * kTileY, 0, s>>>(                 \
        b->filter, b->filter_first, b->n, parity, b->ks, b->kr);                        \
    break;
    switch (b->radius) {
      OF_BILATERAL_BATCH(3)
      OF_BILATERAL_BATCH(4)
      OF_BILATERAL_BATCH(5)
      OF_BILATERAL_BATCH(6)
      OF_BILATERAL_BATCH(7)
      OF_BILATERAL_BATCH(8)
      OF_BILATERAL_BATCH(9)
      OF_BILATERAL_BATCH(10)
      OF_BILATERAL_BATCH(12)
      default:
        return OF_ERR_INVALID_ARGUMENT;
    }
#undef OF_BILATERAL_BATCH
  }
  for (int l = 1; l < b->levels; ++l)
    k_pyr_down_batch<<<b->pyr_blocks[l], dim3(32, 8), 0, s>>>(b->pyr[l], b->pyr_first[l], b->n,
                                                              b->guard);
  k_vertex_normal_batch<<<b->vn_blocks, dim3(32, 8), 0, s>>>(b->vn, b->vn_first, b->vn_jobs);
  return of_launch_status();
}

}  // namespace of

extern "C" of_status_t of_preprocess(const of_camera_t *cam, const of_filter_params_t *fp,
                                     const uint16_t *d_depth, int32_t pitch, void *d_frame,
                                     of_stream_t stream) {
  OF_RANGE("of_preprocess");
  if (!of_camera_valid(cam) || !fp || !d_depth || !d_frame || pitch < cam->width)
    return OF_ERR_INVALID_ARGUMENT;
  if (fp->levels < 1 || fp->levels > kMaxLevels || fp->sigma_space_px <= 0.f ||
      fp->sigma_range_mm <= 0.f)
    return OF_ERR_INVALID_ARGUMENT;
  int R = fp->radius_px > 0 ? fp->radius_px : (int)ceilf(2.0f * fp->sigma_space_px);
  if (R > kMaxRadius || fp->radius_px < -1) return OF_ERR_INVALID_ARGUMENT;
  of_pyramid_layout_t lay;
  of_status_t st = of_pyramid_layout(cam, fp->levels, &lay);
  if (st != OF_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  char *base = (char *)d_frame;
  const double log2e = 1.4426950408889634;
  float ks = (float)(log2e / (2.0 * (double)fp->sigma_space_px * fp->sigma_space_px));
  float kr = (float)(log2e / (2.0 * (double)fp->sigma_range_mm * fp->sigma_range_mm));
  if (fp->radius_px == -1) {
    dim3 blk(32, 8);
    dim3 grid((cam->width + 31) / 32, (cam->height + 7) / 8);
    k_depth_raw<<<grid, blk, 0, s>>>(d_depth, pitch, cam->width, cam->height, cam->min_depth_mm,
                                     cam->max_depth_mm, (float *)(base + lay.depth_offset[0]));
  } else {
    dim3 grid((cam->width + kTileX - 1) / kTileX, (cam->height + kTileY - 1) / kTileY);
    size_t smem = (size_t)(kTileX + 2 * R) * (kTileY + 2 * R) * sizeof(float);
    float *o = (float *)(base + lay.depth_offset[0]);
    const int W = cam->width, H = cam->height;
    const float dmn = cam->min_depth_mm, dmx = cam->max_depth_mm;
#define OF_BILATERAL_CASE(RR)                                                           \
  case RR: {                                                                            \
    size_t dyn_ = 0;                                                                    \
    const cudaError_t fe_ = filter_footprint(k_bilateral_r<RR>, &dyn_);                 \
    if (fe_ != cudaSuccess) return of_set_cuda_error(fe_);                              \
    k_bilateral_r<RR><<<grid, kTileX * kTileY, dyn_, s>>>(d_depth, pitch, W, H, dmn, dmx, \
                                                           ks, kr, o);                  \
  } break;
    switch (R) {
      OF_BILATERAL_CASE(3)
      OF_BILATERAL_CASE(4)
      OF_BILATERAL_CASE(5)
      OF_BILATERAL_CASE(6)
      OF_BILATERAL_CASE(7)
      OF_BILATERAL_CASE(8)
      OF_BILATERAL_CASE(9)
      OF_BILATERAL_CASE(10)
      OF_BILATERAL_CASE(12)
      default:
        k_bilateral<<<grid, kTileX * kTileY, smem, s>>>(d_depth, pitch, W, H, dmn, dmx, R, ks, kr,
                                                        o);
    }
#undef OF_BILATERAL_CASE
  }
  float guard = 3.0f * fp->sigma_range_mm;
  for (int l = 1; l < fp->levels; ++l) {
    dim3 blk(32, 8);
    dim3 grid((lay.width[l] + 31) / 32, (lay.height[l] + 7) / 8);
    k_pyr_down<<<grid, blk, 0, s>>>((const float *)(base + lay.depth_offset[l - 1]),
                                    lay.width[l - 1], lay.height[l - 1],
                                    (float *)(base + lay.depth_offset[l]), lay.width[l],
                                    lay.height[l], guard);
  }
  for (int l = 0; l < fp->levels; ++l) {
    of_camera_t c = camera_level(*cam, l);
    dim3 blk(32, 8);
    dim3 grid((c.width + 31) / 32, (c.height + 7) / 8);
    k_vertex_normal<<<grid, blk, 0, s>>>((const float *)(base + lay.depth_offset[l]), c.width,
                                         c.height, c.cx, c.cy, (float)(1.0 / (double)c.fx),
                                         (float)(1.0 / (double)c.fy),
                                         (float4 *)(base + lay.points_offset[l]));
  }
  return of_launch_status();
}
