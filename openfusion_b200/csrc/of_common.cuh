// of_common.cuh -- shared device/host helpers of the sm_100a fusion path.
//
// Camera conventions follow the reference (Source/include/CudaUtilities.cuh:9-64):
// camera-space z is negative in front of the camera, a pixel (u, v) of depth D
// back-projects to (-D (u-cx)/fx, -D (v-cy)/fy, -D), and a point projects as
// u = fx X / Z + cx. Pixel rounding is the reference's roundFloat (frac < 0.5 ?
// floor : ceil, CudaUtilities.cuh:62-64).
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <math.h>

#include "openfusion_b200.h"

#include <nvtx3/nvToolsExt.h>

// An NVTX range around a C-ABI call (visible in Nsight timelines; near-zero
// cost when no tool is attached). Host-side only: a graph replay shows the
// call that launched it, not the captured stages.
struct OfNvtxRange {
  explicit OfNvtxRange(const char *name) { nvtxRangePushA(name); }
  ~OfNvtxRange() { nvtxRangePop(); }
};
#define OF_RANGE(name) OfNvtxRange of_nvtx_range_(name)

#define OF_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) return of_set_cuda_error(_e);    \
  } while (0)

of_status_t of_set_cuda_error(cudaError_t e);
of_status_t of_launch_status();

namespace of {

constexpr int kBrick = 8;            // brick edge, voxels
constexpr int kBrickVoxels = 512;    // 8^3
constexpr float kQ = 32767.0f;       // int16 tsdf scale (tsdf / trunc * kQ)
constexpr int kMaxLevels = 4;
constexpr int kSmCount = 148;

// ---------------------------------------------------------------- cameras --

struct Cam {
  int w, h;
  float fx, fy, cx, cy;
  float ifx, ify;   // 1/fx, 1/fy (rounded from FP64)
  float dmin, dmax;
};

__host__ __device__ inline Cam make_cam(const of_camera_t &c) {
  Cam k;
  k.w = c.width; k.h = c.height;
  k.fx = c.fx; k.fy = c.fy; k.cx = c.cx; k.cy = c.cy;
  k.ifx = (float)(1.0 / (double)c.fx);
  k.ify = (float)(1.0 / (double)c.fy);
  k.dmin = c.min_depth_mm; k.dmax = c.max_depth_mm;
  return k;
}

// Level l intrinsics: fx/2^l, c_{l+1} = (c_l - 0.5) / 2 (pixel (x, y) of level
// l+1 covers pixels 2x..2x+1 of level l, centred at 2x + 0.5).
__host__ __device__ inline of_camera_t camera_level(const of_camera_t &c, int level) {
  of_camera_t o = c;
  for (int l = 0; l < level; ++l) {
    o.width = (o.width + 1) / 2;
    o.height = (o.height + 1) / 2;
    o.fx *= 0.5f; o.fy *= 0.5f;
    o.cx = (o.cx - 0.5f) * 0.5f;
    o.cy = (o.cy - 0.5f) * 0.5f;
  }
  return o;
}

// roundFloat (CudaUtilities.cuh:62-64).
__device__ __forceinline__ int round_ref(float a) {
  float f = floorf(a);
  return (a - f) < 0.5f ? (int)f : (int)ceilf(a);
}

// ------------------------------------------------------------------ poses --

// A rigid transform in FP32: y = R x + t, R row-major.
struct Rigid {
  float r[9];
  float t[3];
};

__device__ __forceinline__ float3 apply(const Rigid &T, float3 p) {
  return make_float3(fmaf(T.r[0], p.x, fmaf(T.r[1], p.y, fmaf(T.r[2], p.z, T.t[0]))),
                     fmaf(T.r[3], p.x, fmaf(T.r[4], p.y, fmaf(T.r[5], p.z, T.t[1]))),
                     fmaf(T.r[6], p.x, fmaf(T.r[7], p.y, fmaf(T.r[8], p.z, T.t[2]))));
}
__device__ __forceinline__ float3 rotate(const Rigid &T, float3 p) {
  return make_float3(fmaf(T.r[0], p.x, fmaf(T.r[1], p.y, T.r[2] * p.z)),
                     fmaf(T.r[3], p.x, fmaf(T.r[4], p.y, T.r[5] * p.z)),
                     fmaf(T.r[6], p.x, fmaf(T.r[7], p.y, T.r[8] * p.z)));
}

// FP64 pose (row-major 4x4 camera-to-world) -> FP32 camera-to-world and
// world-to-camera (rigid inverse R^T, -R^T t), both rounded from FP64.
__device__ inline void pose_to_rigid(const double *P, Rigid *c2w, Rigid *w2c) {
  if (c2w) {
    for (int i = 0; i < 3; ++i) {
      for (int j = 0; j < 3; ++j) c2w->r[3 * i + j] = (float)P[4 * i + j];
      c2w->t[i] = (float)P[4 * i + 3];
    }
  }
  if (w2c) {
    for (int i = 0; i < 3; ++i) {
      double acc = 0.0;
      for (int j = 0; j < 3; ++j) {
        w2c->r[3 * i + j] = (float)P[4 * j + i];
        acc = fma(-P[4 * j + i], P[4 * j + 3], acc);
      }
      w2c->t[i] = (float)acc;
    }
  }
}

// ------------------------------------------------- float-pair arithmetic --
// Error-free transformations (Knuth two-sum, fma two-product) used where an
// FP32 result must match an FP64 oracle to better than one int16 tsdf step.

__device__ __forceinline__ float2 two_sum(float a, float b) {
  float s = __fadd_rn(a, b);
  float bb = __fsub_rn(s, a);
  float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return make_float2(s, e);
}
__device__ __forceinline__ float2 two_prod(float a, float b) {
  float p = __fmul_rn(a, b);
  return make_float2(p, __fmaf_rn(a, b, -p));
}
// (hi, lo) = x^2 for x = (xh, xl).
__device__ __forceinline__ float2 df_sq(float xh, float xl) {
  float2 p = two_prod(xh, xh);
  p.y = __fmaf_rn(2.0f * xh, xl, p.y);
  return p;
}
__device__ __forceinline__ float2 df_add(float2 a, float2 b) {
  float2 s = two_sum(a.x, b.x);
  float lo = __fadd_rn(s.y, __fadd_rn(a.y, b.y));
  return two_sum(s.x, lo);
}
// sqrt of a float pair (a.x >= 0): r = a.x * rsqrt(a.x), within a few ulp,
// then one Newton correction (a - r^2) / (2 r) from the residual, which the
// fma forms exactly; the pair (r, correction) is within ~(ulp of r)^2 / r of
// the root, some 1e-10 of the value.
__device__ __forceinline__ float2 df_sqrt(float2 a) {
  const float y = rsqrtf(a.x);
  const bool pos = a.x > 0.f;
  const float r = pos ? a.x * y : 0.f;
  const float e = __fadd_rn(__fmaf_rn(-r, r, a.x), a.y);
  return make_float2(r, pos ? e * (0.5f * y) : 0.f);
}

// ------------------------------------------------------------------ voxels --

struct VolGeom {
  int n;          // voxels per edge
  int nb;         // bricks per edge
  float vs;       // voxel size, mm (rounded)
  float origin;   // -size/2, mm (rounded)
  float trunc;    // mm
  float inv_trunc;
  int max_w;
};

__host__ __device__ inline VolGeom make_geom(const of_volume_desc_t &d) {
  VolGeom g;
  g.n = d.resolution;
  g.nb = d.resolution / kBrick;
  g.vs = (float)((double)d.size_mm / (double)d.resolution);
  g.origin = (float)(-0.5 * (double)d.size_mm);
  g.trunc = d.trunc_mm;
  g.inv_trunc = (float)(1.0 / (double)d.trunc_mm);
  g.max_w = d.max_weight;
  return g;
}

// Brick-major address of voxel (i, j, k): bricks in x-major order, voxels
// inside a brick x-major with z fastest.
__host__ __device__ __forceinline__ size_t vox_index(int nb, int i, int j, int k) {
  size_t b = ((size_t)(i >> 3) * nb + (size_t)(j >> 3)) * nb + (size_t)(k >> 3);
  return (b << 9) | (size_t)(((i & 7) << 6) | ((j & 7) << 3) | (k & 7));
}

// Brick flags follow the voxels: one byte per brick, set (sticky) on a brick
// and its 26 neighbours when a voxel of the brick is written with |tsdf| < 1.
// An unflagged brick and all its neighbours hold only saturated (+1) or
// unobserved voxels.
__host__ __device__ __forceinline__ uint8_t *brick_flags(void *vol, int n) {
  return (uint8_t *)vol + (size_t)n * n * n * sizeof(uint32_t);
}
// One flag byte per super-brick of 4^3 bricks (32^3 voxels) after the brick
// flags: set iff one of its bricks' flags is set (both are sticky).
constexpr int kSuper = 4;
__host__ __device__ __forceinline__ int super_count(int n) { return (n / 8 + kSuper - 1) / kSuper; }
__host__ __device__ __forceinline__ uint8_t *super_flags(void *vol, int n) {
  const size_t nb = (size_t)(n / 8);
  return brick_flags(vol, n) + ((nb * nb * nb + 255) & ~(size_t)255);
}

// One byte per brick after the super-brick flags: bit w (w = 0..3) set when,
// after the last integration that processed the brick, its voxels 128 w ..
// 128 w + 127 were all +1 at the maximum weight; 0xF = saturated free space.
// Updating a saturated brick with +1 leaves every word as it is, so the tiled
// integration does not list it for its free-space modes.
__host__ __device__ __forceinline__ uint8_t *saturated_flags(void *vol, int n) {
  const size_t ns = (size_t)super_count(n);
  return super_flags(vol, n) + ((ns * ns * ns + 255) & ~(size_t)255);
}

template <int STORAGE>
struct VoxelCodec;

template <>
struct VoxelCodec<OF_TSDF_I16> {
  static constexpr uint32_t kOneBits = 32767u;  // stored bits of tsdf = +1
  // normalised tsdf in [-1, 1]; int16 <-> float without I2F/F2I: for |q| <
  // 2^22, 1.5 * 2^23 + q is exact in FP32 and adding 1.5 * 2^23 rounds to the
  // nearest integer, ties to even (the FP32 default rounding).
  __device__ __forceinline__ static float tsdf(uint32_t w) {
    int q = ((int)(w << 16)) >> 16;
    return (__int_as_float(0x4B400000 + q) - 12582912.0f) * (1.0f / kQ);
  }
  __device__ __forceinline__ static uint32_t pack(float tsdf_norm, uint32_t weight) {
    float x = fminf(fmaxf(tsdf_norm * kQ, -kQ), kQ);
    int q = __float_as_int(x + 12582912.0f) - 0x4B400000;
    return ((uint32_t)q & 0xffffu) | (weight << 16);
  }
};

template <>
struct VoxelCodec<OF_TSDF_F16> {
  static constexpr uint32_t kOneBits = 0x3C00u;  // IEEE half 1.0
  __device__ __forceinline__ static float tsdf(uint32_t w) {
    return __half2float(__ushort_as_half((unsigned short)(w & 0xffffu)));
  }
  __device__ __forceinline__ static uint32_t pack(float tsdf_norm, uint32_t weight) {
    tsdf_norm = fminf(1.0f, fmaxf(-1.0f, tsdf_norm));
    return (uint32_t)__half_as_ushort(__float2half_rn(tsdf_norm)) | (weight << 16);
  }
};

// Normalised tsdf of a voxel word; an unobserved voxel (weight 0) reads +1
// (the reference initialises tsdf to +TRUNCATION, General.cu:27-50).
template <int STORAGE>
__device__ __forceinline__ float vox_value(uint32_t w) {
  return (w >> 16) == 0u ? 1.0f : VoxelCodec<STORAGE>::tsdf(w);
}

// --------------------------------------------------------------- pyramids --

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace of
