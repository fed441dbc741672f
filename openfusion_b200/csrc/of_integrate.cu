// of_integrate.cu -- TSDF integration of one raw depth frame.
//
// Per voxel this is d_integrateVolume (Source/src/VolumeIntegrator.cu:86-187)
// with the intended indexing (voxel x lives in slab x):
//   p_c = T^-1 p_w; pixel = roundFloat(project(p_c)); skip if the pixel is in
//   the 2-pixel border or |z| is outside [min, max] depth (:12-16, :131) or the
//   voxel is behind the camera; skip if the depth at the pixel is invalid
//   (:136-140); SDF = |v_depth - c| - |p_w - c| (:146) where |v_depth - c| =
//   lambda(pixel) * D; skip if SDF < -trunc, else tsdf' = min(SDF, trunc)
//   (:148-160); running average with weight 1, weight capped at max_weight
//   (:165-166).
//
// B200 layout: one 32-bit word per voxel (int16 or fp16 tsdf/trunc + uint16
// weight), 8^3 bricks. 128 threads own one brick; each thread owns four
// z-consecutive voxels and touches memory with one 16-byte load and store,
// only when one of them is updated. A whole brick is skipped before any
// memory access when its 8 corner voxel centres lie outside one frustum plane.
// of_integrate_tiled adds whole-brick decisions from per-tile bounds of the
// depth frame: bricks that lie entirely behind the surface (beyond the
// truncation band) are skipped, bricks that lie entirely in free space are
// updated with +1 without projecting a voxel; the volume written is the same.
// The SDF of voxels near the truncation band is evaluated with float-pair
// arithmetic so that the stored int16 value matches an FP64 evaluation to
// within one quantisation step.
#include "of_batch.cuh"

using namespace of;

bool of_camera_valid(const of_camera_t *c);
bool of_volume_valid(const of_volume_desc_t *d);

namespace {

struct IntegrateSetup {
  float m[9];      // world-to-camera rotation scaled by the voxel size
  float o[3];      // camera-space centre of voxel (0,0,0)
  float vs_hi, vs_lo;
  float oc_hi[3], oc_lo[3];  // (origin + vs/2 - c) per axis, float pair
  double mb[9];    // world-to-camera rotation scaled by 8 voxels (one brick), FP64
  double ob[3];    // camera-space centre of voxel (0,0,0), FP64
  float cw[3];     // camera centre in world space
};

__device__ void make_setup(const double *P, const of_volume_desc_t &d, IntegrateSetup &S) {
  double vs = (double)d.size_mm / (double)d.resolution;
  double org = -0.5 * (double)d.size_mm + 0.5 * vs;  // centre of voxel 0
  double c[3] = {P[3], P[7], P[11]};
  for (int a = 0; a < 3; ++a) {
    double acc = 0.0;
    for (int b = 0; b < 3; ++b) {
      double rba = P[4 * b + a];  // (R^T)[a][b]
      S.m[3 * a + b] = (float)(rba * vs);
      S.mb[3 * a + b] = rba * vs * 8.0;
      acc += rba * (org - c[b]);
    }
    S.o[a] = (float)acc;
    S.ob[a] = acc;
    double oc = org - c[a];
    S.oc_hi[a] = (float)oc;
    S.oc_lo[a] = (float)(oc - (double)S.oc_hi[a]);
    S.cw[a] = (float)c[a];
  }
  S.vs_hi = (float)vs;
  S.vs_lo = (float)(vs - (double)S.vs_hi);
}

// (p_w - c)^2 along axis a for voxel index i, as a float pair.
__device__ __forceinline__ float2 axis_sq(const IntegrateSetup &S, int a, int i) {
  float fi = (float)i;
  float2 p = two_prod(fi, S.vs_hi);
  p.y = __fmaf_rn(fi, S.vs_lo, p.y);
  float2 q = two_sum(p.x, S.oc_hi[a]);
  float lo = __fadd_rn(__fadd_rn(p.y, q.y), S.oc_lo[a]);
  float2 dd = two_sum(q.x, lo);
  return df_sq(dd.x, dd.y);
}

// Frustum plane in world space: inside <=> n . p + d <= 0.
struct Plane {
  float nx, ny, nz, d;
};

// The six frustum planes (pixel border, min/max depth) in world space, with
// half a pixel / 1 mm of slack: the brick test only has to be conservative,
// the per-voxel test is exact.
__device__ void make_planes(const double *P, const Cam &cam, Plane *pl) {
  double umin = 1.0, umax = (double)cam.w - 2.0;
  double vmin = 1.0, vmax = (double)cam.h - 2.0;
  // camera-space planes (a, b, c, d): inside <=> a X + b Y + c Z + d <= 0
  double cp[6][4] = {{cam.fx, 0.0, cam.cx - umin, 0.0},
                     {-cam.fx, 0.0, umax - cam.cx, 0.0},
                     {0.0, cam.fy, cam.cy - vmin, 0.0},
                     {0.0, -cam.fy, vmax - cam.cy, 0.0},
                     {0.0, 0.0, 1.0, cam.dmin - 1.0},
                     {0.0, 0.0, -1.0, -cam.dmax - 1.0}};
  // X_cam = R^T (p - c): n_w = R n_c, d_w = d - n_w . c
  for (int q = 0; q < 6; ++q) {
    double nw[3];
    for (int i = 0; i < 3; ++i)
      nw[i] = P[4 * i] * cp[q][0] + P[4 * i + 1] * cp[q][1] + P[4 * i + 2] * cp[q][2];
    double dw = cp[q][3] - (nw[0] * P[3] + nw[1] * P[7] + nw[2] * P[11]);
    pl[q] = {(float)nw[0], (float)nw[1], (float)nw[2], (float)dw};
  }
}

constexpr int kChunk = 32;  // bricks tested per batch (one warp ballot)
constexpr int kTile = 8;    // depth-bound tiles are 8x8 pixels
constexpr int kMaxTiles = 64;  // a brick whose footprint covers more tiles is evaluated per voxel
// How a listed brick is integrated (of_integrate_tiled's work list).
constexpr int kModeFull = 0;        // per-voxel test, with the frustum/border checks
constexpr int kModeInside = 1;      // per-voxel test; every voxel is inside the frustum
constexpr int kModeFront = 2;       // free space: +1 where the voxel's pixel holds a valid depth
constexpr int kModeFrontDense = 3;  // free space, every pixel it reaches valid: +1 everywhere

// The per-frame constants of of_integrate_tiled, computed once (FP64) by its
// first step and copied to shared memory by the next two.
struct FrameSetup {
  IntegrateSetup S;
  Plane planes[6];
};

__device__ __forceinline__ void load_setup(const FrameSetup *g, FrameSetup *s) {
  static_assert(sizeof(FrameSetup) % 4 == 0, "word copy");
  const uint32_t *src = reinterpret_cast<const uint32_t *>(g);
  uint32_t *dst = reinterpret_cast<uint32_t *>(s);
  for (int i = threadIdx.x; i < (int)(sizeof(FrameSetup) / 4); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}

// of_integrate_tiled, step 1. Per 8x8 pixel tile of the raw depth frame, one
// warp: x = min and |y| = max of L = lambda * D over the tile's valid pixels
// (+inf and 0 if there is none); y carries a minus sign (-0 included) when a
// pixel of the tile is invalid. L is the same FP32 product the integration
// compares |p - c| with.
__device__ __forceinline__ void depth_tiles_block(const Cam &cam, const uint16_t *__restrict__ depth,
                                                  int pitch, const float2 *__restrict__ lam,
                                                  float2 *__restrict__ lmap,
                                                  float2 *__restrict__ tiles, int tiles_x,
                                                  int ntiles, unsigned int *list_count,
                                                  const double *__restrict__ pose,
                                                  const of_volume_desc_t &desc, FrameSetup *setup,
                                                  int bx) {
  const int tile = bx * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  // step 2 may be launched now (it waits for this grid before reading)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  if (bx == 0 && threadIdx.x == 0) {
    // for the next two steps: an empty work list, the frame's setup
    list_count[0] = 0;
    list_count[1] = 0;  // the work counter of step 3
    make_setup(pose, desc, setup->S);
    make_planes(pose, cam, setup->planes);
  }
  if (tile >= ntiles) return;  // warp-uniform
  const int tx = tile % tiles_x, ty = tile / tiles_x;
  const float dlo = fmaxf(cam.dmin, 0.5f), dhi = cam.dmax;
  float lmin = __int_as_float(0x7f800000), lmax = 0.f;
  bool all_valid = true;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int u = tx * kTile + (lane & 7), v = ty * kTile + (lane >> 3) + 4 * k;
    if (u < cam.w && v < cam.h) {
      const float D = (float)__ldg(depth + (size_t)v * pitch + u);
      const float2 lp = __ldg(lam + v * cam.w + u);
      const float2 Lp = two_prod(lp.x, D);
      const float L = Lp.x;
      const bool valid = D >= dlo && D <= dhi;
      all_valid &= valid;
      // the pixel's L = lambda D as a float pair (hi = the FP32 product), or
      // -1 where the depth is invalid
      lmap[v * cam.w + u] = valid ? make_float2(L, __fmaf_rn(lp.y, D, Lp.y)) : make_float2(-1.f, 0.f);
      if (valid) {
        lmin = fminf(lmin, L);
        lmax = fmaxf(lmax, L);
      }
    }
  }
  all_valid = __all_sync(0xffffffffu, all_valid);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lmin = fminf(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
    lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
  }
  if (lane == 0) tiles[tile] = make_float2(lmin, all_valid ? lmax : -lmax);
}
__global__ void __launch_bounds__(256) k_depth_tiles(Cam cam, const uint16_t *__restrict__ depth,
                                                     int pitch, const float2 *__restrict__ lam,
                                                     float2 *__restrict__ lmap,
                                                     float2 *__restrict__ tiles, int tiles_x,
                                                     int ntiles, unsigned int *list_count,
                                                     const double *__restrict__ pose,
                                                     of_volume_desc_t desc, FrameSetup *setup) {
  depth_tiles_block(cam, depth, pitch, lam, lmap, tiles, tiles_x, ntiles, list_count, pose, desc,
                    setup, blockIdx.x);
}

// Whole-brick decision from the tile bounds (one thread per brick). Returns
// -1 when no voxel of the brick can be updated, else the brick's mode:
// kModeFront(Dense) when every voxel whose pixel holds a valid depth is
// updated with tsdf' = +1 (free space), kModeInside / kModeFull when the
// voxels must be evaluated one by one, with or without the per-voxel frustum
// checks. Every verdict is conservative: each carries margins far above the
// FP32 rounding of the per-voxel test, so the volume written is the one the
// per-voxel test alone gives.
//   skip:  for every voxel with a valid depth D in its pixel,
//          |p - c| > L_max + T + slack >= L + T + slack  (the per-voxel skip);
//   inside: every voxel projects inside the border and depth range;
//   front: inside, and for every valid pixel it can reach
//          |p - c| < L_min - T - slack; dense: every pixel it can reach is valid.
// The pixel footprint is bounded by the projections of the 8 corner voxel
// centres (a box projects inside the hull of its corners' projections), one
// pixel wider on each side.
__device__ int classify_brick(const IntegrateSetup &S, const Cam &cam, const float2 *tiles,
                              int tiles_x, float T, float hext, float cx, float cy, float cz,
                              int bx, int by, int bz) {
  // distance range from the camera to the brick's voxel centres (world box)
  const float ex = fabsf(cx - S.cw[0]), ey = fabsf(cy - S.cw[1]), ez = fabsf(cz - S.cw[2]);
  const float ax = fmaxf(ex - hext, 0.f), ay = fmaxf(ey - hext, 0.f), az = fmaxf(ez - hext, 0.f);
  const float fx_ = ex + hext, fy_ = ey + hext, fz_ = ez + hext;
  const float rlo = sqrtf(fmaf(ax, ax, fmaf(ay, ay, az * az))) * (1.f - 1e-5f) - 0.01f;
  const float rhi = sqrtf(fmaf(fx_, fx_, fmaf(fy_, fy_, fz_ * fz_))) * (1.f + 1e-5f) + 0.01f;
  // camera-space corners: voxel (8b + 7i, 8b + 7j, 8b + 7k)
  const float gx = (float)(8 * bx), gy = (float)(8 * by), gz = (float)(8 * bz);
  const float X0 = fmaf(S.m[0], gx, fmaf(S.m[1], gy, fmaf(S.m[2], gz, S.o[0])));
  const float Y0 = fmaf(S.m[3], gx, fmaf(S.m[4], gy, fmaf(S.m[5], gz, S.o[1])));
  const float Z0 = fmaf(S.m[6], gx, fmaf(S.m[7], gy, fmaf(S.m[8], gz, S.o[2])));
  float umin = 3.4e38f, umax = -3.4e38f, vmin = 3.4e38f, vmax = -3.4e38f;
  float zmin = 3.4e38f, zmax = -3.4e38f;  // of -Z
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const float i = (c & 4) ? 7.f : 0.f, j = (c & 2) ? 7.f : 0.f, k = (c & 1) ? 7.f : 0.f;
    const float X = fmaf(S.m[0], i, fmaf(S.m[1], j, fmaf(S.m[2], k, X0)));
    const float Y = fmaf(S.m[3], i, fmaf(S.m[4], j, fmaf(S.m[5], k, Y0)));
    const float Z = fmaf(S.m[6], i, fmaf(S.m[7], j, fmaf(S.m[8], k, Z0)));
    const float rz = 1.0f / Z;
    const float u = fmaf(cam.fx * X, rz, cam.cx), v = fmaf(cam.fy * Y, rz, cam.cy);
    umin = fminf(umin, u); umax = fmaxf(umax, u);
    vmin = fminf(vmin, v); vmax = fmaxf(vmax, v);
    zmin = fminf(zmin, -Z); zmax = fmaxf(zmax, -Z);
  }
  if (!(zmin > 1.0f)) return kModeFull;  // reaches behind the camera: no bounded footprint
  // (clamped so that the integer pixel bounds cannot overflow)
  const int pu0 = __float2int_rd(fmaxf(umin + 0.5f, -1e8f)) - 1;
  const int pu1 = __float2int_rd(fminf(umax + 0.5f, 1e8f)) + 1;
  const int pv0 = __float2int_rd(fmaxf(vmin + 0.5f, -1e8f)) - 1;
  const int pv1 = __float2int_rd(fminf(vmax + 0.5f, 1e8f)) + 1;
  const int tx0 = max(pu0, 0) / kTile, tx1 = min(pu1, cam.w - 1) / kTile;
  const int ty0 = max(pv0, 0) / kTile, ty1 = min(pv1, cam.h - 1) / kTile;
  if (pu1 < 0 || pv1 < 0 || pu0 > cam.w - 1 || pv0 > cam.h - 1) return -1;  // off the image
  if ((tx1 - tx0 + 1) * (ty1 - ty0 + 1) > kMaxTiles) return kModeFull;
  float lmin = 3.4e38f, lmax = 0.f;
  bool dense = true;
  // eight tiles of a row per step, their loads issued together (a near
  // brick's footprint covers up to kMaxTiles tiles, mostly not yet in L1);
  // the padding (3.4e38, +0) changes none of the three bounds
  for (int ty = ty0; ty <= ty1; ++ty) {
    const float2 *row = tiles + ty * tiles_x;
    for (int tx = tx0; tx <= tx1; tx += 8) {
      float2 tb[8];
#pragma unroll
      for (int k = 0; k < 8; ++k)
        tb[k] = tx + k <= tx1 ? __ldg(row + tx + k) : make_float2(3.4e38f, 0.f);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        lmin = fminf(lmin, tb[k].x);
        lmax = fmaxf(lmax, fabsf(tb[k].y));
        dense &= !signbit(tb[k].y);
      }
    }
  }
  const float farb = fmaf(lmax, 1.f + 1e-5f, T + 0.05f) * (1.f + 2e-5f) + 0.02f;
  if (rlo > farb) return -1;
  const bool inside = pu0 >= 2 && pu1 <= cam.w - 3 && pv0 >= 2 && pv1 <= cam.h - 3 &&
                      zmin >= fmaf(zmin, 1e-5f, cam.dmin + 0.05f) &&
                      zmax <= cam.dmax - fmaf(zmax, 1e-5f, 0.05f);
  if (!inside) return kModeFull;
  const float nearb = (fmaf(lmin, 1.f - 1e-5f, -T) - 0.05f) * (1.f - 2e-5f) - 0.02f;
  if (!(rhi < nearb)) return kModeInside;
  return dense ? kModeFrontDense : kModeFront;
}

// What of_integrate's census counts instead of writing the volume.
constexpr int kCensusUpdated = 1;  // voxels the integration would update
constexpr int kCensusVisible = 2;  // voxels whose centre projects inside the
                                   // 2-pixel border within [min, max] depth

// Per-thread constants of the voxel loop.
struct VoxelConsts {
  float T, inv_T, dspan, cxh, cyh, dlo, dhi;
  unsigned uspan, vspan;
  int lx, ly, lz0, nb;
};

__device__ __forceinline__ VoxelConsts voxel_consts(const of_volume_desc_t &desc, const Cam &cam,
                                                    int t) {
  VoxelConsts K;
  K.T = desc.trunc_mm;
  K.inv_T = 1.0f / desc.trunc_mm;
  K.dspan = cam.dmax - cam.dmin;
  K.cxh = cam.cx + 0.5f;
  K.cyh = cam.cy + 0.5f;
  K.dlo = fmaxf(cam.dmin, 0.5f);
  K.dhi = cam.dmax;
  K.uspan = (unsigned)(cam.w - 4);
  K.vspan = (unsigned)(cam.h - 4);
  K.lx = t >> 4;
  K.ly = (t >> 1) & 7;
  K.lz0 = (t & 1) * 4;
  K.nb = desc.resolution >> 3;
  return K;
}

// Camera-space centre of brick (bx, by, bz)'s voxel (0,0,0), FP64 then
// rounded: per-voxel offsets from it stay below 8 voxels, so the FP32
// position error is about one rounding of the brick base.
__device__ __forceinline__ float3 brick_base(const IntegrateSetup &S, int bx, int by, int bz) {
  const double fbx = (double)bx, fby = (double)by, fbz = (double)bz;
  return make_float3((float)fma(S.mb[0], fbx, fma(S.mb[1], fby, fma(S.mb[2], fbz, S.ob[0]))),
                     (float)fma(S.mb[3], fbx, fma(S.mb[4], fby, fma(S.mb[5], fbz, S.ob[1]))),
                     (float)fma(S.mb[6], fbx, fma(S.mb[7], fby, fma(S.mb[8], fbz, S.ob[2]))));
}

// One brick, 128 threads: thread t owns voxels (lx, ly, lz0 .. lz0 + 3) of
// brick b, whose voxel (0,0,0) sits at camera-space `base`. `mode` (kMode*)
// says what is known of the brick: in the free-space modes a voxel is updated
// with tsdf' = +1 when its pixel holds a valid depth (always, when dense),
// with no ray length or distance evaluated; kModeInside drops the per-voxel
// frustum checks.
template <int STORAGE, int CENSUS, bool EARLY_LOAD = false, bool LMAP = false, int MODE = -1>
__device__ __forceinline__ void integrate_brick(
    uint32_t *__restrict__ vol, uint8_t *__restrict__ flags, const of_volume_desc_t &desc,
    const Cam &cam, const uint16_t *__restrict__ depth, int pitch,
    const float2 *__restrict__ lam, const IntegrateSetup &S, const VoxelConsts &K, int t,
    int lane, int b, int bx, int by, int bz, int mode_arg, float3 base, unsigned &my_count,
    int sat_old = -1, const float2 *__restrict__ lmap = nullptr) {
  // the brick's mode, a constant when the caller instantiates one per mode
  const int mode = MODE >= 0 ? MODE : mode_arg;
  const float T = K.T, inv_T = K.inv_T, dspan = K.dspan, cxh = K.cxh, cyh = K.cyh;
  const float dlo = K.dlo, dhi = K.dhi;
  const unsigned uspan = K.uspan, vspan = K.vspan;
  const int lx = K.lx, ly = K.ly, lz0 = K.lz0, nb = K.nb;
  float tnew[4];
  unsigned upd = 0;
  unsigned inb = 0;  // voxels inside the 2-pixel border and the depth range (kModeFull)
  bool near = false;
  uint4 *p4 = reinterpret_cast<uint4 *>(vol + ((size_t)b << 9)) + t;
  uint4 wv = make_uint4(0u, 0u, 0u, 0u);
  uint4 wfin;  // the thread's words after the update
  // listed bricks are nearly always updated: their words are loaded before
  // the depth gathers so that the two memory round trips overlap
  if (EARLY_LOAD && !CENSUS) wv = *p4;
  if (mode == kModeFrontDense) {
    upd = 0xfu;
    tnew[0] = tnew[1] = tnew[2] = tnew[3] = 1.0f;
    goto brick_done;
  }
  {
      const bool check = mode == kModeFull;
      float X0 = fmaf(S.m[0], (float)lx, fmaf(S.m[1], (float)ly, base.x));
      float Y0 = fmaf(S.m[3], (float)lx, fmaf(S.m[4], (float)ly, base.y));
      float Z0 = fmaf(S.m[6], (float)lx, fmaf(S.m[7], (float)ly, base.z));
      // phase 1: project the four voxels; phase 2: issue every gather before
      // any result is used; phase 3: decide
      float Xv[4], Yv[4], Zv[4];
      int pix[4], dix[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const float lz = (float)(lz0 + m);
        float X = fmaf(S.m[2], lz, X0);
        float Y = fmaf(S.m[5], lz, Y0);
        float Z = fmaf(S.m[8], lz, Z0);
        Xv[m] = X; Yv[m] = Y; Zv[m] = Z;
        float rz = __fdividef(1.0f, Z);
        // roundFloat as floor(x + 0.5): identical except within FP32
        // rounding of a half-integer
        int pu = __float2int_rd(fmaf(cam.fx * X, rz, cxh));
        int pv = __float2int_rd(fmaf(cam.fy * Y, rz, cyh));
        // -Z in [dmin, dmax] (and Z < 0), pixel outside the 2-pixel border
        // (known for the whole brick in every mode but kModeFull)
        bool ok = true;
        if (check)
          ok = (-Z - cam.dmin <= dspan) && (-Z >= cam.dmin) && (unsigned)(pu - 2) < uspan &&
               (unsigned)(pv - 2) < vspan;
        inb |= ok ? (1u << m) : 0u;
        pix[m] = ok ? pv * cam.w + pu : 0;
        dix[m] = ok ? pv * pitch + pu : 0;
      }
      if (!inb) goto brick_done;
      if (mode == kModeFront) {
        // free space: a voxel whose pixel holds a valid depth gets +1
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          bool valid;
          if (LMAP) {
            valid = __ldg(reinterpret_cast<const float *>(lmap) + 2 * pix[m]) > 0.f;
          } else {
            const float D = __int_as_float(0x4B000000 | (int)__ldg(depth + dix[m])) - 8388608.0f;
            valid = D >= dlo && D <= dhi;
          }
          tnew[m] = 1.0f;
          if (((inb >> m) & 1u) && valid) upd |= 1u << m;
        }
        goto brick_done;
      }
      {
        // per voxel: L = lambda D of its pixel as a float pair (hi = the
        // rounded FP32 product), hi < 0 where the depth is invalid
        float2 Lv[4];
        bool have_xy = false;
        float2 sxy = make_float2(0.f, 0.f);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          if (LMAP) {
            Lv[m] = __ldg(lmap + pix[m]);
          } else {
            // uint16 -> float without I2F: 2^23 + d is exact
            const float D = __int_as_float(0x4B000000 | (int)__ldg(depth + dix[m])) - 8388608.0f;
            const float2 lp = __ldg(lam + pix[m]);
            const float2 Lp = two_prod(lp.x, D);
            Lv[m] = (D >= dlo && D <= dhi) ? make_float2(Lp.x, __fmaf_rn(lp.y, D, Lp.y))
                                           : make_float2(-1.f, 0.f);
          }
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          tnew[m] = 0.f;
          if (!((inb >> m) & 1u) || !(Lv[m].x > 0.f)) continue;
          const float X = Xv[m], Y = Yv[m], Z = Zv[m];
          // SDF = L - r with L = lambda D, r = |p_c|; decide on squares first
          float r2 = fmaf(X, X, fmaf(Y, Y, Z * Z));
          const float L = Lv[m].x;
          const float slack = fmaf(1e-5f, L, 0.05f);
          float far = L + T + slack;            // SDF < -T - slack  <=>  r > far
          if (r2 > far * far) continue;
          float nearl = L - T - slack;          // SDF >  T + slack  <=>  r < nearl
          float sn = 1.0f;
          if (!(nearl > 0.f && r2 < nearl * nearl)) {
            // |p_w - c| as a float pair: the x and y terms are the thread's
            // constants within the brick, computed on first use
            if (!have_xy) {
              sxy = df_add(axis_sq(S, 0, bx * 8 + lx), axis_sq(S, 1, by * 8 + ly));
              have_xy = true;
            }
            float2 rr = df_sqrt(df_add(sxy, axis_sq(S, 2, bz * 8 + lz0 + m)));
            const float2 Lp = Lv[m];
            float sdf2 = __fadd_rn(__fsub_rn(Lp.x, rr.x), __fsub_rn(Lp.y, rr.y));
            if (sdf2 < -T) continue;
            sn = fminf(sdf2, T) * inv_T;
          }
          upd |= 1u << m;
          tnew[m] = sn;
        }
      }
      }
    brick_done:
      if (CENSUS) {
        my_count += __popc(CENSUS == kCensusVisible ? inb : upd);
      } else if (!upd) {
        if (!EARLY_LOAD) wv = *p4;
        wfin = wv;
      } else {
        if (!EARLY_LOAD) wv = *p4;
        uint32_t w4[4] = {wv.x, wv.y, wv.z, wv.w};
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          if (!(upd & (1u << m))) continue;
          uint32_t word = w4[m];
          uint32_t wt = word >> 16;
          if (tnew[m] == 1.0f && (word & 0xffffu) == VoxelCodec<STORAGE>::kOneBits) {
            // +1 (or unobserved) averaged with +1: the quotient below lies
            // within a few ulp of 1 and packs to the +1 bits again, so only
            // the weight changes
            w4[m] = VoxelCodec<STORAGE>::kOneBits | (min(wt + 1u, (uint32_t)desc.max_weight) << 16);
            continue;
          }
          // weight as float without I2F (2^23 + w is exact)
          float wf = __int_as_float(0x4B000000 | (int)wt) - 8388608.0f;
          float told = wt ? VoxelCodec<STORAGE>::tsdf(word) : 0.f;
          // (told w + tsdf') / (w + 1), within a few ulp of the rounded quotient
          float tn = __fdividef(__fmaf_rn(told, wf, tnew[m]), wf + 1.0f);
          uint32_t wn = min(wt + 1u, (uint32_t)desc.max_weight);
          w4[m] = VoxelCodec<STORAGE>::pack(tn, wn);
          near |= (w4[m] & 0xffffu) != VoxelCodec<STORAGE>::kOneBits;
        }
        // saturated free space (+1 at the maximum weight) stays as it is
        wfin = make_uint4(w4[0], w4[1], w4[2], w4[3]);
        if (w4[0] != wv.x || w4[1] != wv.y || w4[2] != wv.z || w4[3] != wv.w) *p4 = wfin;
      }
      if (!CENSUS) {
        // the brick's saturated byte: bit w belongs to the brick's warp w
        // (voxels 128 w .. 128 w + 127), set while that warp's voxels are all
        // +1 at the maximum weight; only a change of the warp's own state
        // touches memory (one word atomic; the byte shares its word with three
        // other bricks)
        const uint32_t satw = VoxelCodec<STORAGE>::kOneBits | ((uint32_t)desc.max_weight << 16);
        const bool sat = wfin.x == satw && wfin.y == satw && wfin.z == satw && wfin.w == satw;
        const bool vote = __all_sync(0xffffffffu, sat);
        if (lane == 0) {
          unsigned *word = reinterpret_cast<unsigned *>(saturated_flags(vol, desc.resolution)) + (b >> 2);
          const unsigned m = 1u << ((t >> 5) + 8 * (b & 3));
          // the brick's byte as its work-list entry carries it, else from memory
          const bool had = sat_old >= 0 ? ((sat_old >> (t >> 5)) & 1) != 0
                                        : (*reinterpret_cast<volatile unsigned *>(word) & m) != 0u;
          if (vote && !had) atomicOr(word, m);
          if (!vote && had) atomicAnd(word, ~m);
        }
      }
      // a warp that wrote a non-saturated voxel flags the brick and its 26
      // neighbours, and their super-bricks (lanes 0..26), unless an earlier
      // write did: bit 1 of the brick's own flag byte records that (flags are
      // cleared only by a reset). Byte ORs into the flag words, so that the
      // bytes come out the same in any order of the warps.
      if (!CENSUS && __any_sync(0xffffffffu, near)) {
        const bool done = (*reinterpret_cast<volatile uint8_t *>(flags + b) & 2u) != 0u;
        if (!__shfl_sync(0xffffffffu, done, 0) && lane < 27) {
          int ox = lane / 9 - 1, oy = (lane / 3) % 3 - 1, oz = lane % 3 - 1;
          int qx = bx + ox, qy = by + oy, qz = bz + oz;
          if ((unsigned)qx < (unsigned)nb && (unsigned)qy < (unsigned)nb && (unsigned)qz < (unsigned)nb) {
            const unsigned q = (unsigned)((qx * nb + qy) * nb + qz);
            const unsigned v = lane == 13 ? 3u : 1u;  // lane 13: the brick itself
            atomicOr(reinterpret_cast<unsigned *>(flags) + (q >> 2), v << (8 * (q & 3u)));
            const int ns = super_count(desc.resolution);
            const unsigned s = (unsigned)(((qx / kSuper) * ns + qy / kSuper) * ns + qz / kSuper);
            atomicOr(reinterpret_cast<unsigned *>(super_flags(vol, desc.resolution)) + (s >> 2),
                     1u << (8 * (s & 3u)));
          }
        }
      }
}

// The per-voxel integration over every brick of the volume (of_integrate,
// of_integrate_census). Persistent grid; bricks are dealt round-robin (brick b
// goes to CTA b mod grid), so every CTA gets a spatially spread, statistically
// equal share of the frustum. Per batch, warp 0 tests 32 of the CTA's bricks
// against the frustum (one lane each) and compacts the visible ones into a
// shared list; the two 128-thread halves then take list entries alternately.
template <int STORAGE, int CENSUS>
__global__ void __launch_bounds__(256, 4) k_integrate(uint32_t *__restrict__ vol, of_volume_desc_t desc,
                                                   Cam cam, const uint16_t *__restrict__ depth,
                                                   int pitch, const double *__restrict__ pose,
                                                   const float2 *__restrict__ lam,
                                                   unsigned long long *count) {
  __shared__ IntegrateSetup S;
  __shared__ Plane planes[6];
  __shared__ int s_list[kChunk][4];  // visible bricks of a batch: b, bx, by, bz
  __shared__ int s_nvis;
  __shared__ unsigned int s_count;
  if (threadIdx.x == 0) {
    make_setup(pose, desc, S);
    make_planes(pose, cam, planes);
    s_count = 0;
  }
  __syncthreads();
  const int nb = desc.resolution >> 3;
  const int nbricks = nb * nb * nb;
  const int half = threadIdx.x >> 7;
  const int t = threadIdx.x & 127;
  const int lane = threadIdx.x & 31;
  const VoxelConsts K = voxel_consts(desc, cam, t);
  const float vs = S.vs_hi;
  const float org = -0.5f * desc.size_mm;
  const float hext = 3.5f * vs + 1e-3f;  // half extent of a brick's voxel centres
  unsigned int my_count = 0;
  const int nb2 = nb * nb;
  uint8_t *flags = brick_flags(vol, desc.resolution);
  const int G = gridDim.x;
  for (int q0 = 0; blockIdx.x + q0 * G < nbricks; q0 += kChunk) {
    if (threadIdx.x < 32) {
      int b = blockIdx.x + (q0 + lane) * G;
      bool vis = false;
      int bx = 0, by = 0, bz = 0;
      if (b < nbricks) {
        bz = b % nb; by = (b / nb) % nb; bx = b / nb2;
        float cx = fmaf(vs, (float)(8 * bx) + 4.0f, org);
        float cy = fmaf(vs, (float)(8 * by) + 4.0f, org);
        float cz = fmaf(vs, (float)(8 * bz) + 4.0f, org);
        vis = true;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const Plane pl = planes[q];
          float e = fmaf(pl.nx, cx, fmaf(pl.ny, cy, fmaf(pl.nz, cz, pl.d)));
          float r = hext * (fabsf(pl.nx) + fabsf(pl.ny) + fabsf(pl.nz));
          vis &= (e - r) <= 0.f;
        }
      }
      unsigned m = __ballot_sync(0xffffffffu, vis);
      if (vis) {
        int slot = __popc(m & ((1u << lane) - 1u));
        s_list[slot][0] = b; s_list[slot][1] = bx; s_list[slot][2] = by; s_list[slot][3] = bz;
      }
      if (lane == 0) s_nvis = __popc(m);
    }
    __syncthreads();
    const int nvis = s_nvis;
    for (int e = half; e < nvis; e += 2) {
      const int bx = s_list[e][1], by = s_list[e][2], bz = s_list[e][3];
      integrate_brick<STORAGE, CENSUS>(vol, flags, desc, cam, depth, pitch, lam, S, K, t, lane,
                                       s_list[e][0], bx, by, bz, kModeFull,
                                       brick_base(S, bx, by, bz), my_count);
    }
    __syncthreads();
  }
  if (CENSUS) {
    for (int o = 16; o > 0; o >>= 1) my_count += __shfl_xor_sync(0xffffffffu, my_count, o);
    if (lane == 0 && my_count) atomicAdd(&s_count, my_count);
    __syncthreads();
    if (threadIdx.x == 0 && s_count) atomicAdd(count, (unsigned long long)s_count);
  }
}

// of_integrate_tiled, step 2: one thread per brick. Frustum test, then the
// whole-brick decision from the tile bounds; kept bricks are appended to the
// work list (one atomic per warp) as {bx | by << 8 | bz << 16 | mode << 24 |
// saturated-brick bits << 26, camera-space base of the brick (3 floats)}.
// Free-space bricks whose voxels are all saturated (+1 at the maximum weight)
// are left out: updating them would write nothing.
__device__ __forceinline__ void classify_block(const of_volume_desc_t &desc, const Cam &cam,
                                               const float2 *__restrict__ tiles, int tiles_x,
                                               const uint8_t *__restrict__ sat,
                                               uint4 *__restrict__ list,
                                               unsigned int *__restrict__ list_count,
                                               const FrameSetup *__restrict__ setup, int bx) {
  __shared__ FrameSetup F;
  // a programmatic launch (of_integrate_tiled outside graph capture) starts
  // before step 1 has finished: allow step 3's launch, then wait for step 1
  // (both are no-ops for a plain launch)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  load_setup(setup, &F);
  const IntegrateSetup &S = F.S;
  const Plane *planes = F.planes;
  const int nb = desc.resolution >> 3;
  const int nbricks = nb * nb * nb;
  const int lane = threadIdx.x & 31;
  const int b = bx * blockDim.x + threadIdx.x;
  const float vs = S.vs_hi;
  const float org = -0.5f * desc.size_mm;
  const float hext = 3.5f * vs + 1e-3f;
  bool keep = false;
  uint4 entry = make_uint4(0u, 0u, 0u, 0u);
  if (b < nbricks) {
    const int bz = b % nb, by = (b / nb) % nb, bx = b / (nb * nb);
    const float cx = fmaf(vs, (float)(8 * bx) + 4.0f, org);
    const float cy = fmaf(vs, (float)(8 * by) + 4.0f, org);
    const float cz = fmaf(vs, (float)(8 * bz) + 4.0f, org);
    keep = true;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const Plane pl = planes[q];
      float e = fmaf(pl.nx, cx, fmaf(pl.ny, cy, fmaf(pl.nz, cz, pl.d)));
      float r = hext * (fabsf(pl.nx) + fabsf(pl.ny) + fabsf(pl.nz));
      keep &= (e - r) <= 0.f;
    }
    if (keep) {
      const int cls = classify_brick(S, cam, tiles, tiles_x, desc.trunc_mm, hext, cx, cy, cz, bx,
                                     by, bz);
      // free space over saturated free space changes no word
      const bool noop = (cls == kModeFront || cls == kModeFrontDense) && __ldg(sat + b) == 0xF;
      keep = cls >= 0 && !noop;
      const float3 base = brick_base(S, bx, by, bz);
      entry = make_uint4((uint32_t)bx | (uint32_t)by << 8 | (uint32_t)bz << 16 |
                             (uint32_t)max(cls, 0) << 24 | (uint32_t)(__ldg(sat + b) & 0xF) << 26,
                         __float_as_uint(base.x), __float_as_uint(base.y), __float_as_uint(base.z));
    }
  }
  const unsigned m = __ballot_sync(0xffffffffu, keep);
  if (m) {
    const int leader = __ffs(m) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(list_count, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (keep) list[base + __popc(m & ((1u << lane) - 1u))] = entry;
  }
}
__global__ void __launch_bounds__(256) k_classify_bricks(of_volume_desc_t desc, Cam cam,
                                                         const double *__restrict__ pose,
                                                         const float2 *__restrict__ tiles,
                                                         int tiles_x,
                                                         const uint8_t *__restrict__ sat,
                                                         uint4 *__restrict__ list,
                                                         unsigned int *__restrict__ list_count,
                                                         const FrameSetup *__restrict__ setup) {
  classify_block(desc, cam, tiles, tiles_x, sat, list, list_count, setup, blockIdx.x);
}

// of_integrate_tiled, step 3: persistent grid over the work list. The work
// unit is a quarter of a listed brick (the 128 voxels of 2 x-slices, one warp
// of 32 threads with 4 voxels each). The list is cut into N chunks of up to
// kChunkBricks bricks, chunk c holding entries c, c + N, c + 2N, ...: a sample
// of the whole list, so chunks cost about the same although the cost of a
// brick varies by region. Warp w of a block takes quarter w & 3 of every
// other brick of the chunk, so the four quarters of a brick run side by side.
// Block b starts with chunk b; every further chunk comes from a counter (one
// atomic per chunk, requested when the current chunk starts and published at
// its closing barrier), so a block that starts late (its SM held by a
// concurrent branch of the frame graph) takes less work instead of delaying
// the stage by a fixed share.
constexpr unsigned kChunkBricks = 8;
template <int STORAGE>
__device__ __forceinline__ void integrate_list_block(uint32_t *__restrict__ vol,
                                                     const of_volume_desc_t &desc, const Cam &cam,
                                                     const uint16_t *__restrict__ depth, int pitch,
                                                     const float2 *__restrict__ lam,
                                                     const float2 *__restrict__ lmap,
                                                     const uint4 *__restrict__ list,
                                                     unsigned int *__restrict__ list_count,
                                                     const FrameSetup *__restrict__ setup,
                                                     unsigned bx, unsigned gx) {
  static_assert(kChunkBricks % 2 == 0, "two bricks per step of the 8 warps");
  __shared__ FrameSetup F;
  __shared__ unsigned s_chunk[2];
  asm volatile("griddepcontrol.wait;" ::: "memory");  // step 2's list (programmatic launch)
  load_setup(setup, &F);
  const IntegrateSetup &S = F.S;
  const unsigned n = *reinterpret_cast<volatile unsigned *>(list_count);
  const unsigned nchunks = (n + kChunkBricks - 1) / kChunkBricks;
  unsigned *next = list_count + 1;
  const int lane = threadIdx.x & 31;
  const unsigned warp = threadIdx.x >> 5;  // 8 warps
  const int t = (int)((warp & 3u) << 5) + lane;
  const VoxelConsts K = voxel_consts(desc, cam, t);
  uint8_t *flags = brick_flags(vol, desc.resolution);
  const int nb = K.nb;
  unsigned my_count = 0;
  int buf = 0;
  for (unsigned c = bx; c < nchunks; buf ^= 1) {
    unsigned nxt = 0;
    if (threadIdx.x == 0) nxt = gx + atomicAdd(next, 1u);
    for (unsigned k = warp >> 2; k < kChunkBricks; k += 2) {
      const unsigned e = c + k * nchunks;
      if (e >= n) break;
      const uint4 en = __ldg(list + e);
      const int bx = (int)(en.x & 0xffu), by = (int)((en.x >> 8) & 0xffu);
      const int bz = (int)((en.x >> 16) & 0xffu), mode = (int)((en.x >> 24) & 3u);
      const int sat_old = (int)((en.x >> 26) & 0xfu);
      const int b = (bx * nb + by) * nb + bz;
      const float3 base =
          make_float3(__uint_as_float(en.y), __uint_as_float(en.z), __uint_as_float(en.w));
      // (the mode is the same for the whole warp: one instantiation each for
      // the two per-voxel modes, whose tests it fixes)
      if (mode == kModeInside)
        integrate_brick<STORAGE, 0, true, true, kModeInside>(vol, flags, desc, cam, depth, pitch,
                                                              lam, S, K, t, lane, b, bx, by, bz,
                                                              mode, base, my_count, sat_old, lmap);
      else if (mode == kModeFull)
        integrate_brick<STORAGE, 0, true, true, kModeFull>(vol, flags, desc, cam, depth, pitch,
                                                            lam, S, K, t, lane, b, bx, by, bz,
                                                            mode, base, my_count, sat_old, lmap);
      else
        integrate_brick<STORAGE, 0, true, true>(vol, flags, desc, cam, depth, pitch, lam, S, K, t,
                                                lane, b, bx, by, bz, mode, base, my_count,
                                                sat_old, lmap);
    }
    if (threadIdx.x == 0) s_chunk[buf] = nxt;
    __syncthreads();
    c = s_chunk[buf];
  }
}
template <int STORAGE>
__global__ void __launch_bounds__(256, 4) k_integrate_list(uint32_t *__restrict__ vol,
                                                        of_volume_desc_t desc, Cam cam,
                                                        const uint16_t *__restrict__ depth,
                                                        int pitch, const double *__restrict__ pose,
                                                        const float2 *__restrict__ lam,
                                                        const float2 *__restrict__ lmap,
                                                        const uint4 *__restrict__ list,
                                                        unsigned int *__restrict__ list_count,
                                                        const FrameSetup *__restrict__ setup) {
  integrate_list_block<STORAGE>(vol, desc, cam, depth, pitch, lam, lmap, list, list_count, setup,
                                blockIdx.x, gridDim.x);
}

int tiles_x_of(const of_camera_t *cam) { return (cam->width + kTile - 1) / kTile; }
int tiles_of(const of_camera_t *cam) {
  return tiles_x_of(cam) * ((cam->height + kTile - 1) / kTile);
}

// Scratch of of_integrate_tiled: [0, 256) the work-list count and step 3's
// work counter, [256, 768) the frame setup, then the tile bounds (float2 per
// tile), the work list (16 B per brick) and the per-pixel L = lambda D map
// (float2 per pixel).
struct ScratchLayout {
  size_t setup, tiles, list, lmap, total;
};
static_assert(sizeof(FrameSetup) <= 512, "frame setup slot");
ScratchLayout scratch_layout(const of_volume_desc_t *d, const of_camera_t *cam) {
  const size_t nb = (size_t)(d->resolution / 8);
  ScratchLayout L;
  L.setup = 256;
  L.tiles = 768;
  L.list = L.tiles + (((size_t)tiles_of(cam) * sizeof(float2) + 255) & ~(size_t)255);
  L.lmap = L.list + ((nb * nb * nb * sizeof(uint4) + 255) & ~(size_t)255);
  L.total = L.lmap + (((size_t)cam->width * cam->height * sizeof(float2) + 255) & ~(size_t)255);
  return L;
}

unsigned persistent_blocks(const of_volume_desc_t *d) {
  size_t nb = (size_t)(d->resolution / 8);
  size_t nbr = nb * nb * nb;
  // 4 resident CTAs of 256 threads per SM
  return (unsigned)(nbr < (size_t)kSmCount * 4 ? nbr : (size_t)kSmCount * 4);
}

template <int CENSUS>
of_status_t launch_integrate(const of_volume_desc_t *d, void *vol, const of_camera_t *cam,
                             const uint16_t *depth, int pitch, const double *pose,
                             const float *lam, unsigned long long *count, cudaStream_t s) {
  const unsigned blocks = persistent_blocks(d);
  Cam c = make_cam(*cam);
  if (d->storage == OF_TSDF_I16)
    k_integrate<OF_TSDF_I16, CENSUS><<<blocks, 256, 0, s>>>(
        (uint32_t *)vol, *d, c, depth, pitch, pose, (const float2 *)lam, count);
  else
    k_integrate<OF_TSDF_F16, CENSUS><<<blocks, 256, 0, s>>>(
        (uint32_t *)vol, *d, c, depth, pitch, pose, (const float2 *)lam, count);
  return of_launch_status();
}

// Launch of step 2 or 3 of of_integrate_tiled. Outside stream capture the
// kernel is launched programmatically: its blocks may start while the
// previous step's last blocks run and wait (griddepcontrol.wait) for that
// grid's results, which hides the launch gap between the steps. A captured
// step graph launches its nodes back to back already.
template <typename... P, typename... A>
cudaError_t launch_step(void (*k)(P...), unsigned grid, cudaStream_t s, A... args) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  // (a stream whose status cannot be read gets a plain launch)
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) cs = cudaStreamCaptureStatusActive;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(256);
  cfg.stream = s;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr.val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = cs == cudaStreamCaptureStatusNone ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, args...);
}

of_status_t launch_integrate_tiled(const of_volume_desc_t *d, void *vol, const of_camera_t *cam,
                                   const uint16_t *depth, int pitch, const double *pose,
                                   const float *lam, void *scratch, cudaStream_t s) {
  const ScratchLayout L = scratch_layout(d, cam);
  unsigned int *list_count = (unsigned int *)scratch;
  float2 *tiles = (float2 *)((char *)scratch + L.tiles);
  uint4 *list = (uint4 *)((char *)scratch + L.list);
  float2 *lmap = (float2 *)((char *)scratch + L.lmap);
  FrameSetup *setup = (FrameSetup *)((char *)scratch + L.setup);
  Cam c = make_cam(*cam);
  const int tx = tiles_x_of(cam), nt = tiles_of(cam);
  k_depth_tiles<<<(nt + 7) / 8, 256, 0, s>>>(c, depth, pitch, (const float2 *)lam, lmap, tiles, tx,
                                              nt, list_count, pose, *d, setup);
  const size_t nb = (size_t)(d->resolution / 8);
  const unsigned nbr = (unsigned)(nb * nb * nb);
  cudaError_t e = launch_step(k_classify_bricks, (nbr + 255) / 256, s, *d, c, (const double *)pose,
                              (const float2 *)tiles, tx,
                              (const uint8_t *)saturated_flags(vol, d->resolution), list,
                              list_count, (const FrameSetup *)setup);
  if (e != cudaSuccess) return of_set_cuda_error(e);
  const unsigned blocks = persistent_blocks(d);
  const uint16_t *dp = depth;
  const float2 *lp = (const float2 *)lam, *mp = lmap;
  const uint4 *li = list;
  const FrameSetup *su = setup;
  if (d->storage == OF_TSDF_I16)
    e = launch_step(k_integrate_list<OF_TSDF_I16>, blocks, s, (uint32_t *)vol, *d, c, dp, pitch,
                    pose, lp, mp, li, list_count, su);
  else
    e = launch_step(k_integrate_list<OF_TSDF_F16>, blocks, s, (uint32_t *)vol, *d, c, dp, pitch,
                    pose, lp, mp, li, list_count, su);
  if (e != cudaSuccess) return of_set_cuda_error(e);
  return of_launch_status();
}

// ---------------------------------------------------------------- batched --
// One stream of the batched of_integrate_tiled: its three steps run as three
// launches over all streams.
struct IntJob {
  uint32_t *vol;
  of_volume_desc_t desc;
  Cam cam;
  const uint16_t *depth[2];
  int pitch;
  const double *pose;
  const float2 *lam;
  float2 *tiles;
  uint4 *list;
  float2 *lmap;
  unsigned int *count;
  FrameSetup *setup;
  int tiles_x, ntiles;
};

__global__ void __launch_bounds__(256) k_depth_tiles_batch(const IntJob *__restrict__ jobs,
                                                           const int *__restrict__ first, int n,
                                                           int parity) {
  const int j = batch_job(first, n, blockIdx.x);
  const IntJob &J = jobs[j];
  depth_tiles_block(J.cam, J.depth[parity], J.pitch, J.lam, J.lmap, J.tiles, J.tiles_x, J.ntiles,
                    J.count, J.pose, J.desc, J.setup, blockIdx.x - __ldg(first + j));
}
__global__ void __launch_bounds__(256) k_classify_batch(const IntJob *__restrict__ jobs,
                                                        const int *__restrict__ first, int n) {
  const int j = batch_job(first, n, blockIdx.x);
  const IntJob &J = jobs[j];
  classify_block(J.desc, J.cam, J.tiles, J.tiles_x, saturated_flags(J.vol, J.desc.resolution),
                 J.list, J.count, J.setup, blockIdx.x - __ldg(first + j));
}
template <int STORAGE>
__global__ void __launch_bounds__(256, 4) k_integrate_list_batch(const IntJob *__restrict__ jobs,
                                                              const int *__restrict__ first, int n,
                                                              int parity) {
  const int j = batch_job(first, n, blockIdx.x);
  const IntJob &J = jobs[j];
  const int b0 = __ldg(first + j);
  integrate_list_block<STORAGE>(J.vol, J.desc, J.cam, J.depth[parity], J.pitch, J.lam, J.lmap,
                                J.list, J.count, J.setup, blockIdx.x - b0,
                                __ldg(first + j + 1) - b0);
}

// list_div candidates of the batched integration (blocks per stream =
// ceil(bricks / list_div), at most the single-stream persistent grid)
constexpr int kListDivs[] = {16, 32, 64, 128, 256};
constexpr int kNumListDivs = (int)(sizeof(kListDivs) / sizeof(kListDivs[0]));

}  // namespace

namespace of {

struct IntegrateBatch {
  int n = 0, storage = OF_TSDF_I16;
  IntJob *jobs = nullptr;
  int *tiles_first = nullptr, tiles_blocks = 0;
  int *classify_first = nullptr, classify_blocks = 0;
  int *list_first[kNumListDivs] = {}, list_blocks[kNumListDivs] = {};
};

void integrate_batch_destroy(IntegrateBatch *b) {
  if (!b) return;
  cudaFree(b->jobs);
  cudaFree(b->tiles_first);
  cudaFree(b->classify_first);
  for (int i = 0; i < kNumListDivs; ++i) cudaFree(b->list_first[i]);
  delete b;
}

int integrate_list_div(int knob) { return kListDivs[knob < 0 ? 0 : knob % kNumListDivs]; }

of_status_t integrate_batch_create(const BatchStream *s, int n, IntegrateBatch **out) {
  if (n < 1) return OF_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < n; ++i)
    if (s[i].vol_desc.storage != s[0].vol_desc.storage || !s[i].scratch ||
        ((uintptr_t)s[i].scratch & 255u))
      return OF_ERR_INVALID_ARGUMENT;
  IntegrateBatch *b = new IntegrateBatch();
  b->n = n;
  b->storage = s[0].vol_desc.storage;
  IntJob *jobs = new IntJob[n];
  int *ft = new int[n + 1], *fc = new int[n + 1], *fl = new int[n + 1];
  ft[0] = fc[0] = 0;
  for (int i = 0; i < n; ++i) {
    const ScratchLayout L = scratch_layout(&s[i].vol_desc, &s[i].cam);
    char *sc = (char *)s[i].scratch;
    IntJob &J = jobs[i];
    J.vol = (uint32_t *)s[i].volume;
    J.desc = s[i].vol_desc;
    J.cam = make_cam(s[i].cam);
    J.depth[0] = s[i].depth[0];
    J.depth[1] = s[i].depth[1];
    J.pitch = s[i].cam.width;
    J.pose = s[i].pose;
    J.lam = (const float2 *)s[i].lambda;
    J.tiles = (float2 *)(sc + L.tiles);
    J.list = (uint4 *)(sc + L.list);
    J.lmap = (float2 *)(sc + L.lmap);
    J.count = (unsigned int *)sc;
    J.setup = (FrameSetup *)(sc + L.setup);
    J.tiles_x = tiles_x_of(&s[i].cam);
    J.ntiles = tiles_of(&s[i].cam);
    const int nb = s[i].vol_desc.resolution / 8;
    ft[i + 1] = ft[i] + (J.ntiles + 7) / 8;
    fc[i + 1] = fc[i] + (nb * nb * nb + 255) / 256;
  }
  b->tiles_blocks = ft[n];
  b->classify_blocks = fc[n];
  of_status_t st = upload_jobs(jobs, ft, n, &b->jobs, &b->tiles_first);
  IntJob *tmp = nullptr;
  if (st == OF_OK) {
    st = upload_jobs(jobs, fc, n, &tmp, &b->classify_first);
    cudaFree(tmp);
  }
  for (int k = 0; k < kNumListDivs && st == OF_OK; ++k) {
    fl[0] = 0;
    for (int i = 0; i < n; ++i) {
      const size_t nb = (size_t)(s[i].vol_desc.resolution / 8);
      const size_t want = (nb * nb * nb + kListDivs[k] - 1) / kListDivs[k];
      const size_t cap = persistent_blocks(&s[i].vol_desc);
      fl[i + 1] = fl[i] + (int)(want < cap ? want : cap);
    }
    b->list_blocks[k] = fl[n];
    st = upload_jobs(jobs, fl, n, &tmp, &b->list_first[k]);
    cudaFree(tmp);
  }
  delete[] jobs;
  delete[] ft;
  delete[] fc;
  delete[] fl;
  if (st != OF_OK) {
    integrate_batch_destroy(b);
    return st;
  }
  *out = b;
  return OF_OK;
}

of_status_t integrate_batch_launch(const IntegrateBatch *b, int parity, const BatchKnobs &k,
                                   cudaStream_t s) {
  const int d = k.list_div < 0 ? 0 : k.list_div % kNumListDivs;
  k_depth_tiles_batch<<<b->tiles_blocks, 256, 0, s>>>(b->jobs, b->tiles_first, b->n, parity);
  k_classify_batch<<<b->classify_blocks, 256, 0, s>>>(b->jobs, b->classify_first, b->n);
  if (b->storage == OF_TSDF_I16)
    k_integrate_list_batch<OF_TSDF_I16><<<b->list_blocks[d], 256, 0, s>>>(b->jobs, b->list_first[d],
                                                                        b->n, parity);
  else
    k_integrate_list_batch<OF_TSDF_F16><<<b->list_blocks[d], 256, 0, s>>>(b->jobs, b->list_first[d],
                                                                        b->n, parity);
  return of_launch_status();
}

}  // namespace of

extern "C" of_status_t of_integrate(const of_volume_desc_t *d, void *vol, const of_camera_t *cam,
                                    const uint16_t *depth, int32_t pitch, const double *pose,
                                    const float *lam, of_stream_t s) {
  OF_RANGE("of_integrate");
  if (!of_volume_valid(d) || !of_camera_valid(cam) || !vol || !depth || !pose || !lam ||
      pitch < cam->width)
    return OF_ERR_INVALID_ARGUMENT;
  return launch_integrate<0>(d, vol, cam, depth, pitch, pose, lam, nullptr, (cudaStream_t)s);
}

extern "C" of_status_t of_integrate_scratch_bytes(const of_volume_desc_t *d,
                                                  const of_camera_t *cam, size_t *bytes) {
  if (!of_volume_valid(d) || !of_camera_valid(cam) || !bytes) return OF_ERR_INVALID_ARGUMENT;
  *bytes = scratch_layout(d, cam).total;
  return OF_OK;
}

extern "C" of_status_t of_integrate_tiled(const of_volume_desc_t *d, void *vol,
                                          const of_camera_t *cam, const uint16_t *depth,
                                          int32_t pitch, const double *pose, const float *lam,
                                          void *scratch, of_stream_t s) {
  OF_RANGE("of_integrate_tiled");
  if (!of_volume_valid(d) || !of_camera_valid(cam) || !vol || !depth || !pose || !lam ||
      !scratch || pitch < cam->width || ((uintptr_t)scratch & 255u))
    return OF_ERR_INVALID_ARGUMENT;
  return launch_integrate_tiled(d, vol, cam, depth, pitch, pose, lam, scratch, (cudaStream_t)s);
}

extern "C" of_status_t of_integrate_census(const of_volume_desc_t *d, const void *vol,
                                           const of_camera_t *cam, const uint16_t *depth,
                                           int32_t pitch, const double *pose, const float *lam,
                                           unsigned long long *count, of_stream_t s) {
  if (!of_volume_valid(d) || !of_camera_valid(cam) || !vol || !depth || !pose || !lam ||
      !count || pitch < cam->width)
    return OF_ERR_INVALID_ARGUMENT;
  return launch_integrate<kCensusUpdated>(d, (void *)vol, cam, depth, pitch, pose, lam, count,
                                (cudaStream_t)s);
}

extern "C" of_status_t of_integrate_visible_census(const of_volume_desc_t *d, const void *vol,
                                                   const of_camera_t *cam, const uint16_t *depth,
                                                   int32_t pitch, const double *pose,
                                                   const float *lam, unsigned long long *count,
                                                   of_stream_t s) {
  if (!of_volume_valid(d) || !of_camera_valid(cam) || !vol || !depth || !pose || !lam ||
      !count || pitch < cam->width)
    return OF_ERR_INVALID_ARGUMENT;
  return launch_integrate<kCensusVisible>(d, (void *)vol, cam, depth, pitch, pose, lam, count,
                                          (cudaStream_t)s);
}
