// of_raycast.cuh -- the per-ray device code of the raycast, shared by the
// single-stream and the batched raycast launches (of_raycast.cu).
//
// Follows d_raycast (Source/src/Raycaster.cu:97-230): one ray per pixel from
// the camera position through the pixel's point at z = -1 in camera space
// (:117-125), clipped to the cube with a slab test (:35-55, here the box of
// voxel centres), marched until the first surface, writing the world-space
// vertex and normal maps (:202-212) and optionally the shaded RGBA of
// :214-228. Where the reference samples the nearest voxel at fixed 1.5 mm
// steps and stops at the first tsdf <= 0 (:152-188), this follows the
// KinectFusion method the reference left commented out (:246-351): trilinear
// samples, steps of max(min_step, far_frac * tsdf * trunc), a + to - zero
// crossing whose bracket is first narrowed to one minimum step and then refined
// by Illinois regula falsi on the trilinear field, and the normal as
// the central-difference gradient of trilinear samples one voxel apart. The
// march runs between the min and max depth along the ray.
#pragma once

#include "of_batch.cuh"

using namespace of;

namespace {

struct RaySetup {
  Rigid c2w;
  float cpos[3];
  float lo, hi;   // box of voxel centres, mm (same for every axis)
  float inv_vs;
};

// Stored tsdf of a voxel word, in storage units: q for int16 (q / 32767 is
// the normalised tsdf), the value itself for fp16. An unobserved voxel
// (weight 0) holds the +1 pattern (the reset and import write it), so no
// weight test is needed. int16 by an integer-to-float conversion (exact):
// the raycast's integer/logic pipe is its busiest (57 % at C2) and the
// conversion pipe its idlest (12 %), so the conversion beats the
// mask-and-add form that runs one logic operation per corner (raycast
// stage 115.1 -> 111.8 us, the same bits).
template <int STORAGE>
__device__ __forceinline__ float ray_value(uint32_t w) {
  if (STORAGE == OF_TSDF_I16)
    return __int2float_rn((int)(short)(w & 0xffffu));
  else
    return __half2float(__ushort_as_half((unsigned short)(w & 0xffffu)));
}
template <int STORAGE>
constexpr float ray_scale() {
  return STORAGE == OF_TSDF_I16 ? 1.0f / kQ : 1.0f;
}

// floor(g) clamped to [0, n-2]: the unsigned conversion saturates negative
// values (and NaN) to 0 itself, which leaves one integer min.
__device__ __forceinline__ int cell_index(float g, int n) {
  return (int)min(__float2uint_rd(g), (unsigned)(n - 2));
}

// Trilinear tsdf at a world position. Corner (i0, j0, k0) is clamped to
// [0, n-2]; the seven other corners are the base address plus an axis step
// that crosses into the next brick when the local coordinate is 7. Volume
// indices fit in 32 bits (n <= 1024).
template <int STORAGE>
__device__ __forceinline__ float trilinear(const uint32_t *__restrict__ vol, int n, int nb,
                                           float org, float inv_vs, float px, float py, float pz,
                                           int3 *cell = nullptr) {
  float gx = fmaf(px - org, inv_vs, -0.5f);
  float gy = fmaf(py - org, inv_vs, -0.5f);
  float gz = fmaf(pz - org, inv_vs, -0.5f);
  int ix = cell_index(gx, n), iy = cell_index(gy, n), iz = cell_index(gz, n);
  float fx = gx - (float)ix, fy = gy - (float)iy, fz = gz - (float)iz;
  if (cell) *cell = make_int3(ix, iy, iz);
  unsigned base = ((((unsigned)(ix >> 3) * nb + (unsigned)(iy >> 3)) * nb + (unsigned)(iz >> 3)) << 9) |
                  (unsigned)(((ix & 7) << 6) | ((iy & 7) << 3) | (iz & 7));
  unsigned dx = (ix & 7) == 7 ? (unsigned)nb * nb * 512u - 448u : 64u;
  unsigned dy = (iy & 7) == 7 ? (unsigned)nb * 512u - 56u : 8u;
  unsigned dz = (iz & 7) == 7 ? 505u : 1u;
  const uint32_t *p0 = vol + base;
  float c000 = ray_value<STORAGE>(__ldg(p0));
  float c001 = ray_value<STORAGE>(__ldg(p0 + dz));
  float c010 = ray_value<STORAGE>(__ldg(p0 + dy));
  float c011 = ray_value<STORAGE>(__ldg(p0 + dy + dz));
  float c100 = ray_value<STORAGE>(__ldg(p0 + dx));
  float c101 = ray_value<STORAGE>(__ldg(p0 + dx + dz));
  float c110 = ray_value<STORAGE>(__ldg(p0 + dx + dy));
  float c111 = ray_value<STORAGE>(__ldg(p0 + dx + dy + dz));
  float c00 = fmaf(fz, c001 - c000, c000);
  float c01 = fmaf(fz, c011 - c010, c010);
  float c10 = fmaf(fz, c101 - c100, c100);
  float c11 = fmaf(fz, c111 - c110, c110);
  float c0 = fmaf(fy, c01 - c00, c00);
  float c1 = fmaf(fy, c11 - c10, c10);
  return fmaf(fx, c1 - c0, c0) * ray_scale<STORAGE>();
}

// Central differences of the trilinear field one voxel apart along each axis
// at p: (f(p + vs e_a) - f(p - vs e_a)) for a = x, y, z. The six samples take
// p's cell fractions (equal to their own up to FP32 rounding of the shifted
// position), so their 48 corner reads come from the 32 voxels of p's cell
// widened by one voxel along each axis in turn. Each sample is interpolated
// in trilinear()'s order (z, then y, then x). p's cell base must lie in
// [1, n-3] on every axis (the caller keeps p one voxel inside the box).
template <int STORAGE>
__device__ __forceinline__ float3 central_gradient(const uint32_t *__restrict__ vol, int n, int nb,
                                                   float org, float inv_vs, float px, float py,
                                                   float pz) {
  const float gx = fmaf(px - org, inv_vs, -0.5f);
  const float gy = fmaf(py - org, inv_vs, -0.5f);
  const float gz = fmaf(pz - org, inv_vs, -0.5f);
  const int ix = min(max(__float2int_rd(gx), 1), n - 3);
  const int iy = min(max(__float2int_rd(gy), 1), n - 3);
  const int iz = min(max(__float2int_rd(gz), 1), n - 3);
  const float fx = gx - (float)ix, fy = gy - (float)iy, fz = gz - (float)iz;
  // word offset of index i-1 .. i+2 along each axis (brick part + local part)
  unsigned ox[4], oy[4], oz[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const unsigned a = (unsigned)(ix - 1 + k), b = (unsigned)(iy - 1 + k), c = (unsigned)(iz - 1 + k);
    ox[k] = (((a >> 3) * (unsigned)nb * (unsigned)nb) << 9) + ((a & 7u) << 6);
    oy[k] = (((b >> 3) * (unsigned)nb) << 9) + ((b & 7u) << 3);
    oz[k] = ((c >> 3) << 9) + (c & 7u);
  }
  auto v = [&](int kx, int ky, int kz) {
    return ray_value<STORAGE>(__ldg(vol + ox[kx] + oy[ky] + oz[kz]));
  };
  auto lerp = [](float a, float b, float f) { return fmaf(f, b - a, a); };
  // z-interpolated rows at x = kx, y = ky, over the cell's own z pair (1, 2)
  float Lz[4][4];
#pragma unroll
  for (int kx = 0; kx < 4; ++kx)
#pragma unroll
    for (int ky = 0; ky < 4; ++ky) {
      const bool need = (ky == 1 || ky == 2) || (kx == 1 || kx == 2);
      Lz[kx][ky] = need ? lerp(v(kx, ky, 1), v(kx, ky, 2), fz) : 0.f;
    }
  // x: cells (ix - 1) and (ix + 1)
  const float xm = lerp(lerp(Lz[0][1], Lz[0][2], fy), lerp(Lz[1][1], Lz[1][2], fy), fx);
  const float xp = lerp(lerp(Lz[2][1], Lz[2][2], fy), lerp(Lz[3][1], Lz[3][2], fy), fx);
  // y: cells (iy - 1) and (iy + 1)
  const float ym = lerp(lerp(Lz[1][0], Lz[1][1], fy), lerp(Lz[2][0], Lz[2][1], fy), fx);
  const float yp = lerp(lerp(Lz[1][2], Lz[1][3], fy), lerp(Lz[2][2], Lz[2][3], fy), fx);
  // z: cells (iz - 1) and (iz + 1), over the cell's own x and y pairs
  float zm, zp;
  {
    const float m11 = lerp(v(1, 1, 0), v(1, 1, 1), fz), m12 = lerp(v(1, 2, 0), v(1, 2, 1), fz);
    const float m21 = lerp(v(2, 1, 0), v(2, 1, 1), fz), m22 = lerp(v(2, 2, 0), v(2, 2, 1), fz);
    const float p11 = lerp(v(1, 1, 2), v(1, 1, 3), fz), p12 = lerp(v(1, 2, 2), v(1, 2, 3), fz);
    const float p21 = lerp(v(2, 1, 2), v(2, 1, 3), fz), p22 = lerp(v(2, 2, 2), v(2, 2, 3), fz);
    zm = lerp(lerp(m11, m12, fy), lerp(m21, m22, fy), fx);
    zp = lerp(lerp(p11, p12, fy), lerp(p21, p22, fy), fx);
  }
  const float sc = ray_scale<STORAGE>();
  return make_float3(xp * sc - xm * sc, yp * sc - ym * sc, zp * sc - zm * sc);
}

__device__ __forceinline__ uint32_t rgba_pack(float x, float y, float z, float w) {
  // rgbaFloatToInt (Raycaster.cu:26-33)
  x = __saturatef(x); y = __saturatef(y); z = __saturatef(z); w = __saturatef(w);
  return ((uint32_t)(w * 255.f) << 24) | ((uint32_t)(z * 255.f) << 16) |
         ((uint32_t)(y * 255.f) << 8) | (uint32_t)(x * 255.f);
}

// Levels 1 .. levels-1 of the model pyramid written by the raycast itself:
// pixel (x, y) of level l is the ray of level-0 pixel (2^l x, 2^l y), the
// value the chain of 2x subsamplings (k_model_down) gives.
struct ModelLevels {
  float4 *pts[kMaxLevels];
  int w[kMaxLevels];
  int levels;
};

// (out of line: the kernel keeps its registers for the march)
__device__ __noinline__ void write_coarse(const ModelLevels &coarse, int x, int y, float4 vtx,
                                          float4 nrm) {
  for (int l = 1; l < coarse.levels; ++l) {
    const int m = (1 << l) - 1;
    if ((x & m) | (y & m)) break;
    const size_t q = (size_t)(y >> l) * coarse.w[l] + (x >> l);
    coarse.pts[l][2 * q] = vtx;
    coarse.pts[l][2 * q + 1] = nrm;
  }
}

// The per-launch constants of a raycast at `pose` (one thread computes them).
__device__ __forceinline__ void ray_setup(const double *__restrict__ pose,
                                          const of_volume_desc_t &desc, RaySetup *S) {
  pose_to_rigid(pose, &S->c2w, nullptr);
  S->cpos[0] = S->c2w.t[0]; S->cpos[1] = S->c2w.t[1]; S->cpos[2] = S->c2w.t[2];
  double vs = (double)desc.size_mm / desc.resolution;
  S->lo = (float)(-0.5 * desc.size_mm + 0.5 * vs + 1e-3);
  S->hi = (float)(0.5 * desc.size_mm - 0.5 * vs - 1e-3);
  S->inv_vs = (float)(1.0 / vs);
}

// The ray of pixel (x, y), inside the image: march, refine, normal; writes
// the pixel's model point (and the coarser levels' where (x, y) is one of
// theirs) and the shaded RGBA when `rgba` is given.
template <int STORAGE>
__device__ __forceinline__ void raycast_pixel(const uint32_t *__restrict__ vol,
                                              const of_volume_desc_t &desc, const Cam &cam,
                                              const of_raycast_params_t &rp, const RaySetup &S,
                                              int x, int y, float4 *__restrict__ pts,
                                              uint32_t *rgba, const ModelLevels *coarse) {
  const int n = desc.resolution, nb = n >> 3;
  const float vs = desc.size_mm / (float)n;
  const float org = -0.5f * desc.size_mm;
  const float T = desc.trunc_mm;
  // ray direction: pixel at z = -1 (Raycaster.cu:117-125)
  float3 dc = make_float3(-((float)x - cam.cx) * cam.ifx, -((float)y - cam.cy) * cam.ify, -1.f);
  float lam = sqrtf(dc.x * dc.x + dc.y * dc.y + 1.f);
  float3 dw = rotate(S.c2w, dc);
  float il = 1.f / lam;
  float3 dir = make_float3(dw.x * il, dw.y * il, dw.z * il);
  const float ox = S.cpos[0], oy = S.cpos[1], oz = S.cpos[2];
  // slab test (Raycaster.cu:35-55) against the box of voxel centres
  float tnear = -1e30f, tfar = 1e30f;
  {
    const float o3[3] = {ox, oy, oz};
    const float d3[3] = {dir.x, dir.y, dir.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (fabsf(d3[a]) < 1e-12f) {
        if (o3[a] < S.lo || o3[a] > S.hi) { tnear = 1e30f; tfar = -1e30f; }
      } else {
        float inv = 1.f / d3[a];
        float t0 = (S.lo - o3[a]) * inv, t1 = (S.hi - o3[a]) * inv;
        tnear = fmaxf(tnear, fminf(t0, t1));
        tfar = fminf(tfar, fmaxf(t0, t1));
      }
    }
  }
  float t0 = fmaxf(tnear, cam.dmin * lam);
  float t1 = fminf(tfar, cam.dmax * lam);
  bool hit = false;
  float ts = 0.f;
  if (t0 < t1) {
    const float min_step = rp.min_step_vox * vs;
    const float far_k = rp.far_step_frac * T;
    const uint8_t *__restrict__ flags = brick_flags((void *)vol, n);
    const float inv_vs = S.inv_vs;
    const float eps = 0.01f * vs;
    const uint8_t *__restrict__ sflags = super_flags((void *)vol, n);
    const int ns = super_count(n);
    // per-axis reciprocal of the direction (0 where the ray is parallel to
    // the axis planes: that axis bounds no jump)
    const bool ux = fabsf(dir.x) > 1e-12f, uy = fabsf(dir.y) > 1e-12f, uz = fabsf(dir.z) > 1e-12f;
    const float rdx = ux ? 1.0f / dir.x : 0.f, rdy = uy ? 1.0f / dir.y : 0.f, rdz = uz ? 1.0f / dir.z : 0.f;
    float t = t0;
    float fp = 1.0f;
    bool sampled = false;
    int cur_b = -1, cur_s = -1;  // brick / super-brick the march is in, and their flags
    bool cur_flag = false, cur_sflag = false;
    // the clamped cell base of the position at t when the last sample was
    // taken there (the same expression as below, so the same brick)
    int3 cell = make_int3(0, 0, 0);
    bool have_cell = false;
    for (int it = 0; it < (1 << 16); ++it) {
      if (!have_cell) {
        const float px = fmaf(t, dir.x, ox), py = fmaf(t, dir.y, oy), pz = fmaf(t, dir.z, oz);
        cell.x = cell_index(fmaf(px - org, inv_vs, -0.5f), n);
        cell.y = cell_index(fmaf(py - org, inv_vs, -0.5f), n);
        cell.z = cell_index(fmaf(pz - org, inv_vs, -0.5f), n);
      }
      have_cell = false;
      const int bi = cell.x >> 3, bj = cell.y >> 3, bk = cell.z >> 3;
      // (cell indices are clamped to >= 0: unsigned division is a shift)
      const int si = (int)((unsigned)bi / kSuper), sj = (int)((unsigned)bj / kSuper),
                sk = (int)((unsigned)bk / kSuper);
      const int sidx = (si * ns + sj) * ns + sk;
      if (sidx != cur_s) {
        cur_s = sidx;
        cur_sflag = __ldg(sflags + sidx) != 0;
      }
      bool skip = !cur_sflag;
      if (!skip) {
        const int b = (bi * nb + bj) * nb + bk;
        if (b != cur_b) {
          cur_b = b;
          cur_flag = __ldg(flags + b) != 0;
        }
        skip = !cur_flag;
      }
      if (skip) {
        // every sample with its cell base in this brick (or, when the
        // super-brick's flag is clear, in this super-brick) reads exactly +1:
        // jump just past the region; the landing cell is +1 as well. The
        // region of cell bases [8b, 8b + 8) along an axis is
        // p in [org + vs (8b + 0.5), org + vs (8b + 8.5)); R = 32 for a
        // super-brick.
        const float R = cur_sflag ? 8.0f : (float)(8 * kSuper);
        const int ci = cur_sflag ? bi : si, cj = cur_sflag ? bj : sj, ck = cur_sflag ? bk : sk;
        const float rvs = R * vs, h = org + 0.5f * vs;
        float te = 1e30f;
        if (ux) te = fminf(te, (fmaf(rvs, (float)(dir.x > 0.f ? ci + 1 : ci), h) - ox) * rdx);
        if (uy) te = fminf(te, (fmaf(rvs, (float)(dir.y > 0.f ? cj + 1 : cj), h) - oy) * rdy);
        if (uz) te = fminf(te, (fmaf(rvs, (float)(dir.z > 0.f ? ck + 1 : ck), h) - oz) * rdz);
        t = fmaxf(te, t) + eps;
        fp = 1.0f;
        sampled = true;
        if (t > t1) break;
        continue;
      }
      if (!sampled) {
        fp = trilinear<STORAGE>(vol, n, nb, org, inv_vs, fmaf(t, dir.x, ox), fmaf(t, dir.y, oy),
                                fmaf(t, dir.z, oz));
        sampled = true;
      }
      float step = fp > 0.f ? fmaxf(min_step, far_k * fp) : min_step;
      float tn = t + step;
      if (tn > t1) break;
      float fn = trilinear<STORAGE>(vol, n, nb, org, inv_vs, fmaf(tn, dir.x, ox),
                                    fmaf(tn, dir.y, oy), fmaf(tn, dir.z, oz), &cell);
      if (fp > 0.f && fn <= 0.f) {
        float ta = t, fa = fp, tb = tn, fb = fn;
        // shrink a long bracket with minimum steps from its positive end, so
        // the refined root does not depend on where the march samples fell
        while (tb - ta > min_step * 1.0001f) {
          float tm = ta + min_step;
          float fm = trilinear<STORAGE>(vol, n, nb, org, inv_vs, fmaf(tm, dir.x, ox),
                                        fmaf(tm, dir.y, oy), fmaf(tm, dir.z, oz));
          if (fm > 0.f) { ta = tm; fa = fm; } else { tb = tm; fb = fm; break; }
        }
        // Illinois regula falsi on the trilinear field
        int side = 0;
        for (int r = 0; r < rp.refine_iters; ++r) {
          float tm = fmaf(tb - ta, fa / (fa - fb), ta);
          float fm = trilinear<STORAGE>(vol, n, nb, org, inv_vs, fmaf(tm, dir.x, ox),
                                        fmaf(tm, dir.y, oy), fmaf(tm, dir.z, oz));
          if (fm > 0.f) {
            ta = tm; fa = fm;
            if (side == 1) fb *= 0.5f;
            side = 1;
          } else {
            tb = tm; fb = fm;
            if (side == -1) fa *= 0.5f;
            side = -1;
          }
        }
        ts = fmaf(tb - ta, fa / (fa - fb), ta);
        hit = true;
        break;
      }
      if (fp < 0.f && fn > 0.f) break;  // back face
      t = tn;
      fp = fn;
      have_cell = true;
    }
  }
  const size_t p = (size_t)y * cam.w + x;
  float4 vtx = make_float4(0.f, 0.f, 0.f, 0.f), nrm = make_float4(0.f, 0.f, 0.f, 0.f);
  if (hit) {
    float px = fmaf(ts, dir.x, ox), py = fmaf(ts, dir.y, oy), pz = fmaf(ts, dir.z, oz);
    vtx = make_float4(px, py, pz, 1.f);
    float lo = S.lo, hi = S.hi;
    if (px - vs >= lo && px + vs <= hi && py - vs >= lo && py + vs <= hi && pz - vs >= lo &&
        pz + vs <= hi) {
      const float3 g = central_gradient<STORAGE>(vol, n, nb, org, S.inv_vs, px, py, pz);
      const float gx = g.x, gy = g.y, gz = g.z;
      float l2 = gx * gx + gy * gy + gz * gz;
      if (l2 > 0.f) {
        float inv = rsqrtf(l2);
        inv = inv * (1.5f - 0.5f * l2 * inv * inv);
        nrm = make_float4(gx * inv, gy * inv, gz * inv, 1.f);
      }
    }
  }
  pts[2 * p] = vtx;
  pts[2 * p + 1] = nrm;
  if (coarse && ((x | y) & 1) == 0) write_coarse(*coarse, x, y, vtx, nrm);
  if (rgba) {
    // shaded output of Raycaster.cu:221-227 (showNormal == false)
    float dd = -(dir.x * nrm.x + dir.y * nrm.y + dir.z * nrm.z);
    float g = fabsf(dd) < 1e-6f ? 0.f : 0.6f * dd + 0.2f;
    rgba[p] = fabsf(dd) < 1e-6f ? rgba_pack(0.f, 0.f, 0.f, 0.f) : rgba_pack(g, g, g, 0.f);
  }
}

// One block of pixels (bx, by) with the block's own setup.
template <int STORAGE>
__device__ __forceinline__ void raycast_tile(const uint32_t *__restrict__ vol,
                                             const of_volume_desc_t &desc, const Cam &cam,
                                             const of_raycast_params_t &rp,
                                             const double *__restrict__ pose,
                                             float4 *__restrict__ pts, uint32_t *rgba, int bx,
                                             int by, const ModelLevels *coarse = nullptr) {
  __shared__ RaySetup S;
  if (threadIdx.x == 0 && threadIdx.y == 0) ray_setup(pose, desc, &S);
  __syncthreads();
  const int x = bx * blockDim.x + threadIdx.x;
  const int y = by * blockDim.y + threadIdx.y;
  if (x >= cam.w || y >= cam.h) return;
  raycast_pixel<STORAGE>(vol, desc, cam, rp, S, x, y, pts, rgba, coarse);
}

}  // namespace
