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
// The SDF of voxels near the truncation band is evaluated with float-pair
// arithmetic so that the stored int16 value matches an FP64 evaluation to
// within one quantisation step.
#include "of_common.cuh"

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
  }
  S.vs_hi = (float)vs;
  S.vs_lo = (float)(vs - (double)S.vs_hi);
}

// |p_w - c| for voxel index (i, j, k) as a float pair.
__device__ __forceinline__ float2 voxel_range(const IntegrateSetup &S, int i, int j, int k) {
  float2 acc = make_float2(0.f, 0.f);
  const int idx[3] = {i, j, k};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float fi = (float)idx[a];
    float2 p = two_prod(fi, S.vs_hi);
    p.y = __fmaf_rn(fi, S.vs_lo, p.y);
    float2 q = two_sum(p.x, S.oc_hi[a]);
    float lo = __fadd_rn(__fadd_rn(p.y, q.y), S.oc_lo[a]);
    float2 dd = two_sum(q.x, lo);
    acc = df_add(acc, df_sq(dd.x, dd.y));
  }
  return df_sqrt(acc);
}

struct Plane {
  float a, b, c, d;  // inside <=> a X + b Y + c Z + d <= 0
};

template <int STORAGE, bool CENSUS>
__global__ void __launch_bounds__(256) k_integrate(uint32_t *__restrict__ vol, of_volume_desc_t desc,
                                                   Cam cam, const uint16_t *__restrict__ depth,
                                                   int pitch, const double *__restrict__ pose,
                                                   const float2 *__restrict__ lam,
                                                   unsigned long long *count) {
  __shared__ IntegrateSetup S;
  __shared__ Plane planes[6];
  __shared__ unsigned int s_count;
  if (threadIdx.x == 0) {
    make_setup(pose, desc, S);
    // frustum planes in camera space with half a pixel / 1 mm of slack; the
    // per-voxel test below is exact, this one only has to be conservative.
    float umin = 1.5f - 0.5f, umax = (float)cam.w - 2.5f + 0.5f;
    float vmin = 1.5f - 0.5f, vmax = (float)cam.h - 2.5f + 0.5f;
    planes[0] = {cam.fx, 0.f, cam.cx - umin, 0.f};
    planes[1] = {-cam.fx, 0.f, umax - cam.cx, 0.f};
    planes[2] = {0.f, cam.fy, cam.cy - vmin, 0.f};
    planes[3] = {0.f, -cam.fy, vmax - cam.cy, 0.f};
    planes[4] = {0.f, 0.f, 1.f, cam.dmin - 1.f};
    planes[5] = {0.f, 0.f, -1.f, -cam.dmax - 1.f};
    s_count = 0;
  }
  __syncthreads();
  const int nb = desc.resolution >> 3;
  const int nbricks = nb * nb * nb;
  const int half = threadIdx.x >> 7;
  const int t = threadIdx.x & 127;
  const int lane = threadIdx.x & 31;
  const int lx = t >> 4, ly = (t >> 1) & 7, lz0 = (t & 1) * 4;
  const float T = desc.trunc_mm, inv_T = 1.0f / desc.trunc_mm;
  const float dspan = cam.dmax - cam.dmin;
  const unsigned uspan = (unsigned)(cam.w - 4), vspan = (unsigned)(cam.h - 4);
  // brick b = 2 * pair + half walks the grid with a fixed stride; its (x, y, z)
  // brick coordinates advance by the stride's digits with carries.
  int b = 2 * blockIdx.x + half;
  const int stride = 2 * gridDim.x;
  const int sz = stride % nb, sy = (stride / nb) % nb, sx = stride / (nb * nb);
  int bz = b % nb, by = (b / nb) % nb, bx = b / (nb * nb);
  unsigned int my_count = 0;
  for (; b < nbricks; b += stride) {
    // camera-space centre of the brick's voxel (0,0,0), FP64 then rounded:
    // per-voxel offsets from it stay below 8 voxels, so the FP32 position
    // error is about one rounding of the brick base.
    const double fbx = (double)bx, fby = (double)by, fbz = (double)bz;
    const float BX = (float)fma(S.mb[0], fbx, fma(S.mb[1], fby, fma(S.mb[2], fbz, S.ob[0])));
    const float BY = (float)fma(S.mb[3], fbx, fma(S.mb[4], fby, fma(S.mb[5], fbz, S.ob[1])));
    const float BZ = (float)fma(S.mb[6], fbx, fma(S.mb[7], fby, fma(S.mb[8], fbz, S.ob[2])));
    const int cbx = bx, cby = by, cbz = bz;
    bz += sz; if (bz >= nb) { bz -= nb; ++by; }
    by += sy; if (by >= nb) { by -= nb; ++bx; }
    bx += sx;
    // ---- brick cull: lanes 0..7 take one corner voxel centre each
    bool culled = false;
    {
      float ci = (lane & 4) ? 7.f : 0.f, cj = (lane & 2) ? 7.f : 0.f, ck = (lane & 1) ? 7.f : 0.f;
      float X = fmaf(S.m[0], ci, fmaf(S.m[1], cj, fmaf(S.m[2], ck, BX)));
      float Y = fmaf(S.m[3], ci, fmaf(S.m[4], cj, fmaf(S.m[5], ck, BY)));
      float Z = fmaf(S.m[6], ci, fmaf(S.m[7], cj, fmaf(S.m[8], ck, BZ)));
#pragma unroll
      for (int p = 0; p < 6; ++p) {
        float e = planes[p].a * X + planes[p].b * Y + planes[p].c * Z + planes[p].d;
        unsigned out = __ballot_sync(0xffffffffu, e > 0.f) & 0xffu;
        culled |= (out == 0xffu);
      }
    }
    if (culled) continue;
    const int i = cbx * 8 + lx, j = cby * 8 + ly;
    float X0 = fmaf(S.m[0], (float)lx, fmaf(S.m[1], (float)ly, BX));
    float Y0 = fmaf(S.m[3], (float)lx, fmaf(S.m[4], (float)ly, BY));
    float Z0 = fmaf(S.m[6], (float)lx, fmaf(S.m[7], (float)ly, BZ));
    float tnew[4];
    unsigned upd = 0;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const float lz = (float)(lz0 + m);
      tnew[m] = 0.f;
      float X = fmaf(S.m[2], lz, X0);
      float Y = fmaf(S.m[5], lz, Y0);
      float Z = fmaf(S.m[8], lz, Z0);
      // -Z in [dmin, dmax] (and Z < 0): one unsigned-style range test
      if (!(-Z - cam.dmin <= dspan && -Z >= cam.dmin)) continue;
      float rz = __frcp_rn(Z);
      // roundFloat as floor(x + 0.5): identical except within one FP32 ulp of
      // a half-integer
      int pu = __float2int_rd(fmaf(cam.fx * X, rz, cam.cx) + 0.5f);
      int pv = __float2int_rd(fmaf(cam.fy * Y, rz, cam.cy) + 0.5f);
      if ((unsigned)(pu - 2) >= uspan || (unsigned)(pv - 2) >= vspan) continue;
      float D = (float)__ldg(depth + pv * pitch + pu);
      if (!(D - cam.dmin <= dspan && D >= cam.dmin && D > 0.f)) continue;
      float2 lm = __ldg(lam + pv * cam.w + pu);
      // SDF = L - r with L = lambda D, r = |p_c|; decide on squares first
      float r2 = fmaf(X, X, fmaf(Y, Y, Z * Z));
      float L = lm.x * D;
      const float slack = 0.05f + 1e-5f * L;
      float far = L + T + slack;            // SDF < -T - slack  <=>  r > far
      if (r2 > far * far) continue;
      float nearl = L - T - slack;          // SDF >  T + slack  <=>  r < nearl
      float sn;
      if (nearl > 0.f && r2 < nearl * nearl) {
        sn = 1.0f;
      } else {
        float2 rr = voxel_range(S, i, j, cbz * 8 + lz0 + m);
        float2 Lp = two_prod(lm.x, D);
        Lp.y = __fmaf_rn(lm.y, D, Lp.y);
        float sdf2 = __fadd_rn(__fsub_rn(Lp.x, rr.x), __fsub_rn(Lp.y, rr.y));
        if (sdf2 < -T) continue;
        sn = fminf(sdf2, T) * inv_T;
      }
      upd |= 1u << m;
      tnew[m] = sn;
    }
    if (CENSUS) {
      my_count += __popc(upd);
    } else if (upd) {
      uint4 *p4 = reinterpret_cast<uint4 *>(vol + ((size_t)b << 9)) + t;
      uint4 wv = *p4;
      uint32_t w4[4] = {wv.x, wv.y, wv.z, wv.w};
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        if (!(upd & (1u << m))) continue;
        uint32_t word = w4[m];
        uint32_t wt = word >> 16;
        float told = wt ? VoxelCodec<STORAGE>::tsdf(word) : 0.f;
        // (told w + tsdf') / (w + 1), within a few ulp of the rounded quotient
        float tn = __fdividef(__fmaf_rn(told, (float)wt, tnew[m]), (float)(wt + 1u));
        uint32_t wn = min(wt + 1u, (uint32_t)desc.max_weight);
        w4[m] = VoxelCodec<STORAGE>::pack(tn, wn);
      }
      *p4 = make_uint4(w4[0], w4[1], w4[2], w4[3]);
    }
  }
  if (CENSUS) {
    for (int o = 16; o > 0; o >>= 1) my_count += __shfl_xor_sync(0xffffffffu, my_count, o);
    if (lane == 0 && my_count) atomicAdd(&s_count, my_count);
    __syncthreads();
    if (threadIdx.x == 0 && s_count) atomicAdd(count, (unsigned long long)s_count);
  }
}

template <bool CENSUS>
of_status_t launch_integrate(const of_volume_desc_t *d, void *vol, const of_camera_t *cam,
                             const uint16_t *depth, int pitch, const double *pose,
                             const float *lam, unsigned long long *count, cudaStream_t s) {
  size_t nb = (size_t)(d->resolution / 8);
  size_t pairs = (nb * nb * nb + 1) / 2;
  // persistent grid: 8 resident CTAs of 256 threads per SM
  unsigned blocks = (unsigned)(pairs < (size_t)kSmCount * 8 ? pairs : (size_t)kSmCount * 8);
  Cam c = make_cam(*cam);
  if (d->storage == OF_TSDF_I16)
    k_integrate<OF_TSDF_I16, CENSUS><<<blocks, 256, 0, s>>>(
        (uint32_t *)vol, *d, c, depth, pitch, pose, (const float2 *)lam, count);
  else
    k_integrate<OF_TSDF_F16, CENSUS><<<blocks, 256, 0, s>>>(
        (uint32_t *)vol, *d, c, depth, pitch, pose, (const float2 *)lam, count);
  return of_launch_status();
}

}  // namespace

extern "C" of_status_t of_integrate(const of_volume_desc_t *d, void *vol, const of_camera_t *cam,
                                    const uint16_t *depth, int32_t pitch, const double *pose,
                                    const float *lam, of_stream_t s) {
  if (!of_volume_valid(d) || !of_camera_valid(cam) || !vol || !depth || !pose || !lam ||
      pitch < cam->width)
    return OF_ERR_INVALID_ARGUMENT;
  return launch_integrate<false>(d, vol, cam, depth, pitch, pose, lam, nullptr, (cudaStream_t)s);
}

extern "C" of_status_t of_integrate_census(const of_volume_desc_t *d, const void *vol,
                                           const of_camera_t *cam, const uint16_t *depth,
                                           int32_t pitch, const double *pose, const float *lam,
                                           unsigned long long *count, of_stream_t s) {
  if (!of_volume_valid(d) || !of_camera_valid(cam) || !vol || !depth || !pose || !lam ||
      !count || pitch < cam->width)
    return OF_ERR_INVALID_ARGUMENT;
  return launch_integrate<true>(d, (void *)vol, cam, depth, pitch, pose, lam, count,
                                (cudaStream_t)s);
}
