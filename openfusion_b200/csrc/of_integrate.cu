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
      acc += rba * (org - c[b]);
    }
    S.o[a] = (float)acc;
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
  const size_t nbricks = (size_t)nb * nb * nb;
  const int half = threadIdx.x >> 7;
  const int t = threadIdx.x & 127;
  const int lane = threadIdx.x & 31;
  const size_t b = (size_t)blockIdx.x * 2 + half;
  unsigned int my_count = 0;
  if (b < nbricks) {
    const int bz = (int)(b % nb);
    const int by = (int)((b / nb) % nb);
    const int bx = (int)(b / ((size_t)nb * nb));
    // ---- brick cull: lanes 0..7 take one corner voxel centre each
    bool culled = false;
    {
      int ci = bx * 8 + ((lane & 4) ? 7 : 0);
      int cj = by * 8 + ((lane & 2) ? 7 : 0);
      int ck = bz * 8 + ((lane & 1) ? 7 : 0);
      float X = fmaf(S.m[0], (float)ci, fmaf(S.m[1], (float)cj, fmaf(S.m[2], (float)ck, S.o[0])));
      float Y = fmaf(S.m[3], (float)ci, fmaf(S.m[4], (float)cj, fmaf(S.m[5], (float)ck, S.o[1])));
      float Z = fmaf(S.m[6], (float)ci, fmaf(S.m[7], (float)cj, fmaf(S.m[8], (float)ck, S.o[2])));
#pragma unroll
      for (int p = 0; p < 6; ++p) {
        float e = planes[p].a * X + planes[p].b * Y + planes[p].c * Z + planes[p].d;
        unsigned out = __ballot_sync(0xffffffffu, e > 0.f) & 0xffu;
        culled |= (out == 0xffu);
      }
    }
    if (!culled) {
      const int lx = t >> 4, ly = (t >> 1) & 7, lz0 = (t & 1) * 4;
      const int i = bx * 8 + lx, j = by * 8 + ly;
      float X0 = fmaf(S.m[0], (float)i, fmaf(S.m[1], (float)j, S.o[0]));
      float Y0 = fmaf(S.m[3], (float)i, fmaf(S.m[4], (float)j, S.o[1]));
      float Z0 = fmaf(S.m[6], (float)i, fmaf(S.m[7], (float)j, S.o[2]));
      float tnew[4];
      bool upd[4];
      bool any = false;
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int k = bz * 8 + lz0 + m;
        upd[m] = false;
        tnew[m] = 0.f;
        float X = fmaf(S.m[2], (float)k, X0);
        float Y = fmaf(S.m[5], (float)k, Y0);
        float Z = fmaf(S.m[8], (float)k, Z0);
        if (!(Z < 0.f) || -Z < cam.dmin || -Z > cam.dmax) continue;
        float rz = __frcp_rn(Z);
        float uf = fmaf(cam.fx * X, rz, cam.cx);
        float vf = fmaf(cam.fy * Y, rz, cam.cy);
        int pu = round_ref(uf), pv = round_ref(vf);
        if (pu < 2 || pu >= cam.w - 2 || pv < 2 || pv >= cam.h - 2) continue;
        float D = (float)__ldg(depth + (size_t)pv * pitch + pu);
        if (!(D > 0.f && D >= cam.dmin && D <= cam.dmax)) continue;
        float2 lm = __ldg(lam + (size_t)pv * cam.w + pu);
        float r = sqrtf(fmaf(X, X, fmaf(Y, Y, Z * Z)));
        float sdf = fmaf(lm.x, D, -r);
        const float slack = 0.05f + 1e-5f * r;
        if (sdf < -desc.trunc_mm - slack) continue;
        float sn;
        if (sdf > desc.trunc_mm + slack) {
          sn = 1.0f;
        } else {
          float2 rr = voxel_range(S, i, j, k);
          float2 L = two_prod(lm.x, D);
          L.y = __fmaf_rn(lm.y, D, L.y);
          float sdf2 = __fadd_rn(__fsub_rn(L.x, rr.x), __fsub_rn(L.y, rr.y));
          if (sdf2 < -desc.trunc_mm) continue;
          sn = __fdiv_rn(fminf(sdf2, desc.trunc_mm), desc.trunc_mm);
        }
        upd[m] = true;
        tnew[m] = sn;
        any = true;
      }
      if (CENSUS) {
        my_count = (unsigned)upd[0] + (unsigned)upd[1] + (unsigned)upd[2] + (unsigned)upd[3];
      } else if (any) {
        uint4 *p4 = reinterpret_cast<uint4 *>(vol + (b << 9)) + t;
        uint4 wv = *p4;
        uint32_t w4[4] = {wv.x, wv.y, wv.z, wv.w};
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          if (!upd[m]) continue;
          uint32_t word = w4[m];
          uint32_t wt = word >> 16;
          float told = wt ? VoxelCodec<STORAGE>::tsdf(word) : 0.f;
          float tn = __fdiv_rn(__fmaf_rn(told, (float)wt, tnew[m]), (float)(wt + 1u));
          uint32_t wn = min(wt + 1u, (uint32_t)desc.max_weight);
          w4[m] = VoxelCodec<STORAGE>::pack(tn, wn);
        }
        *p4 = make_uint4(w4[0], w4[1], w4[2], w4[3]);
      }
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
  size_t nbricks = nb * nb * nb;
  unsigned blocks = (unsigned)((nbricks + 1) / 2);
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
