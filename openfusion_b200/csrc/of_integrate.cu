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

template <int STORAGE, bool CENSUS>
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
  const int lx = t >> 4, ly = (t >> 1) & 7, lz0 = (t & 1) * 4;
  const float T = desc.trunc_mm, inv_T = 1.0f / desc.trunc_mm;
  const float dspan = cam.dmax - cam.dmin;
  const unsigned uspan = (unsigned)(cam.w - 4), vspan = (unsigned)(cam.h - 4);
  const float vs = S.vs_hi;
  const float org = -0.5f * desc.size_mm;
  const float hext = 3.5f * vs + 1e-3f;  // half extent of a brick's voxel centres
  unsigned int my_count = 0;
  const float cxh = cam.cx + 0.5f, cyh = cam.cy + 0.5f;
  const float dlo = fmaxf(cam.dmin, 0.5f), dhi = cam.dmax;
  const int nb2 = nb * nb;
  uint8_t *flags = brick_flags(vol, desc.resolution);
  // Bricks are dealt round-robin (brick b goes to CTA b mod grid), so every
  // CTA gets a spatially spread, statistically equal share of the frustum.
  // Per batch, warp 0 tests 32 of the CTA's bricks (one lane each) and
  // compacts the visible ones into a shared list; the two 128-thread halves
  // then take list entries alternately.
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
      const int b = s_list[e][0], bx = s_list[e][1], by = s_list[e][2], bz = s_list[e][3];
      // camera-space centre of the brick's voxel (0,0,0), FP64 then rounded:
      // per-voxel offsets from it stay below 8 voxels, so the FP32 position
      // error is about one rounding of the brick base.
      const double fbx = (double)bx, fby = (double)by, fbz = (double)bz;
      const float BX = (float)fma(S.mb[0], fbx, fma(S.mb[1], fby, fma(S.mb[2], fbz, S.ob[0])));
      const float BY = (float)fma(S.mb[3], fbx, fma(S.mb[4], fby, fma(S.mb[5], fbz, S.ob[1])));
      const float BZ = (float)fma(S.mb[6], fbx, fma(S.mb[7], fby, fma(S.mb[8], fbz, S.ob[2])));
      float X0 = fmaf(S.m[0], (float)lx, fmaf(S.m[1], (float)ly, BX));
      float Y0 = fmaf(S.m[3], (float)lx, fmaf(S.m[4], (float)ly, BY));
      float Z0 = fmaf(S.m[6], (float)lx, fmaf(S.m[7], (float)ly, BZ));
      float tnew[4];
      unsigned upd = 0;
      bool near = false;
      // phase 1: project the four voxels; phase 2: issue every gather before
      // any result is used; phase 3: decide
      float Xv[4], Yv[4], Zv[4];
      int pix[4], dix[4];
      unsigned inb = 0;
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
        bool ok = (-Z - cam.dmin <= dspan) && (-Z >= cam.dmin) &&
                  (unsigned)(pu - 2) < uspan && (unsigned)(pv - 2) < vspan;
        inb |= ok ? (1u << m) : 0u;
        pix[m] = ok ? pv * cam.w + pu : 0;
        dix[m] = ok ? pv * pitch + pu : 0;
      }
      if (!inb) goto brick_done;
      {
        float Dv[4], Lh[4];
        bool have_xy = false;
        float2 sxy = make_float2(0.f, 0.f);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          // uint16 -> float without I2F: 2^23 + d is exact
          Dv[m] = __int_as_float(0x4B000000 | (int)__ldg(depth + dix[m])) - 8388608.0f;
          Lh[m] = __ldg(reinterpret_cast<const float *>(lam) + 2 * pix[m]);
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          tnew[m] = 0.f;
          const float D = Dv[m];
          if (!((inb >> m) & 1u) || !(D >= dlo && D <= dhi)) continue;
          const float X = Xv[m], Y = Yv[m], Z = Zv[m];
          // SDF = L - r with L = lambda D, r = |p_c|; decide on squares first
          float r2 = fmaf(X, X, fmaf(Y, Y, Z * Z));
          float L = Lh[m] * D;
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
            float llo = __ldg(reinterpret_cast<const float *>(lam) + 2 * pix[m] + 1);
            float2 Lp = two_prod(Lh[m], D);
            Lp.y = __fmaf_rn(llo, D, Lp.y);
            float sdf2 = __fadd_rn(__fsub_rn(Lp.x, rr.x), __fsub_rn(Lp.y, rr.y));
            if (sdf2 < -T) continue;
            sn = fminf(sdf2, T) * inv_T;
          }
          upd |= 1u << m;
          tnew[m] = sn;
        }
      }
    brick_done:
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
          // weight as float without I2F (2^23 + w is exact)
          float wf = __int_as_float(0x4B000000 | (int)wt) - 8388608.0f;
          float told = wt ? VoxelCodec<STORAGE>::tsdf(word) : 0.f;
          // (told w + tsdf') / (w + 1), within a few ulp of the rounded quotient
          float tn = __fdividef(__fmaf_rn(told, wf, tnew[m]), wf + 1.0f);
          uint32_t wn = min(wt + 1u, (uint32_t)desc.max_weight);
          w4[m] = VoxelCodec<STORAGE>::pack(tn, wn);
          near |= (w4[m] & 0xffffu) != VoxelCodec<STORAGE>::kOneBits;
        }
        *p4 = make_uint4(w4[0], w4[1], w4[2], w4[3]);
      }
      // a warp that wrote a non-saturated voxel flags the brick and its 26
      // neighbours (idempotent byte stores, lanes 0..26)
      if (!CENSUS && __any_sync(0xffffffffu, near) && lane < 27) {
        int ox = lane / 9 - 1, oy = (lane / 3) % 3 - 1, oz = lane % 3 - 1;
        int qx = bx + ox, qy = by + oy, qz = bz + oz;
        if ((unsigned)qx < (unsigned)nb && (unsigned)qy < (unsigned)nb && (unsigned)qz < (unsigned)nb)
          flags[(qx * nb + qy) * nb + qz] = 1;
      }
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

template <bool CENSUS>
of_status_t launch_integrate(const of_volume_desc_t *d, void *vol, const of_camera_t *cam,
                             const uint16_t *depth, int pitch, const double *pose,
                             const float *lam, unsigned long long *count, cudaStream_t s) {
  size_t nb = (size_t)(d->resolution / 8);
  size_t nbr = nb * nb * nb;
  // persistent grid: 4 resident CTAs of 256 threads per SM
  unsigned blocks = (unsigned)(nbr < (size_t)kSmCount * 4 ? nbr : (size_t)kSmCount * 4);
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
