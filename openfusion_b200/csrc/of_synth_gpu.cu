// of_synth_gpu.cu -- the seeded synthetic depth renderer of of_synth.cpp on
// the device, for generating training and evaluation sequences at GPU speed.
//
// Same scenes (of_synth_scene_t, built on the host by of_synth_scene), same
// ray/primitive intersections in FP64, same counter-based noise and dropout
// hashes; one thread per pixel, many frames per launch. The host renderer
// calls the host libm and this one CUDA's FP64 sqrt/log/cos, so a depth can
// differ by 1 mm where a noisy depth lies within rounding of a half
// millimetre.
#include "of_common.cuh"
#include "of_synth.h"

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ uint64_t hash3(uint64_t a, uint64_t b, uint64_t c) {
  return mix64(a ^ mix64(b ^ mix64(c)));
}
__device__ __forceinline__ double unit01(uint64_t h) {
  return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

// Ray parameter of the first hit of o + t d with a primitive (t > 1e-6), or -1.
__device__ double hit_prim(const of_synth_prim_t &p, double3 o, double3 d) {
  const double eps = 1e-6;
  if (p.kind == OF_PRIM_PLANE) {
    const double den = p.p[0] * d.x + p.p[1] * d.y + p.p[2] * d.z;
    if (fabs(den) < 1e-12) return -1.0;
    const double t = (p.p[3] - (p.p[0] * o.x + p.p[1] * o.y + p.p[2] * o.z)) / den;
    return t > eps ? t : -1.0;
  }
  if (p.kind == OF_PRIM_SPHERE) {
    const double3 oc = make_double3(o.x - p.p[0], o.y - p.p[1], o.z - p.p[2]);
    const double r = p.p[3];
    const double a = d.x * d.x + d.y * d.y + d.z * d.z;
    const double b = oc.x * d.x + oc.y * d.y + oc.z * d.z;
    const double cc = oc.x * oc.x + oc.y * oc.y + oc.z * oc.z - r * r;
    const double disc = b * b - a * cc;
    if (disc < 0.0) return -1.0;
    const double sq = sqrt(disc);
    double t = (-b - sq) / a;
    if (t > eps) return t;
    t = (-b + sq) / a;
    return t > eps ? t : -1.0;
  }
  // box with yaw about +y
  const double cy = cos((double)p.p[6]), sy = sin((double)p.p[6]);
  const double3 ol = make_double3(o.x - p.p[0], o.y - p.p[1], o.z - p.p[2]);
  const double lo[3] = {cy * ol.x - sy * ol.z, ol.y, sy * ol.x + cy * ol.z};
  const double ld[3] = {cy * d.x - sy * d.z, d.y, sy * d.x + cy * d.z};
  const double h[3] = {p.p[3], p.p[4], p.p[5]};
  double tn = -1e300, tf = 1e300;
  for (int a = 0; a < 3; ++a) {
    if (fabs(ld[a]) < 1e-15) {
      if (lo[a] < -h[a] || lo[a] > h[a]) return -1.0;
      continue;
    }
    double t0 = (-h[a] - lo[a]) / ld[a], t1 = (h[a] - lo[a]) / ld[a];
    if (t0 > t1) { const double q = t0; t0 = t1; t1 = q; }
    tn = fmax(tn, t0);
    tf = fmin(tf, t1);
  }
  if (tn > tf) return -1.0;
  if (tn > eps) return tn;
  return tf > eps ? tf : -1.0;
}

__global__ void __launch_bounds__(256) k_synth_render(const of_synth_scene_t *__restrict__ scene,
                                                      int w, int h, float fx, float fy, float cx,
                                                      float cy, const double *__restrict__ poses,
                                                      uint64_t noise_seed, int first_frame,
                                                      float sigma_scale, float dropout,
                                                      uint16_t *__restrict__ depth) {
  __shared__ of_synth_prim_t s_prims[OF_SYNTH_MAX_PRIMS];
  __shared__ int s_count;
  const int f = blockIdx.z;
  if (threadIdx.x == 0) s_count = scene->count;
  for (int i = threadIdx.x; i < OF_SYNTH_MAX_PRIMS; i += blockDim.x) s_prims[i] = scene->prims[i];
  __syncthreads();
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  const int u = px % w, v = px / w;
  if (v >= h || blockIdx.y != 0) return;
  const double *P = poses + 16 * (size_t)f;
  const double3 o = make_double3(P[3], P[7], P[11]);
  const double dcx = -((double)u - cx) / fx, dcy = -((double)v - cy) / fy;
  const double3 d = make_double3(P[0] * dcx + P[1] * dcy - P[2], P[4] * dcx + P[5] * dcy - P[6],
                                 P[8] * dcx + P[9] * dcy - P[10]);
  double best = -1.0;
  for (int i = 0; i < s_count; ++i) {
    const double t = hit_prim(s_prims[i], o, d);
    if (t > 0.0 && (best < 0.0 || t < best)) best = t;
  }
  const size_t p = (size_t)v * w + u;
  uint16_t out = 0;
  if (best > 0.0 && best < 10000.0) {
    const uint64_t hh = hash3(noise_seed, (uint64_t)(first_frame + f), (uint64_t)p);
    const double u1 = unit01(mix64(hh ^ 1)), u2 = unit01(mix64(hh ^ 2)), u3 = unit01(mix64(hh ^ 3));
    const double zm = best * 1e-3 - 0.4;
    const double sigma = 1000.0 * (0.0012 + 0.0019 * zm * zm) * sigma_scale;
    const double g = sqrt(-2.0 * log(u1)) * cos(2.0 * 3.14159265358979323846 * u2);
    double dn = floor(best + sigma * g + 0.5);
    dn = fmin(fmax(dn, 1.0), 65535.0);
    out = (u3 < dropout) ? 0 : (uint16_t)dn;
  }
  depth[(size_t)f * w * h + p] = out;
}

}  // namespace

extern "C" of_status_t of_synth_render_device(const void *d_scene, int32_t width, int32_t height,
                                              float fx, float fy, float cx, float cy,
                                              const double *d_poses, int32_t frames,
                                              uint64_t noise_seed, int32_t first_frame,
                                              float sigma_scale, float dropout, uint16_t *d_depth,
                                              of_stream_t stream) {
  if (!d_scene || !d_poses || !d_depth || width <= 0 || height <= 0 || frames <= 0 ||
      (long)width * height > (1L << 26) || frames > 65535 || fx <= 0.f || fy <= 0.f)
    return OF_ERR_INVALID_ARGUMENT;
  const long px = (long)width * height;
  dim3 grid((unsigned)((px + 255) / 256), 1, (unsigned)frames);
  k_synth_render<<<grid, 256, 0, (cudaStream_t)stream>>>(
      (const of_synth_scene_t *)d_scene, width, height, fx, fy, cx, cy, d_poses, noise_seed,
      first_frame, sigma_scale, dropout, d_depth);
  return of_launch_status();
}
