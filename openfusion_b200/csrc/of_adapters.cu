// of_adapters.cu -- conversions between this library's point maps and the
// reference's PointInfo / CameraData maps: AoS float3 in world space, invalid
// vertex = BAD_VERTEX = FLT_MAX (Source/include/Constants.h:36,
// Source/include/BasicTypes.h:40-49), invalid normal = 0
// (CameraHandler.cu:100-126, Raycaster.cu:131-134).
#include "of_common.cuh"

#include <float.h>

using namespace of;

bool of_camera_valid(const of_camera_t *c);
of_status_t of_model_pyramid(const of_camera_t *cam, int levels, void *d_model, cudaStream_t s);

namespace {

__global__ void k_points_to_ref(const float4 *__restrict__ pts, int npx, const double *pose,
                                float *v3, float *n3) {
  __shared__ Rigid T;
  if (threadIdx.x == 0 && pose) pose_to_rigid(pose, &T, nullptr);
  __syncthreads();
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npx) return;
  float4 v = pts[2 * p], n = pts[2 * p + 1];
  float3 vo = make_float3(FLT_MAX, FLT_MAX, FLT_MAX), no = make_float3(0.f, 0.f, 0.f);
  if (v.w != 0.f) vo = pose ? apply(T, make_float3(v.x, v.y, v.z)) : make_float3(v.x, v.y, v.z);
  if (v.w != 0.f && n.w != 0.f)
    no = pose ? rotate(T, make_float3(n.x, n.y, n.z)) : make_float3(n.x, n.y, n.z);
  if (v3) { v3[3 * p] = vo.x; v3[3 * p + 1] = vo.y; v3[3 * p + 2] = vo.z; }
  if (n3) { n3[3 * p] = no.x; n3[3 * p + 1] = no.y; n3[3 * p + 2] = no.z; }
}

// rgbaFloatToIntCamera (Source/src/CameraSupport/CameraHandler.cu:55-62)
__device__ __forceinline__ uint32_t pack_rgba(float x, float y, float z, float w) {
  x = __saturatef(x); y = __saturatef(y); z = __saturatef(z); w = __saturatef(w);
  return ((uint32_t)(w * 255.f) << 24) | ((uint32_t)(z * 255.f) << 16) |
         ((uint32_t)(y * 255.f) << 8) | (uint32_t)(x * 255.f);
}

// gray depth / max depth, opaque (d_convertDepthToWorldVertices, CameraHandler.cu:75-78)
__global__ void k_depth_rgba(const uint16_t *__restrict__ depth, int npx, float inv_max,
                             uint32_t *__restrict__ rgba) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npx) return;
  const float g = (float)depth[p] * inv_max;
  rgba[p] = pack_rgba(g, g, g, 1.f);
}

// (n + 1) / 2 per channel (d_convertDepthToWorldNormals, CameraHandler.cu:128-131;
// the raycast's show-normals mode, Raycaster.cu:214-218); an invalid normal is 0
__global__ void k_normal_rgba(const float4 *__restrict__ pts, int npx, const double *pose,
                              float alpha, uint32_t *__restrict__ rgba) {
  __shared__ Rigid T;
  if (threadIdx.x == 0 && pose) pose_to_rigid(pose, &T, nullptr);
  __syncthreads();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npx) return;
  const float4 v = pts[2 * p], n = pts[2 * p + 1];
  float3 no = make_float3(0.f, 0.f, 0.f);
  if (v.w != 0.f && n.w != 0.f)
    no = pose ? rotate(T, make_float3(n.x, n.y, n.z)) : make_float3(n.x, n.y, n.z);
  rgba[p] = pack_rgba((no.x + 1.f) * 0.5f, (no.y + 1.f) * 0.5f, (no.z + 1.f) * 0.5f, alpha);
}

__global__ void k_points_from_ref(const float *__restrict__ v3, const float *__restrict__ n3,
                                  int npx, float4 *pts) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npx) return;
  float vx = v3[3 * p], vy = v3[3 * p + 1], vz = v3[3 * p + 2];
  bool vok = !(vx == FLT_MAX || vy == FLT_MAX || vz == FLT_MAX);
  float nx = n3[3 * p], ny = n3[3 * p + 1], nz = n3[3 * p + 2];
  bool nok = vok && !(nx == 0.f && ny == 0.f && nz == 0.f);
  pts[2 * p] = vok ? make_float4(vx, vy, vz, 1.f) : make_float4(0.f, 0.f, 0.f, 0.f);
  pts[2 * p + 1] = nok ? make_float4(nx, ny, nz, 1.f) : make_float4(0.f, 0.f, 0.f, 0.f);
}

}  // namespace

extern "C" of_status_t of_points_to_reference(const of_camera_t *cam, const void *d_pyr,
                                              const double *d_pose, float *v3, float *n3,
                                              of_stream_t s) {
  if (!of_camera_valid(cam) || !d_pyr || (!v3 && !n3)) return OF_ERR_INVALID_ARGUMENT;
  of_pyramid_layout_t lay;
  of_status_t st = of_pyramid_layout(cam, 1, &lay);
  if (st != OF_OK) return st;
  int npx = cam->width * cam->height;
  k_points_to_ref<<<(npx + 255) / 256, 256, 0, (cudaStream_t)s>>>(
      (const float4 *)((const char *)d_pyr + lay.points_offset[0]), npx, d_pose, v3, n3);
  return of_launch_status();
}

extern "C" of_status_t of_points_from_reference(const of_camera_t *cam, int32_t levels,
                                                const float *v3, const float *n3, void *d_model,
                                                of_stream_t s) {
  if (!of_camera_valid(cam) || !v3 || !n3 || !d_model || levels < 1 || levels > kMaxLevels)
    return OF_ERR_INVALID_ARGUMENT;
  of_pyramid_layout_t lay;
  of_status_t st = of_pyramid_layout(cam, levels, &lay);
  if (st != OF_OK) return st;
  int npx = cam->width * cam->height;
  k_points_from_ref<<<(npx + 255) / 256, 256, 0, (cudaStream_t)s>>>(
      v3, n3, npx, (float4 *)((char *)d_model + lay.points_offset[0]));
  st = of_launch_status();
  if (st != OF_OK) return st;
  return of_model_pyramid(cam, levels, d_model, (cudaStream_t)s);
}

extern "C" of_status_t of_depth_to_rgba(const of_camera_t *cam, const uint16_t *d_depth,
                                        uint32_t *d_rgba, of_stream_t s) {
  if (!of_camera_valid(cam) || !d_depth || !d_rgba || cam->max_depth_mm <= 0.f)
    return OF_ERR_INVALID_ARGUMENT;
  const int npx = cam->width * cam->height;
  k_depth_rgba<<<(npx + 255) / 256, 256, 0, (cudaStream_t)s>>>(d_depth, npx,
                                                               1.f / cam->max_depth_mm, d_rgba);
  return of_launch_status();
}

extern "C" of_status_t of_normals_to_rgba(const of_camera_t *cam, const void *d_pyramid,
                                          const double *d_pose, float alpha, uint32_t *d_rgba,
                                          of_stream_t s) {
  if (!of_camera_valid(cam) || !d_pyramid || !d_rgba) return OF_ERR_INVALID_ARGUMENT;
  of_pyramid_layout_t lay;
  of_status_t st = of_pyramid_layout(cam, 1, &lay);
  if (st != OF_OK) return st;
  const int npx = cam->width * cam->height;
  k_normal_rgba<<<(npx + 255) / 256, 256, 0, (cudaStream_t)s>>>(
      (const float4 *)((const char *)d_pyramid + lay.points_offset[0]), npx, d_pose, alpha, d_rgba);
  return of_launch_status();
}

