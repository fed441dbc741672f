// Harness around d_initVoxelArray (Source/src/General.cu:27-50) and
// d_integrateVolume (Source/src/VolumeIntegrator.cu:86-187). The volume stays
// on the device between calls. d_integrateVolume advances its offset before
// the first use (VolumeIntegrator.cu:115-123), so voxel x is stored in slab
// x + 1 and the last slab writes N^2 elements past N^3: both arrays carry that
// many extra elements here so every access stays in bounds. Test infrastructure.
#include "VolumeIntegrator.cu"
#include "ref_common.h"

#include <vector>

__global__ void d_initVoxelArray(VoxelType *d_voxel_array, VoxelWeightType *d_weight_array);

struct RefVolume {
  VoxelType *tsdf;
  VoxelWeightType *w;
};
static RefVolume g_vol = {nullptr, nullptr};
static const size_t kElems = (size_t)VOLUME_SIZE * VOLUME_SIZE * VOLUME_SIZE +
                             (size_t)VOLUME_SIZE * VOLUME_SIZE;

extern "C" int ref_volume_size(void) { return (int)VOLUME_SIZE; }
extern "C" float ref_world_volume(void) { return (float)worldVolume; }
extern "C" float ref_truncation(void) { return (float)TRUNCATION; }
extern "C" int ref_max_weight(void) { return (int)MAX_WEIGHT; }

// (Re)initialises the volume like General::InitVoxelArray (General.cpp:42-49);
// the padding slab gets the same initial values.
extern "C" int ref_volume_init(void) {
  if (!g_vol.tsdf) {
    REF_TRY(cudaMalloc(&g_vol.tsdf, kElems * sizeof(VoxelType)));
    REF_TRY(cudaMalloc(&g_vol.w, kElems * sizeof(VoxelWeightType)));
  }
  dim3 grid(VOLUME_SIZE, VOLUME_SIZE);
  d_initVoxelArray<<<grid, VOLUME_SIZE>>>(g_vol.tsdf, g_vol.w);
  REF_TRY(cudaDeviceSynchronize());
  std::vector<float> pad((size_t)VOLUME_SIZE * VOLUME_SIZE, (float)TRUNCATION);
  size_t n3 = (size_t)VOLUME_SIZE * VOLUME_SIZE * VOLUME_SIZE;
  REF_TRY(cudaMemcpy(g_vol.tsdf + n3, pad.data(), pad.size() * 4, cudaMemcpyHostToDevice));
  REF_TRY(cudaMemset(g_vol.w + n3, 0, pad.size()));
  return 0;
}

extern "C" int ref_volume_free(void) {
  if (g_vol.tsdf) cudaFree(g_vol.tsdf);
  if (g_vol.w) cudaFree(g_vol.w);
  g_vol.tsdf = nullptr;
  g_vol.w = nullptr;
  return 0;
}

// One VolumeIntegrator::Integrate call (VolumeIntegrator.cu:199-201): world
// vertex map (float3 W*H), world-to-camera float[16], camera position.
extern "C" int ref_integrate(const ref_cam *c, const float *h_vertex, const float *h_invT,
                             const float *h_campos) {
  CameraParams p;
  memset(&p, 0, sizeof(p));
  p.m_intrinsic.Set(c->fx, c->fy, c->cx, c->cy);
  p.m_invIntrinsic.Set(c->ifx, c->ify, c->icx, c->icy);
  p.m_width = c->w;
  p.m_height = c->h;
  p.m_min_depth = c->dmin;
  p.m_max_depth = c->dmax;
  size_t n = (size_t)c->w * c->h;
  CameraData d;
  memset(&d, 0, sizeof(d));
  float *dinv = nullptr;
  float3 *dpos = nullptr;
  REF_TRY(cudaMalloc(&d.vertex, n * sizeof(float3)));
  REF_TRY(cudaMalloc(&dinv, 64));
  REF_TRY(cudaMalloc(&dpos, sizeof(float3)));
  REF_TRY(cudaMemcpy(d.vertex, h_vertex, n * sizeof(float3), cudaMemcpyHostToDevice));
  REF_TRY(cudaMemcpy(dinv, h_invT, 64, cudaMemcpyHostToDevice));
  REF_TRY(cudaMemcpy(dpos, h_campos, sizeof(float3), cudaMemcpyHostToDevice));
  VolumeIntegrator vi(&p);
  vi.Integrate(g_vol.tsdf, g_vol.w, dinv, d, dpos);
  REF_TRY(cudaDeviceSynchronize());
  cudaFree(d.vertex); cudaFree(dinv); cudaFree(dpos);
  return 0;
}

// Reads the stored values at `count` storage indices (x*N*N + y*N + z,
// x up to N so the padding slab is reachable).
extern "C" int ref_volume_read(const int64_t *idx, int64_t count, float *tsdf, uint8_t *w) {
  std::vector<float> t(kElems);
  std::vector<uint8_t> ww(kElems);
  REF_TRY(cudaMemcpy(t.data(), g_vol.tsdf, kElems * 4, cudaMemcpyDeviceToHost));
  REF_TRY(cudaMemcpy(ww.data(), g_vol.w, kElems, cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < count; ++i) {
    tsdf[i] = t[(size_t)idx[i]];
    w[i] = ww[(size_t)idx[i]];
  }
  return 0;
}

// Whole arrays (N^3 + N^2 elements each) for the raycast and pipeline harness.
extern "C" void *ref_volume_device_tsdf(void) { return g_vol.tsdf; }
void *ref_volume_device_weight(void) { return g_vol.w; }
