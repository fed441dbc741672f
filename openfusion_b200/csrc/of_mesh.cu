// of_mesh.cu -- triangle mesh of the fused surface, and the volume written as
// the reference's SavedVolume.raw.
//
// The reference saves the raw float volume (RunApp::saveVolumeToFile,
// Source/src/MainApp.cpp:181-276) and leaves its marching-cubes extraction
// commented out (:277-328). Here the tsdf = 0 surface of the observed voxels is
// extracted on the device by marching tetrahedra: every cell (the cube of 8
// neighbouring voxel centres) is split into the 6 tetrahedra around its
// main diagonal (Kuhn's triangulation: vertices 0, e_a, e_a + e_b, 7 for
// each order a, b, c of the axes, corner index = dx | dy << 1 | dz << 2).
// Neighbouring cells split their shared face along the same diagonal, so the
// surface has no cracks. In a tetrahedron the corners with tsdf < 0 are
// inside; one corner apart from the other three gives one triangle on its
// three edges, two against two give a quadrilateral (two triangles). A vertex
// lies on its edge where the linear interpolation of the tsdf crosses 0,
// computed from the edge's lower-addressed voxel so that a vertex shared by
// cells is bit-identical. Triangles face the outside: their normal points
// from the inside corners to the outside ones. Only cells whose 8 voxels are
// all observed produce triangles, and cells of unflagged bricks (which hold
// only +1) are skipped whole.
#include "of_common.cuh"

#include <cstdio>
#include <vector>

using namespace of;

bool of_volume_valid(const of_volume_desc_t *d);

namespace {

// the 6 tetrahedra of a cell, as corner indices (dx | dy << 1 | dz << 2)
__constant__ unsigned char c_tets[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7},
                                           {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};

constexpr int kMeshThreads = 512;  // one brick's 8^3 cells per block

struct Corner {
  float v;     // normalised tsdf
  float3 p;    // world position, mm
  size_t a;    // brick-major address (orders the ends of an edge)
};

__device__ __forceinline__ float3 edge_point(const Corner &x, const Corner &y) {
  const Corner &lo = x.a < y.a ? x : y;
  const Corner &hi = x.a < y.a ? y : x;
  const float t = lo.v / (lo.v - hi.v);
  return make_float3(fmaf(t, hi.p.x - lo.p.x, lo.p.x), fmaf(t, hi.p.y - lo.p.y, lo.p.y),
                     fmaf(t, hi.p.z - lo.p.z, lo.p.z));
}

__device__ __forceinline__ void put_tri(float *out, float3 a, float3 b, float3 c, float3 dir) {
  // normal (b - a) x (c - a) along dir (inside -> outside), else swap b, c
  const float ux = b.x - a.x, uy = b.y - a.y, uz = b.z - a.z;
  const float vx = c.x - a.x, vy = c.y - a.y, vz = c.z - a.z;
  const float nx = uy * vz - uz * vy, ny = uz * vx - ux * vz, nz = ux * vy - uy * vx;
  if (nx * dir.x + ny * dir.y + nz * dir.z < 0.f) {
    const float3 t = b;
    b = c;
    c = t;
  }
  out[0] = a.x; out[1] = a.y; out[2] = a.z;
  out[3] = b.x; out[4] = b.y; out[5] = b.z;
  out[6] = c.x; out[7] = c.y; out[8] = c.z;
}

// triangles of tetrahedron q of a cell: 0, 1 or 2
__device__ __forceinline__ int tet_triangles(const float *v, int q) {
  int in = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) in += v[c_tets[q][i]] < 0.f;
  return (in == 0 || in == 4) ? 0 : (in == 2 ? 2 : 1);
}

template <int STORAGE>
__global__ void __launch_bounds__(kMeshThreads) k_mesh(const uint32_t *__restrict__ vol,
                                                       VolGeom g, float *__restrict__ tris,
                                                       unsigned long long *__restrict__ ids,
                                                       unsigned int max_tris,
                                                       unsigned int *__restrict__ count) {
  const int n = g.n, nb = g.nb;
  const uint8_t *flags = brick_flags((void *)vol, n);
  const int lane = threadIdx.x & 31;
  const int nbr = nb * nb * nb;
  for (int b = blockIdx.x; b < nbr; b += gridDim.x) {
    if (__ldg(flags + b) == 0) continue;  // the brick and its neighbours hold only +1
    const int bx = b / (nb * nb), by = (b / nb) % nb, bz = b % nb;
    const int i = 8 * bx + (threadIdx.x >> 6), j = 8 * by + ((threadIdx.x >> 3) & 7),
              k = 8 * bz + (threadIdx.x & 7);
    float v[8];
    bool live = i < n - 1 && j < n - 1 && k < n - 1;
    if (live) {
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const uint32_t w = __ldg(vol + vox_index(nb, i + (c & 1), j + ((c >> 1) & 1), k + (c >> 2)));
        live &= (w >> 16) != 0u;
        v[c] = VoxelCodec<STORAGE>::tsdf(w);
      }
    }
    int cnt = 0;
    if (live)
#pragma unroll
      for (int q = 0; q < 6; ++q) cnt += tet_triangles(v, q);
    // one atomic per warp: inclusive scan of the counts
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned int base = 0;
    if (lane == 31 && total > 0) base = atomicAdd(count, (unsigned)total);
    base = __shfl_sync(0xffffffffu, base, 31) + (unsigned)(incl - cnt);
    if (cnt == 0) continue;
    Corner C[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int ci = i + (c & 1), cj = j + ((c >> 1) & 1), ck = k + (c >> 2);
      C[c].v = v[c];
      C[c].p = make_float3(fmaf(g.vs, (float)ci + 0.5f, g.origin), fmaf(g.vs, (float)cj + 0.5f, g.origin),
                           fmaf(g.vs, (float)ck + 0.5f, g.origin));
      C[c].a = vox_index(nb, ci, cj, ck);
    }
    const unsigned long long cell = ((unsigned long long)i * n + j) * n + k;
    unsigned int slot = base;
    for (int q = 0; q < 6; ++q) {
      const int t0 = c_tets[q][0], t1 = c_tets[q][1], t2 = c_tets[q][2], t3 = c_tets[q][3];
      const int tv[4] = {t0, t1, t2, t3};
      int inside[4], outside[4], ni = 0, no = 0;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (v[tv[r]] < 0.f) inside[ni++] = tv[r];
        else outside[no++] = tv[r];
      }
      if (ni == 0 || ni == 4) continue;
      // inside -> outside direction: mean outside corner minus mean inside corner
      float3 dir = make_float3(0.f, 0.f, 0.f);
      for (int r = 0; r < no; ++r) {
        dir.x += C[outside[r]].p.x * ni; dir.y += C[outside[r]].p.y * ni; dir.z += C[outside[r]].p.z * ni;
      }
      for (int r = 0; r < ni; ++r) {
        dir.x -= C[inside[r]].p.x * no; dir.y -= C[inside[r]].p.y * no; dir.z -= C[inside[r]].p.z * no;
      }
      if (ni == 2) {
        const int p = inside[0], qq = inside[1], r = outside[0], s = outside[1];
        const float3 epr = edge_point(C[p], C[r]), eqr = edge_point(C[qq], C[r]);
        const float3 eqs = edge_point(C[qq], C[s]), eps = edge_point(C[p], C[s]);
        if (slot < max_tris) {
          put_tri(tris + 9 * (size_t)slot, epr, eqr, eqs, dir);
          if (ids) ids[slot] = cell * 12ull + (unsigned long long)(2 * q);
        }
        ++slot;
        if (slot < max_tris) {
          put_tri(tris + 9 * (size_t)slot, epr, eqs, eps, dir);
          if (ids) ids[slot] = cell * 12ull + (unsigned long long)(2 * q + 1);
        }
        ++slot;
      } else {
        // the corner on its own side, and the other three
        const int s = ni == 1 ? inside[0] : outside[0];
        const int *rest = ni == 1 ? outside : inside;
        const float3 a = edge_point(C[s], C[rest[0]]), bq = edge_point(C[s], C[rest[1]]),
                     c = edge_point(C[s], C[rest[2]]);
        if (slot < max_tris) {
          put_tri(tris + 9 * (size_t)slot, a, bq, c, dir);
          if (ids) ids[slot] = cell * 12ull + (unsigned long long)(2 * q);
        }
        ++slot;
      }
    }
  }
}

}  // namespace

extern "C" of_status_t of_mesh_extract(const of_volume_desc_t *d, const void *vol, float *d_tris,
                                       uint64_t *d_ids, uint32_t max_triangles, uint32_t *d_count,
                                       of_stream_t stream) {
  OF_RANGE("of_mesh_extract");
  if (!of_volume_valid(d) || !vol || !d_count || (max_triangles > 0 && !d_tris))
    return OF_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  OF_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(uint32_t), s));
  const VolGeom g = make_geom(*d);
  const int nbr = g.nb * g.nb * g.nb;
  const int blocks = nbr < kSmCount * 4 ? nbr : kSmCount * 4;
  if (d->storage == OF_TSDF_I16)
    k_mesh<OF_TSDF_I16><<<blocks, kMeshThreads, 0, s>>>((const uint32_t *)vol, g, d_tris,
                                                       (unsigned long long *)d_ids, max_triangles,
                                                       d_count);
  else
    k_mesh<OF_TSDF_F16><<<blocks, kMeshThreads, 0, s>>>((const uint32_t *)vol, g, d_tris,
                                                       (unsigned long long *)d_ids, max_triangles,
                                                       d_count);
  return of_launch_status();
}

extern "C" of_status_t of_mesh_write_obj(const char *path, const float *tris, uint32_t count) {
  if (!path || (count > 0 && !tris)) return OF_ERR_INVALID_ARGUMENT;
  FILE *f = fopen(path, "w");
  if (!f) return OF_ERR_IO;
  fprintf(f, "# %u triangles, world mm\n", count);
  for (size_t i = 0; i < (size_t)count * 3; ++i)
    fprintf(f, "v %.6g %.6g %.6g\n", tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]);
  // OBJ vertex indices count from 1
  for (size_t t = 0; t < count; ++t)
    fprintf(f, "f %zu %zu %zu\n", 3 * t + 1, 3 * t + 2, 3 * t + 3);
  const bool ok = ferror(f) == 0;
  return fclose(f) == 0 && ok ? OF_OK : OF_ERR_IO;
}

extern "C" of_status_t of_volume_save_raw(const of_volume_desc_t *d, const void *vol,
                                          const char *path, of_stream_t stream) {
  if (!of_volume_valid(d) || !vol || !path) return OF_ERR_INVALID_ARGUMENT;
  const size_t n3 = (size_t)d->resolution * d->resolution * d->resolution;
  float *d_tsdf = nullptr;
  uint16_t *d_w = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMalloc(&d_tsdf, n3 * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_w, n3 * sizeof(uint16_t));
  if (e != cudaSuccess) {
    cudaFree(d_tsdf);
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? OF_ERR_OUT_OF_MEMORY : of_set_cuda_error(e);
  }
  std::vector<float> host;
  of_status_t st = of_volume_export(d, vol, d_tsdf, d_w, stream);
  if (st == OF_OK) {
    host.resize(n3);
    e = cudaMemcpyAsync(host.data(), d_tsdf, n3 * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = of_set_cuda_error(e);
  }
  cudaFree(d_tsdf);
  cudaFree(d_w);
  if (st != OF_OK) return st;
  FILE *f = fopen(path, "wb");
  if (!f) return OF_ERR_IO;
  const size_t wrote = fwrite(host.data(), sizeof(float), n3, f);
  return fclose(f) == 0 && wrote == n3 ? OF_OK : OF_ERR_IO;
}
