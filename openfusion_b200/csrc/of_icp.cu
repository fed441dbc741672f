// of_icp.cu -- multi-level point-to-plane ICP, entirely on the device.
//
// The whole coarse-to-fine ICP of a frame runs in one cooperative launch
// (k_icp_fused; k_icp_iter is the one-iteration form behind of_icp_system).
// Together they do what the reference spreads over d_find_corresponding
// (Source/src/ICP.cu:116-251) and the host loop of ICP::Iterate_ICP
// (Source/src/ICP.cpp:84-182):
//   for every model pixel with a valid world vertex s and normal n_s:
//     s_c = T^-1 s; pixel = roundFloat(project(s_c)), rejected when outside
//     the image or s_c.z >= -eps (ICP.cu:90-95, :152-167);
//     d = T v(pixel), n_d = R n(pixel) from the frame's camera-space maps
//     (the reference re-converts the frame to world space at every
//     iteration instead, ICP.cpp:174);
//     inlier if |d - s| < dist and thresh < n_d . n_s < 1 + eps (ICP.cu:179-181);
//     row A = [n_s x d, n_s], b = n_s . (s - d) (ICP.cu:186-201);
//   sum the 21 upper A^T A entries, 6 A^T b entries, b^2 and the inlier count
//   in FP32 (per-thread sums, pairwise shuffle trees per warp and block,
//   Kahan over the blocks' partials);
//   solve A^T A x = A^T b in FP64, negate the rotation part (ICP.cpp:162-168),
//   build dT = [Rz(g) Ry(b) Rx(a) | t] and compose T <- dT T in FP64
//   (ICP.cu:266-305). A singular system restores the frame's starting pose and
//   stops the remaining iterations (ICP.cpp:152-158).
#include "of_batch.cuh"

#include <mutex>
#include <string.h>

using namespace of;

bool of_camera_valid(const of_camera_t *c);

namespace {

constexpr int kIcpThreads = 256;
constexpr int kIcpMaxBlocks = 2 * kSmCount;
constexpr int kVals = 29;  // 21 + 6 + residual^2 + inliers
constexpr float kEps = 1e-6f;  // _EPSILON_ (Constants.h:14)

constexpr int kFusedThreads = 1024;
constexpr int kFusedMaxBlocks = 2 * kSmCount;
// model points a block of the fused kernel keeps in shared memory (192 KiB)
constexpr int kMaxCachePts = 6144;
// A partial-sum row slot of the fused kernel is one 64-bit word: the value's
// bits, and above them the slot's sequence number (the frame's epoch << 13 |
// the iteration + 1), so a reader that sees the number sees the value with it.
constexpr int kIterBits = 13;  // up to 2 passes x 4 levels x 1000 iterations
constexpr unsigned kEpochMask = (1u << (32 - kIterBits)) - 1u;
// A grid barrier gives up after about 0.15 s (this many 32 ns sleeps) and
// reports status 2 instead of waiting forever.
constexpr unsigned kSpinLimit = 1u << 22;

struct IcpWorkspace {
  unsigned int ticket;
  int stop;
  int iterations;
  int error;
  unsigned int bar_count;
  unsigned int bar_gen;
  int pad0[2];
  double pose_init[16];
  double prior[16];
  double warm_pose[16];  // this frame's warm start (of_icp_track_warm)
  int has_prior;
  int hold_barrier;  // fault injection: arrivals a grid barrier waits for that never come
  int has_warm;
  int pad2;
  float partials[kIcpMaxBlocks][32];
  unsigned long long fused_rows[2][kFusedMaxBlocks][32];
  unsigned int epoch;  // frames begun on this workspace (k_icp_begin), mod 2^19
  unsigned int magic;  // kWorkspaceMagic once k_icp_begin has cleared the rows
};
constexpr unsigned kWorkspaceMagic = 0x4F46494Bu;

enum IcpMode { kModeUpdate = 0, kModeSystem = 1 };

__device__ __forceinline__ void kahan_add(float &sum, float &comp, float x) {
  float y = x - comp;
  float t = sum + y;
  comp = (t - sum) - y;
  sum = t;
}

// FP64 6x6 Cholesky solve of H x = g (H given by its 21 upper entries).
// Returns false when a pivot is not larger than 1e-12 x the largest diagonal
// entry or is not finite; *minpiv gets the smallest pivot / largest diagonal.
__device__ __noinline__ bool chol_solve6(const double *up, const double *g, double *x,
                                        double *minpiv) {
  double H[6][6];
  int q = 0;
  for (int i = 0; i < 6; ++i)
    for (int j = i; j < 6; ++j) {
      H[i][j] = up[q];
      H[j][i] = up[q];
      ++q;
    }
  double dmax = 0.0;
  for (int i = 0; i < 6; ++i) dmax = fmax(dmax, H[i][i]);
  double L[6][6] = {};
  double mp = 1e300;
  bool ok = dmax > 0.0 && isfinite(dmax);
  double inv[6];
  const double inv_dmax = 1.0 / dmax;
  for (int j = 0; j < 6 && ok; ++j) {
    double s = H[j][j];
    for (int k = 0; k < j; ++k) s -= L[j][k] * L[j][k];
    mp = fmin(mp, s * inv_dmax);
    if (!(s > 1e-12 * dmax) || !isfinite(s)) { ok = false; break; }
    double ljj = sqrt(s);
    inv[j] = 1.0 / ljj;
    L[j][j] = ljj;
    for (int i = j + 1; i < 6; ++i) {
      double t = H[i][j];
      for (int k = 0; k < j; ++k) t -= L[i][k] * L[j][k];
      L[i][j] = t * inv[j];
    }
  }
  *minpiv = ok ? mp : fmin(mp, 0.0);
  if (!ok) return false;
  double y[6];
  for (int i = 0; i < 6; ++i) {
    double t = g[i];
    for (int k = 0; k < i; ++k) t -= L[i][k] * y[k];
    y[i] = t * inv[i];
  }
  for (int i = 5; i >= 0; --i) {
    double t = y[i];
    for (int k = i + 1; k < 6; ++k) t -= L[k][i] * x[k];
    x[i] = t * inv[i];
  }
  return true;
}

// dT of Cpu_buildNewTransformMatrix (ICP.cu:266-290) in FP64, then P <- dT P.
__device__ __noinline__ void compose_increment(const double *xo, double *P) {
  double al = xo[0], be = xo[1], ga = xo[2];
  double ca, sa, cb, sb, cg, sg;
  sincos(al, &sa, &ca);
  sincos(be, &sb, &cb);
  sincos(ga, &sg, &cg);
  double D[16] = {cg * cb, -sg * ca + cg * sb * sa, sg * sa + cg * sb * ca, xo[3],
                  sg * cb, cg * ca + sg * sb * sa,  -cg * sa + sg * sb * ca, xo[4],
                  -sb,     cb * sa,                 cb * ca,                 xo[5],
                  0.0,     0.0,                     0.0,                     1.0};
  double O[16];
  for (int i = 0; i < 16; ++i) O[i] = P[i];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double a = 0.0;
      for (int k = 0; k < 4; ++k) a += D[4 * i + k] * O[4 * k + j];
      P[4 * i + j] = a;
    }
}

template <int MODE>
__global__ void __launch_bounds__(kIcpThreads)
    k_icp_iter(const float4 *__restrict__ model, int mw, int mh, const float4 *__restrict__ frame,
               Cam cam, float dist_thresh, float normal_thresh, double *pose, IcpWorkspace *ws,
               of_icp_stats_t *stats, float *system_out) {
  __shared__ Rigid s_c2w, s_w2c;
  __shared__ int s_stop;
  __shared__ float s_red[kIcpThreads / 32][32];
  __shared__ bool s_last;
  if (threadIdx.x == 0) {
    s_stop = (MODE == kModeUpdate) ? ws->stop : 0;
    if (!s_stop) pose_to_rigid(pose, &s_c2w, &s_w2c);
  }
  __syncthreads();
  if (s_stop) return;

  float acc[kVals], cmp[kVals];
#pragma unroll
  for (int v = 0; v < kVals; ++v) { acc[v] = 0.f; cmp[v] = 0.f; }

  const int npx = mw * mh;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npx; p += gridDim.x * blockDim.x) {
    float4 s = model[2 * p];
    float4 ns = model[2 * p + 1];
    if (s.w == 0.f || ns.w == 0.f) continue;
    float3 sc = apply(s_w2c, make_float3(s.x, s.y, s.z));
    if (sc.z >= -kEps) continue;
    float rz = __frcp_rn(sc.z);
    int pu = round_ref(fmaf(cam.fx * sc.x, rz, cam.cx));
    int pv = round_ref(fmaf(cam.fy * sc.y, rz, cam.cy));
    if (pu < 0 || pu >= cam.w || pv < 0 || pv >= cam.h) continue;
    size_t q = (size_t)pv * cam.w + pu;
    float4 dc = __ldg(frame + 2 * q);
    float4 nc = __ldg(frame + 2 * q + 1);
    if (dc.w == 0.f || nc.w == 0.f) continue;
    float3 d = apply(s_c2w, make_float3(dc.x, dc.y, dc.z));
    float3 nd = rotate(s_c2w, make_float3(nc.x, nc.y, nc.z));
    float ex = d.x - s.x, ey = d.y - s.y, ez = d.z - s.z;
    if (!(sqrtf(ex * ex + ey * ey + ez * ez) < dist_thresh)) continue;
    float dn = nd.x * ns.x + nd.y * ns.y + nd.z * ns.z;
    if (!(dn > normal_thresh && dn < 1.f + kEps)) continue;
    float a[6];
    a[0] = ns.y * d.z - ns.z * d.y;
    a[1] = ns.z * d.x - ns.x * d.z;
    a[2] = ns.x * d.y - ns.y * d.x;
    a[3] = ns.x; a[4] = ns.y; a[5] = ns.z;
    float b = -(ns.x * ex + ns.y * ey + ns.z * ez);
    int k = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int j = i; j < 6; ++j) { kahan_add(acc[k], cmp[k], a[i] * a[j]); ++k; }
#pragma unroll
    for (int i = 0; i < 6; ++i) kahan_add(acc[21 + i], cmp[21 + i], a[i] * b);
    kahan_add(acc[27], cmp[27], b * b);
    acc[28] += 1.f;
  }
  // warp tree, then block tree over the 8 warps
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int v = 0; v < kVals; ++v) {
    float x = acc[v] - cmp[v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) s_red[warp][v] = x;
  }
  __syncthreads();
  if (warp == 0) {
    float x = 0.f;
    if (lane < kVals) {
      float y[kIcpThreads / 32];
#pragma unroll
      for (int w = 0; w < kIcpThreads / 32; ++w) y[w] = s_red[w][lane];
#pragma unroll
      for (int span = 1; span < kIcpThreads / 32; span *= 2)
#pragma unroll
        for (int w = 0; w + span < kIcpThreads / 32; w += 2 * span) y[w] += y[w + span];
      x = y[0];
    }
    ws->partials[blockIdx.x][lane] = x;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&ws->ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!s_last) return;
  __threadfence();

  // ---- last block: combine the per-block partials (Kahan per group, tree)
  {
    const int v = threadIdx.x & 31, grp = threadIdx.x >> 5;
    float sum = 0.f, c = 0.f;
    if (v < kVals)
      for (int r = grp; r < (int)gridDim.x; r += kIcpThreads / 32)
        kahan_add(sum, c, __ldcg(&ws->partials[r][v]));
    s_red[grp][v] = sum - c;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  float tot[kVals];
  for (int v = 0; v < kVals; ++v) {
    float y[kIcpThreads / 32];
    for (int w = 0; w < kIcpThreads / 32; ++w) y[w] = s_red[w][v];
    for (int span = 1; span < kIcpThreads / 32; span *= 2)
      for (int w = 0; w + span < kIcpThreads / 32; w += 2 * span) y[w] += y[w + span];
    tot[v] = y[0];
  }
  ws->ticket = 0;
  if (MODE == kModeSystem) {
    for (int v = 0; v < kVals; ++v) system_out[v] = tot[v];
    return;
  }
  double up[21], g[6], xs[6], minpiv = 0.0;
  for (int v = 0; v < 21; ++v) up[v] = (double)tot[v];
  for (int v = 0; v < 6; ++v) g[v] = (double)tot[21 + v];
  int inliers = (int)tot[28];
  bool ok = inliers >= 6 && chol_solve6(up, g, xs, &minpiv);
  ws->iterations += 1;
  if (ok) {
    double xo[6] = {-xs[0], -xs[1], -xs[2], xs[3], xs[4], xs[5]};
    compose_increment(xo, pose);
  } else {
    for (int i = 0; i < 16; ++i) pose[i] = ws->pose_init[i];
    ws->stop = 1;
  }
  if (stats) {
    stats->status = ok ? 0 : 1;
    stats->inliers = inliers;
    stats->iterations = ws->iterations;
    stats->residual_sq = (double)tot[27];
    stats->min_pivot = minpiv;
  }
}

struct IcpLevel {
  const float4 *model;
  const float4 *frame;
  Cam cam;      // level intrinsics (of the frame's image)
  int mw, mh;   // model map size at this level
  int iters;
};

struct IcpPlan {
  IcpLevel lv[kMaxLevels];
  int levels;
  float dist_thresh, normal_thresh;
  int cache_pts;  // model points a block keeps in shared memory per level
  float stop_rot, stop_trans;  // early exit (0: every iteration)
  float judge_rms, judge_frac, judge_rot, judge_trans;
  int warm_levels;  // levels of a warm-started pass (<= levels)
  // optional pose history (a ring of hist_cap row-major poses and its running
  // count): the final pose is appended by the kernel's last store
  double *hist;
  unsigned long long *hist_count;
  int hist_cap;
};

// Grid-wide exchange of a co-resident grid. Each block publishes its row of
// partial sums and then, with a release store, the row's sequence number (the
// iteration, counted from 1 within a frame; the begin kernel zeroes them);
// a reader acquires a row's sequence number before it reads the row. A wait
// is bounded; on timeout the workspace error flag is set.
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_gpu(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_gpu(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Waits (acquire) until *p == v; gives up after kSpinLimit polls or as soon as
// another block has reported a failed wait. Returns whether *p reached v.
__device__ __forceinline__ bool wait_seq(IcpWorkspace *ws, const unsigned *p, unsigned v) {
  unsigned spins = 0;
  while (ld_acquire_gpu(p) != v) {
    if (++spins > kSpinLimit) return false;
    if ((spins & 255u) == 0u && ld_acquire_gpu(reinterpret_cast<unsigned *>(&ws->error)) != 0u)
      return false;
    __nanosleep(32);
  }
  return true;
}

// 1 / d for a positive normal FP64 d: the approximate FP64 reciprocal of the
// PTX ISA (rcp.approx.ftz.f64; measured on B200 at most 9.8e-7 relative,
// about 2^-20) refined by two Newton-Raphson steps r <- r + r (1 - d r), each
// of which squares the relative error (to below 2^-80, under FP64 rounding).
// No conversion to FP32 and back is needed.
__device__ __forceinline__ double recip_pos(double d) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
  r = fma(r, fma(-d, r, 1.0), r);
  return fma(r, fma(-d, r, 1.0), r);
}

// sin and cos from their Maclaurin series (Horner in x^2): through x^9 and
// x^10 for |x| <= 1/32, through x^13 and x^14 for |x| <= 1/4; the truncation
// error is below 1e-20 relative in both cases, far under FP64 rounding.
// Larger angles use the library.
__device__ __forceinline__ void sincos_small(double x, double *s, double *c) {
  if (!(fabs(x) <= 0.25)) {
    sincos(x, s, c);
    return;
  }
  const double x2 = x * x;
  if (fabs(x) <= 0.03125) {
    double ps = 1.0 / 362880.0;               // 1/9!
    ps = fma(ps, x2, -1.0 / 5040.0);          // -1/7!
    ps = fma(ps, x2, 1.0 / 120.0);            // 1/5!
    ps = fma(ps, x2, -1.0 / 6.0);             // -1/3!
    *s = fma(x * x2, ps, x);                  // x + x^3 (-1/3! + x^2/5! - ...)
    double pc = -1.0 / 3628800.0;             // -1/10!
    pc = fma(pc, x2, 1.0 / 40320.0);          // 1/8!
    pc = fma(pc, x2, -1.0 / 720.0);           // -1/6!
    pc = fma(pc, x2, 1.0 / 24.0);             // 1/4!
    pc = fma(pc, x2, -0.5);                   // -1/2!
    *c = fma(x2, pc, 1.0);                    // 1 + x^2 (-1/2! + x^2/4! - ...)
    return;
  }
  double ps = -1.0 / 6227020800.0;            // -1/13!
  ps = fma(ps, x2, 1.0 / 39916800.0);         // 1/11!
  ps = fma(ps, x2, -1.0 / 362880.0);          // -1/9!
  ps = fma(ps, x2, 1.0 / 5040.0);             // 1/7!
  ps = fma(ps, x2, -1.0 / 120.0);             // -1/5!
  ps = fma(ps, x2, 1.0 / 6.0);                // 1/3!
  // sin x = x - x^3 q(x^2) with q = 1/3! - x^2/5! + x^4/7! - ... + x^10/13!
  *s = fma(-x * x2, ps, x);
  double pc = 1.0 / 87178291200.0;            // 1/14!
  pc = fma(pc, x2, -1.0 / 479001600.0);       // -1/12!
  pc = fma(pc, x2, 1.0 / 3628800.0);          // 1/10!
  pc = fma(pc, x2, -1.0 / 40320.0);           // -1/8!
  pc = fma(pc, x2, 1.0 / 720.0);              // 1/6!
  pc = fma(pc, x2, -1.0 / 24.0);              // -1/4!
  pc = fma(pc, x2, 0.5);                      // 1/2!
  // cos x = 1 - x2/2! + x2^2/4! - ... = 1 - x2 (1/2! - x2/4! + ...)
  *c = fma(-x2, pc, 1.0);
}

// Warp-parallel FP64 solve of the 6x6 normal equations (21 upper entries and
// 6 right-hand sides in tot[0..26], inliers in tot[28]) and the SE(3) update
// of P (row-major 4x4, shared memory); all 32 lanes of one warp call it.
// Lane i < 6 holds row i of [H | g] and the rows are eliminated in order
// (Gaussian elimination without pivoting, which on the symmetric system is the
// LDL^T factorisation: its pivots d_j equal the squared Cholesky pivots, so
// the singularity rule is the Cholesky solve's: a pivot not above 1e-12 x the
// largest diagonal entry, a non-finite pivot, or fewer than 6 inliers). Back
// substitution by one shuffle per unknown, rotation part negated
// (ICP.cpp:162-168), dT = [Rz(g) Ry(b) Rx(a) | t] (ICP.cu:274-290) and
// P <- dT P with one entry per lane. Returns the warp-uniform success flag;
// *minpiv gets min d_j / max H_ii, *inc_rot / *inc_trans the largest
// rotation (rad) / translation (mm) component of the increment. With c2w /
// w2c given, the lanes also write the FP32 rigid transforms of the new pose
// (pose_to_rigid's values) on success.
__device__ __forceinline__ double shfl_d(double v, int src) {
  return __shfl_sync(0xffffffffu, v, src);
}
__device__ __forceinline__ int upper_index(int i, int j) {  // i <= j
  return i * 6 - i * (i - 1) / 2 + (j - i);
}
__device__ bool warp_solve_update(const float *tot, double *P, double *minpiv, float *inc_rot,
                                  float *inc_trans, Rigid *c2w = nullptr, Rigid *w2c = nullptr) {
  const int lane = threadIdx.x & 31;
  const int row = lane < 6 ? lane : 5;  // lanes 6.. shadow row 5
  double a[7];
#pragma unroll
  for (int k = 0; k < 6; ++k)
    a[k] = (double)tot[row <= k ? upper_index(row, k) : upper_index(k, row)];
  a[6] = (double)tot[21 + row];
  double dmax = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) dmax = fmax(dmax, (double)tot[upper_index(i, i)]);
  bool ok = tot[28] >= 6.f && dmax > 0.0 && isfinite(dmax);
  const double thr = 1e-12 * dmax;
  double dmin = 1e300, rmine = 0.0;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    double pj[7];
#pragma unroll
    for (int k = j; k < 7; ++k) pj[k] = shfl_d(a[k], j);
    const double dj = pj[j];
    dmin = fmin(dmin, dj);
    ok = ok && (dj > thr) && isfinite(dj);
    const double rj = recip_pos(fmax(dj, 1e-300));
    if (row == j) rmine = rj;
    if (row > j) {
      const double f = a[j] * rj;
#pragma unroll
      for (int k = j + 1; k < 7; ++k) a[k] = fma(-f, pj[k], a[k]);
    }
  }
  *minpiv = ok ? dmin / dmax : fmin(dmin / dmax, 0.0);
  if (!ok) return false;
  double x[6];
#pragma unroll
  for (int i = 5; i >= 0; --i) {
    x[i] = shfl_d(a[6] * rmine, i);
    if (row < i) a[6] = fma(-a[i], x[i], a[6]);
  }
  *inc_rot = (float)fmax(fabs(x[0]), fmax(fabs(x[1]), fabs(x[2])));
  *inc_trans = (float)fmax(fabs(x[3]), fmax(fabs(x[4]), fabs(x[5])));
  double sv = 0.0, cv = 1.0;
  if (lane < 3) sincos_small(-x[lane], &sv, &cv);
  const double sa = shfl_d(sv, 0), ca = shfl_d(cv, 0);
  const double sb = shfl_d(sv, 1), cb = shfl_d(cv, 1);
  const double sg = shfl_d(sv, 2), cg = shfl_d(cv, 2);
  // lane l < 12 forms entry (l / 4, l % 4) of dT P; row 3 stays 0 0 0 1
  const int r = (lane >> 2) % 3, c = lane & 3;
  double D0, D1, D2, D3;
  if (r == 0) { D0 = cg * cb; D1 = -sg * ca + cg * sb * sa; D2 = sg * sa + cg * sb * ca; D3 = x[3]; }
  else if (r == 1) { D0 = sg * cb; D1 = cg * ca + sg * sb * sa; D2 = -cg * sa + sg * sb * ca; D3 = x[4]; }
  else { D0 = -sb; D1 = cb * sa; D2 = cb * ca; D3 = x[5]; }
  const double v = fma(D0, P[c], fma(D1, P[4 + c], fma(D2, P[8 + c], D3 * P[12 + c])));
  __syncwarp();
  if (lane < 12) P[lane] = v;
  if (c2w) {
    // entry (r, c) of the new pose is v on lane 4 r + c (lanes 0..11)
    if (lane < 12) {
      if (c < 3) {
        c2w->r[3 * r + c] = (float)v;
        w2c->r[3 * c + r] = (float)v;
      } else {
        c2w->t[r] = (float)v;
      }
    }
    // w2c.t[i] = -(column i of R) . t, lane i < 3
    const int ci = lane < 3 ? lane : 0;
    const double r0 = shfl_d(v, ci), r1 = shfl_d(v, 4 + ci), r2 = shfl_d(v, 8 + ci);
    const double t0 = shfl_d(v, 3), t1 = shfl_d(v, 7), t2 = shfl_d(v, 11);
    if (lane < 3) {
      double acc = 0.0;
      acc = fma(-r0, t0, acc);
      acc = fma(-r1, t1, acc);
      acc = fma(-r2, t2, acc);
      w2c->t[lane] = (float)acc;
    }
  }
  __syncwarp();
  return true;
}

// Point-to-plane row of one correspondence (ICP.cu:186-201) added to acc.
__device__ __forceinline__ void add_row(float *acc, float4 s, float4 ns, float3 d) {
  const float ex = d.x - s.x, ey = d.y - s.y, ez = d.z - s.z;
  float a[6];
  a[0] = ns.y * d.z - ns.z * d.y;
  a[1] = ns.z * d.x - ns.x * d.z;
  a[2] = ns.x * d.y - ns.y * d.x;
  a[3] = ns.x; a[4] = ns.y; a[5] = ns.z;
  const float b = -(ns.x * ex + ns.y * ey + ns.z * ez);
  int k = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = i; j < 6; ++j) { acc[k] = fmaf(a[i], a[j], acc[k]); ++k; }
#pragma unroll
  for (int i = 0; i < 6; ++i) acc[21 + i] = fmaf(a[i], b, acc[21 + i]);
  acc[27] = fmaf(b, b, acc[27]);
  acc[28] += 1.f;
}

// Data association of one model point (ICP.cu:90-95, :152-181): the frame
// pixel it projects to, or -1.
__device__ __forceinline__ int associate(const Rigid &w2c, const Cam &cam, float4 s) {
  const float3 sc = apply(w2c, make_float3(s.x, s.y, s.z));
  if (sc.z >= -kEps) return -1;
  const float rz = __frcp_rn(sc.z);
  const int pu = __float2int_rd(fmaf(cam.fx * sc.x, rz, cam.cx) + 0.5f);
  const int pv = __float2int_rd(fmaf(cam.fy * sc.y, rz, cam.cy) + 0.5f);
  if ((unsigned)pu >= (unsigned)cam.w || (unsigned)pv >= (unsigned)cam.h) return -1;
  return pv * cam.w + pu;
}

// Inlier test and row of a model point s, n_s and the frame point at its pixel.
__device__ __forceinline__ void try_row(float *acc, const Rigid &c2w, float4 s, float4 ns,
                                        float4 dc, float4 nc, float dist2, float nthr) {
  if (dc.w == 0.f || nc.w == 0.f) return;
  const float3 d = apply(c2w, make_float3(dc.x, dc.y, dc.z));
  const float3 nd = rotate(c2w, make_float3(nc.x, nc.y, nc.z));
  const float ex = d.x - s.x, ey = d.y - s.y, ez = d.z - s.z;
  if (!(fmaf(ex, ex, fmaf(ey, ey, ez * ez)) < dist2)) return;
  const float dn = nd.x * ns.x + nd.y * ns.y + nd.z * ns.z;
  if (!(dn > nthr && dn < 1.f + kEps)) return;
  add_row(acc, s, ns, d);
}

// Judge of a warm-started ICP result P (warm start W): kept when the last
// iteration's RMS point-to-plane residual, its inlier fraction among the
// examined model points, and its rotation / translation away from W are all
// within the thresholds.
__device__ __forceinline__ bool judge_keep(const IcpPlan &plan, const double *W, const double *P,
                                        double res_sq, int inliers, int examined) {
  double tr = 0.0, dt2 = 0.0;
  for (int i = 0; i < 3; ++i) {
    for (int k = 0; k < 3; ++k) tr += W[4 * k + i] * P[4 * k + i];
    const double d = P[4 * i + 3] - W[4 * i + 3];
    dt2 += d * d;
  }
  const double rot = acos(fmin(1.0, fmax(-1.0, 0.5 * (tr - 1.0))));
  const double rms = sqrt(res_sq / (double)max(inliers, 1));
  const double frac = (double)inliers / (double)max(examined, 1);
  return rms <= plan.judge_rms && frac >= plan.judge_frac && rot <= plan.judge_rot &&
         sqrt(dt2) <= plan.judge_trans;
}

// The whole multi-level ICP of one frame in one cooperative launch. Each
// block owns every grid-th 32-pixel chunk of every level's model; at the
// start of a level it copies its chunks' valid model points (vertex, normal)
// into shared memory in chunk order, up to the dynamic shared-memory capacity
// (the rest is read from global memory at every iteration). Per
// iteration: every block associates its points two at a time (both frame
// gathers in flight together), accumulates the rows (tree sums), writes 29
// partials, meets the others at one grid barrier, then reduces all blocks'
// partials in the same fixed order and one warp solves the 6x6 system, so
// every block holds the same new pose without a second barrier. Partials
// alternate between two buffers: a block can only overwrite buffer i%2 after
// the barrier of iteration i+1, which every block reaches only after reading it.
__global__ void __launch_bounds__(kFusedThreads, 1)
    k_icp_fused(IcpPlan plan, double *pose, IcpWorkspace *ws, of_icp_stats_t *stats) {
  extern __shared__ float4 s_pts[];  // 2 per cached model point
  __shared__ double s_pose[16];
  __shared__ Rigid s_c2w, s_w2c;
  __shared__ float s_red[kFusedThreads / 32][32];
  __shared__ float s_tot[32];
  __shared__ int s_chunk_off[kMaxCachePts / 32];  // per cached chunk: its valid points, then their offset
  __shared__ int s_stop, s_inl, s_its, s_err, s_npts, s_conv, s_warm, s_examined;
  __shared__ double s_res, s_piv;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kWarps = kFusedThreads / 32;
  // pass 0 starts from the warm start when this frame has one, else from the
  // frame's starting pose (ws->pose_init: the begin step's, with any prior
  // applied); pass 1, from the starting pose, runs only when the judge
  // replaces the warm-started result
  const bool warm = ws->has_warm != 0;
  const unsigned epoch = ws->epoch;
  if (threadIdx.x < 16)
    s_pose[threadIdx.x] = warm ? ws->warm_pose[threadIdx.x] : ws->pose_init[threadIdx.x];
  if (threadIdx.x == 0) {
    s_stop = 0; s_err = 0; s_its = 0; s_inl = 0; s_res = 0.0; s_piv = 0.0; s_examined = 0;
    s_warm = warm ? 1 : 0;
  }
  __syncthreads();  // every thread reads the flags and the pose below
  if (threadIdx.x == 0) pose_to_rigid(s_pose, &s_c2w, &s_w2c);
  // the fault-injection hook holds every exchange for an arrival that never
  // comes
  const bool hold = ws->hold_barrier > 0;
  const float dist2 = plan.dist_thresh * plan.dist_thresh, nthr = plan.normal_thresh;
  int iter_global = 0;
  for (int pass = 0; pass < 2; ++pass) {
    const int top = (pass == 0 && warm) ? plan.warm_levels - 1 : plan.levels - 1;
    for (int l = top; l >= 0 && !s_stop && !s_err; --l) {
      const IcpLevel L = plan.lv[l];
      const int npx = L.mw * L.mh;
      // model pixels are dealt to blocks in chunks of 32 (one warp), round
      // robin, so every block gets an even, spatially spread share: chunk
      // c_k = block + k * grid, k = 0 .. my_chunks - 1; the first kc chunks
      // are kept in shared memory, the rest is read at every iteration
      const int G = (int)gridDim.x;
      const int nchunks = (npx + 31) >> 5;
      const int my_chunks = nchunks > (int)blockIdx.x ? (nchunks - 1 - (int)blockIdx.x) / G + 1 : 0;
      const int kc = min(my_chunks, plan.cache_pts >> 5);
      // ---- cache this block's valid model points of the level, in chunk
      // order: warp w counts the valid points of chunks w, w + 32, ...; one
      // warp scans the counts into offsets; every warp stores its chunks'
      // points there (reloaded, now from L1). Three block barriers per level.
      for (int k = warp; k < kc; k += kWarps) {
        const int p = ((int)blockIdx.x + k * G) * 32 + lane;
        bool valid = false;
        if (p < npx) valid = __ldg(&L.model[2 * p].w) != 0.f && __ldg(&L.model[2 * p + 1].w) != 0.f;
        const unsigned m = __ballot_sync(0xffffffffu, valid);
        if (lane == 0) s_chunk_off[k] = __popc(m);
      }
      __syncthreads();
      // every thread has read the previous level's exit flag by now
      if (threadIdx.x == 0) s_conv = 0;
      if (warp == 0) {
        constexpr int kPer = (kMaxCachePts / 32 + 31) / 32;
        int c[kPer];
        int tot = 0;
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
          const int k = lane * kPer + i;
          c[i] = k < kc ? s_chunk_off[k] : 0;
          tot += c[i];
        }
        int inc = tot;  // inclusive scan over the lanes
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, inc, o);
          if (lane >= o) inc += y;
        }
        int run = inc - tot;
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
          const int k = lane * kPer + i;
          if (k < kc) s_chunk_off[k] = run;
          run += c[i];
        }
        if (lane == 31) s_npts = inc;
      }
      __syncthreads();
      for (int k = warp; k < kc; k += kWarps) {
        const int p = ((int)blockIdx.x + k * G) * 32 + lane;
        float4 s = make_float4(0.f, 0.f, 0.f, 0.f), ns = s;
        bool valid = false;
        if (p < npx) {
          s = __ldg(L.model + 2 * p);
          ns = __ldg(L.model + 2 * p + 1);
          valid = s.w != 0.f && ns.w != 0.f;
        }
        const unsigned m = __ballot_sync(0xffffffffu, valid);
        if (valid) {
          const int slot = s_chunk_off[k] + __popc(m & ((1u << lane) - 1u));
          s_pts[2 * slot] = s;
          s_pts[2 * slot + 1] = ns;
        }
      }
      __syncthreads();
      const int n = s_npts;
      for (int it = 0; it < L.iters; ++it) {
        float acc[kVals];
        float examined = 0.f;  // model points that project into the frame
#pragma unroll
        for (int v = 0; v < kVals; ++v) acc[v] = 0.f;
        // cached points, two per step
        for (int i = threadIdx.x; i < n; i += 2 * kFusedThreads) {
          const int j = i + kFusedThreads;
          const int qA = associate(s_w2c, L.cam, s_pts[2 * i]);
          const int qB = j < n ? associate(s_w2c, L.cam, s_pts[2 * j]) : -1;
          float4 dA = make_float4(0.f, 0.f, 0.f, 0.f), cA = dA, dB = dA, cB = dA;
          if (qA >= 0) { dA = __ldg(L.frame + 2 * qA); cA = __ldg(L.frame + 2 * qA + 1); }
          if (qB >= 0) { dB = __ldg(L.frame + 2 * qB); cB = __ldg(L.frame + 2 * qB + 1); }
          // the model points are read again from shared memory rather than
          // held in registers across the gathers
          asm volatile("" ::: "memory");
          if (qA >= 0) {
            examined += 1.f;
            try_row(acc, s_c2w, s_pts[2 * i], s_pts[2 * i + 1], dA, cA, dist2, nthr);
          }
          if (qB >= 0) {
            examined += 1.f;
            try_row(acc, s_c2w, s_pts[2 * j], s_pts[2 * j + 1], dB, cB, dist2, nthr);
          }
        }
        // the rest of the block's chunks, from global memory
        for (int k = kc + warp; k < my_chunks; k += kWarps) {
          const int p = ((int)blockIdx.x + k * G) * 32 + lane;
          if (p >= npx) continue;
          const float4 s = __ldg(L.model + 2 * p);
          const float4 ns = __ldg(L.model + 2 * p + 1);
          if (s.w == 0.f || ns.w == 0.f) continue;
          const int q = associate(s_w2c, L.cam, s);
          if (q < 0) continue;
          examined += 1.f;
          try_row(acc, s_c2w, s, ns, __ldg(L.frame + 2 * q), __ldg(L.frame + 2 * q + 1), dist2,
                  nthr);
        }
        // pairwise sums: a recursive-halving exchange across the warp (lanes
        // trade half of their remaining values each step, 31 shuffles for 32
        // values) leaves lane v with the warp's sum of value v; then a tree
        // over the block's warps. Value kVals is the examined-point count. A
        // warp that examined no point (the coarse levels leave most warps
        // idle) holds only +0 and writes its zeros directly.
        if (!__any_sync(0xffffffffu, examined > 0.f)) {
          s_red[warp][lane] = 0.f;
        } else {
          float r[32];
#pragma unroll
          for (int v = 0; v < 32; ++v) r[v] = v < kVals ? acc[v] : (v == kVals ? examined : 0.f);
#pragma unroll
          for (int sft = 16; sft >= 1; sft >>= 1) {
            const bool upper = (lane & sft) != 0;
#pragma unroll
            for (int i = 0; i < sft; ++i) {
              float send = upper ? r[i] : r[i + sft];
              float keep = upper ? r[i + sft] : r[i];
              r[i] = keep + __shfl_xor_sync(0xffffffffu, send, sft);
            }
          }
          s_red[warp][lane] = r[0];
        }
        __syncthreads();
        const int buf = iter_global & 1;
        const unsigned seq = (epoch << kIterBits) | (unsigned)(iter_global + 1);
        if (warp == 0) {
          float y[kWarps];
#pragma unroll
          for (int w = 0; w < kWarps; ++w) y[w] = s_red[w][lane];
#pragma unroll
          for (int span = 1; span < kWarps; span *= 2)
#pragma unroll
            for (int w = 0; w + span < kWarps; w += 2 * span) y[w] += y[w + span];
          // publish: each value with this iteration's sequence number in one
          // 64-bit store (no fence: a slot validates itself)
          if (lane <= kVals)
            st_relaxed_gpu(&ws->fused_rows[buf][blockIdx.x][lane],
                           (unsigned long long)__float_as_uint(y[0]) |
                               ((unsigned long long)seq << 32));
          // the fault-injection hook: an arrival that never comes
          if (hold && lane == 0 && !wait_seq(ws, &ws->bar_gen, 0xffffffffu)) {
            atomicExch(&ws->error, 1);
            s_err = 1;
          }
        }
        // every block: wait for each block's row of this iteration, then
        // Kahan over its strided share of the rows and a tree over the
        // groups, in a fixed order. Seeing every slot of this iteration is
        // this iteration's grid barrier. Lane v of warp g reads value v of
        // rows g, g + 32, ...; a round re-reads only the slots not yet seen.
        {
          constexpr int kPer = (kFusedMaxBlocks + kWarps - 1) / kWarps;
          const int v = lane, grp = warp;
          float vals[kPer];
          unsigned pending = 0;
#pragma unroll
          for (int q = 0; q < kPer; ++q) {
            vals[q] = 0.f;
            if (v <= kVals && grp + q * kWarps < (int)gridDim.x) pending |= 1u << q;
          }
          unsigned spins = 0;
          for (;;) {
#pragma unroll
            for (int q = 0; q < kPer; ++q) {
              if (!((pending >> q) & 1u)) continue;
              const unsigned long long w =
                  ld_relaxed_gpu(&ws->fused_rows[buf][grp + q * kWarps][v]);
              if ((unsigned)(w >> 32) == seq) {
                vals[q] = __uint_as_float((unsigned)w);
                pending &= ~(1u << q);
              }
            }
            if (__all_sync(0xffffffffu, pending == 0u)) break;
            if (++spins > kSpinLimit ||
                ((spins & 255u) == 0u && ld_acquire_gpu(reinterpret_cast<unsigned *>(&ws->error)))) {
              if (lane == 0) {
                atomicExch(&ws->error, 1);
                s_err = 1;
              }
              break;
            }
            __nanosleep(32);
          }
          float sum = 0.f, c = 0.f;
#pragma unroll
          for (int q = 0; q < kPer; ++q) {
            float y = vals[q] - c;
            float t = sum + y;
            c = (t - sum) - y;
            sum = t;
          }
          s_red[grp][v] = sum - c;
        }
        // a wait that gave up (here or, later, in every other block) ends this
        // frame's tracking; the final status reads the workspace's flag
        __syncthreads();
        if (s_err) break;
        if (threadIdx.x < 32) {
          float y[kWarps];
#pragma unroll
          for (int w = 0; w < kWarps; ++w) y[w] = s_red[w][threadIdx.x];
#pragma unroll
          for (int span = 1; span < kWarps; span *= 2)
#pragma unroll
            for (int w = 0; w + span < kWarps; w += 2 * span) y[w] += y[w + span];
          s_tot[threadIdx.x] = y[0];
          __syncwarp();
          double minpiv = 0.0;
          float inc_rot = 0.f, inc_trans = 0.f;
          // (on success the warp also writes the new pose's rigid transforms)
          const bool ok =
              warp_solve_update(s_tot, s_pose, &minpiv, &inc_rot, &inc_trans, &s_c2w, &s_w2c);
          if (threadIdx.x == 0) {
            s_its += 1;
            s_inl = (int)s_tot[28];
            s_examined = (int)s_tot[kVals];
            s_res = (double)s_tot[27];
            s_piv = minpiv;
            if (!ok) {
              for (int i = 0; i < 16; ++i) s_pose[i] = ws->pose_init[i];
              s_stop = 1;
              pose_to_rigid(s_pose, &s_c2w, &s_w2c);
            } else if (plan.stop_rot > 0.f && inc_rot < plan.stop_rot &&
                       inc_trans < plan.stop_trans) {
              s_conv = 1;  // converged at this level
            }
          }
        }
        __syncthreads();
        ++iter_global;
        if (s_stop || s_conv) break;
      }
    }
    // ---- judge a warm-started result; replace it by plain ICP if it fails
    if (pass == 1 || !warm || s_err) break;
    __syncthreads();  // every thread has left the level loop (it reads s_stop)
    if (threadIdx.x == 0) {
      const bool keep = !s_stop && judge_keep(plan, ws->warm_pose, s_pose, s_res, s_inl, s_examined);
      s_warm = keep ? 1 : 2;
      if (!keep) {
        s_stop = 0;
        for (int i = 0; i < 16; ++i) s_pose[i] = ws->pose_init[i];
        pose_to_rigid(s_pose, &s_c2w, &s_w2c);
      }
    }
    __syncthreads();
    if (s_warm == 1) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int err = *((volatile int *)&ws->error);
    for (int i = 0; i < 16; ++i) pose[i] = err ? ws->pose_init[i] : s_pose[i];
    if (plan.hist) {
      const unsigned long long c = *plan.hist_count;
      double *dst = plan.hist + (size_t)(c % (unsigned long long)plan.hist_cap) * 16;
      for (int i = 0; i < 16; ++i) dst[i] = err ? ws->pose_init[i] : s_pose[i];
      *plan.hist_count = c + 1;
    }
    ws->iterations = s_its;
    if (stats) {
      stats->status = err ? 2 : (s_stop ? 1 : 0);
      stats->inliers = s_inl;
      stats->iterations = s_its;
      stats->warm = warm ? s_warm : 0;
      stats->residual_sq = s_res;
      stats->min_pivot = s_piv;
    }
  }
}

// Start of a frame's tracking: the starting pose (with the optional prior
// increment applied; the caller's pose buffer is left as it is until the
// result is written), the optional warm start (`warm`, a device FP64 pose),
// cleared flags. It reads only the pose of the previous frame, so a tracker
// step runs it on a graph branch beside the fusion.
__global__ void k_icp_begin(double *pose, IcpWorkspace *ws, of_icp_stats_t *stats,
                            const double *warm) {
  // a new epoch: no slot carries this frame's sequence numbers yet. Slots are
  // cleared when the epoch wraps (every 2^19 frames), so an old slot never
  // matches a new number.
  // (and on a workspace's first use, whatever its memory held)
  const bool fresh = ws->magic != kWorkspaceMagic;
  const unsigned epoch = fresh ? 1u : (ws->epoch + 1u) & kEpochMask;
  if (epoch == 0u || fresh) {
    unsigned long long *rows = &ws->fused_rows[0][0][0];
    for (int i = threadIdx.x; i < 2 * kFusedMaxBlocks * 32; i += blockDim.x) rows[i] = 0ull;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  ws->epoch = epoch == 0u ? 1u : epoch;
  ws->magic = kWorkspaceMagic;
  double P[16];
  for (int i = 0; i < 16; ++i) P[i] = pose[i];
  if (ws->has_prior) {
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) {
        double a = 0.0;
        for (int k = 0; k < 4; ++k) a += ws->prior[4 * i + k] * pose[4 * k + j];
        P[4 * i + j] = a;
      }
    ws->has_prior = 0;  // a prior applies to one frame
  }
  for (int i = 0; i < 16; ++i) ws->pose_init[i] = P[i];
  ws->has_warm = warm != nullptr;
  if (warm)
    for (int i = 0; i < 16; ++i) ws->warm_pose[i] = warm[i];
  ws->ticket = 0;
  ws->stop = 0;
  ws->iterations = 0;
  ws->error = 0;
  ws->bar_count = 0;
  if (stats) {
    stats->status = 0;
    stats->inliers = 0;
    stats->iterations = 0;
    stats->warm = 0;
    stats->residual_sq = 0.0;
    stats->min_pivot = 0.0;
  }
}

int icp_blocks(int npx) {
  int g = (npx + kIcpThreads - 1) / kIcpThreads;
  return g < 1 ? 1 : (g > kIcpMaxBlocks ? kIcpMaxBlocks : g);
}

}  // namespace

size_t of_icp_workspace_size() { return sizeof(IcpWorkspace); }

extern "C" of_status_t of_icp_workspace_hold_barrier(void *d_workspace, int32_t extra,
                                                     of_stream_t stream) {
  if (!d_workspace || extra < 0 || extra > 1024) return OF_ERR_INVALID_ARGUMENT;
  IcpWorkspace *ws = (IcpWorkspace *)d_workspace;
  static int values[1025];
  values[extra] = extra;
  OF_CUDA_TRY(cudaMemcpyAsync(&ws->hold_barrier, &values[extra], sizeof(int),
                              cudaMemcpyHostToDevice, (cudaStream_t)stream));
  OF_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  return OF_OK;
}

of_status_t of_icp_set_prior(void *d_workspace, const double *prior_host, cudaStream_t s) {
  IcpWorkspace *ws = (IcpWorkspace *)d_workspace;
  static const int zero = 0, one = 1;
  if (prior_host) {
    OF_CUDA_TRY(cudaMemcpyAsync(ws->prior, prior_host, 16 * sizeof(double),
                                cudaMemcpyHostToDevice, s));
    OF_CUDA_TRY(cudaMemcpyAsync(&ws->has_prior, &one, sizeof(int), cudaMemcpyHostToDevice, s));
  } else {
    OF_CUDA_TRY(cudaMemcpyAsync(&ws->has_prior, &zero, sizeof(int), cudaMemcpyHostToDevice, s));
  }
  return OF_OK;
}

extern "C" of_status_t of_icp_workspace_bytes(const of_camera_t *cam, size_t *bytes) {
  if (!of_camera_valid(cam) || !bytes) return OF_ERR_INVALID_ARGUMENT;
  *bytes = sizeof(IcpWorkspace);
  return OF_OK;
}

static bool icp_params_ok(const of_icp_params_t *p) {
  if (!p || p->levels < 1 || p->levels > kMaxLevels) return false;
  for (int l = 0; l < p->levels; ++l)
    if (p->iters[l] < 0 || p->iters[l] > 1000) return false;
  return p->dist_thresh_mm > 0.f;
}

// Launch shape of the fused kernel on the current device: every block
// co-resident (cooperative launch), with room in shared memory for the
// block's slice of the finest level's model points (up to kMaxCachePts).
struct FusedShape {
  int grid;       // co-resident blocks (may exceed kFusedMaxBlocks: then refused)
  int cache_pts;
  size_t smem;
};
static of_status_t fused_shape(const of_camera_t *cam, FusedShape *fs) {
  constexpr int kMaxDevices = 64;
  static int grid_of[kMaxDevices] = {};
  static std::mutex mu;
  int dev = 0;
  OF_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return OF_ERR_INVALID_ARGUMENT;
  const int max_smem = kMaxCachePts * 2 * (int)sizeof(float4);
  // The shared-memory opt-in belongs to the function in the current context:
  // it is set on every call (a host-side call), so that a context created
  // after cudaDeviceReset gets it too. The grid depends only on the device.
  OF_CUDA_TRY(cudaFuncSetAttribute((const void *)k_icp_fused,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
  {
    std::lock_guard<std::mutex> lock(mu);
    if (grid_of[dev] == 0) {
      int sms = 0, per_sm = 0;
      OF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      OF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_icp_fused,
                                                                kFusedThreads, max_smem));
      grid_of[dev] = sms * (per_sm < 1 ? 1 : per_sm);
    }
    fs->grid = grid_of[dev];
  }
  const long npx = (long)cam->width * cam->height;
  const long per_block = ((npx + 31) / 32 + fs->grid - 1) / fs->grid * 32;
  fs->cache_pts = (int)(per_block < kMaxCachePts ? per_block : kMaxCachePts);
  fs->smem = (size_t)fs->cache_pts * 2 * sizeof(float4);
  return OF_OK;
}

// The start of a frame's tracking on `s` (k_icp_begin): it must precede the
// frame's fused launch.
of_status_t of_icp_begin_launch(double *pose, void *d_ws, of_icp_stats_t *stats,
                                const double *d_warm, cudaStream_t s) {
  k_icp_begin<<<1, 32, 0, s>>>(pose, (IcpWorkspace *)d_ws, stats, d_warm);
  return of_launch_status();
}

// The fused launch of one frame (`begin`: preceded by the begin kernel on
// the same stream; else a begin launch made elsewhere, e.g. on a tracker
// step's graph branch, must precede it).
static of_status_t icp_fused_launch(const of_camera_t *cam, const of_icp_params_t *ip,
                                    const void *d_frame, const void *d_model, double *pose,
                                    void *d_ws, of_icp_stats_t *stats, cudaStream_t s,
                                    const double *d_warm, double *d_hist,
                                    unsigned long long *d_hist_count, int hist_cap, bool begin) {
  of_pyramid_layout_t lay;
  of_status_t st = of_pyramid_layout(cam, ip->levels, &lay);
  if (st != OF_OK) return st;
  IcpWorkspace *ws = (IcpWorkspace *)d_ws;
  FusedShape fs;
  st = fused_shape(cam, &fs);
  if (st != OF_OK) return st;
  if (fs.grid > kFusedMaxBlocks) return OF_ERR_TOO_LARGE;
  IcpPlan plan;
  memset(&plan, 0, sizeof(plan));
  plan.levels = ip->levels;
  plan.cache_pts = fs.cache_pts;
  plan.dist_thresh = ip->dist_thresh_mm;
  plan.normal_thresh = ip->normal_thresh;
  plan.stop_rot = ip->stop_rot_rad;
  plan.stop_trans = ip->stop_trans_mm;
  plan.judge_rms = ip->judge_max_rms_mm;
  plan.judge_frac = ip->judge_min_inlier_frac;
  plan.judge_rot = ip->judge_max_rot_rad;
  plan.judge_trans = ip->judge_max_trans_mm;
  plan.warm_levels = (ip->warm_levels > 0 && ip->warm_levels < ip->levels) ? ip->warm_levels
                                                                          : ip->levels;
  if (d_hist && d_hist_count && hist_cap > 0) {
    plan.hist = d_hist;
    plan.hist_count = d_hist_count;
    plan.hist_cap = hist_cap;
  }
  for (int l = 0; l < ip->levels; ++l) {
    of_camera_t cl = camera_level(*cam, l);
    plan.lv[l].cam = make_cam(cl);
    plan.lv[l].frame = (const float4 *)((const char *)d_frame + lay.points_offset[l]);
    plan.lv[l].model = (const float4 *)((const char *)d_model + lay.points_offset[l]);
    plan.lv[l].mw = cl.width;
    plan.lv[l].mh = cl.height;
    plan.lv[l].iters = ip->iters[l];
  }
  if (begin) {
    st = of_icp_begin_launch(pose, ws, stats, d_warm, s);
    if (st != OF_OK) return st;
  }
  void *args[] = {&plan, &pose, &ws, &stats};
  OF_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)k_icp_fused, dim3(fs.grid),
                                          dim3(kFusedThreads), args, fs.smem, s));
  return OF_OK;
}

// Launches the whole coarse-to-fine ICP of one frame: a begin kernel and one
// cooperative launch of the fused kernel.
of_status_t of_icp_launch(const of_camera_t *cam, const of_icp_params_t *ip, const void *d_frame,
                          const void *d_model, double *pose, void *d_ws, of_icp_stats_t *stats,
                          cudaStream_t s, const double *d_warm, double *d_hist,
                          unsigned long long *d_hist_count, int hist_cap) {
  return icp_fused_launch(cam, ip, d_frame, d_model, pose, d_ws, stats, s, d_warm, d_hist,
                          d_hist_count, hist_cap, true);
}

// The fused launch alone, after the frame's begin launch (made on a tracker
// step's graph branch).
of_status_t of_icp_fused_launch(const of_camera_t *cam, const of_icp_params_t *ip,
                                const void *d_frame, const void *d_model, double *pose, void *d_ws,
                                of_icp_stats_t *stats, cudaStream_t s, double *d_hist,
                                unsigned long long *d_hist_count, int hist_cap) {
  return icp_fused_launch(cam, ip, d_frame, d_model, pose, d_ws, stats, s, nullptr, d_hist,
                          d_hist_count, hist_cap, false);
}

extern "C" of_status_t of_icp_track(const of_camera_t *cam, const of_icp_params_t *ip,
                                    const void *d_frame, const void *d_model, double *pose,
                                    void *d_ws, of_icp_stats_t *stats, of_stream_t s) {
  OF_RANGE("of_icp_track");
  if (!of_camera_valid(cam) || !icp_params_ok(ip) || !d_frame || !d_model || !pose || !d_ws)
    return OF_ERR_INVALID_ARGUMENT;
  return of_icp_launch(cam, ip, d_frame, d_model, pose, d_ws, stats, (cudaStream_t)s, nullptr,
                       nullptr, nullptr, 0);
}

extern "C" of_status_t of_icp_track_warm(const of_camera_t *cam, const of_icp_params_t *ip,
                                         const void *d_frame, const void *d_model, double *pose,
                                         const double *d_warm_pose, void *d_ws,
                                         of_icp_stats_t *stats, of_stream_t s) {
  OF_RANGE("of_icp_track_warm");
  if (!of_camera_valid(cam) || !icp_params_ok(ip) || !d_frame || !d_model || !pose ||
      !d_warm_pose || !d_ws)
    return OF_ERR_INVALID_ARGUMENT;
  return of_icp_launch(cam, ip, d_frame, d_model, pose, d_ws, stats, (cudaStream_t)s, d_warm_pose,
                       nullptr, nullptr, 0);
}

extern "C" of_status_t of_icp_system(const of_camera_t *cam, const of_icp_params_t *ip,
                                     int32_t level, const void *d_frame, const void *d_model,
                                     const double *pose, void *d_ws, float *d_system,
                                     of_stream_t stream) {
  if (!of_camera_valid(cam) || !icp_params_ok(ip) || !d_frame || !d_model || !pose || !d_ws ||
      !d_system || level < 0 || level >= ip->levels)
    return OF_ERR_INVALID_ARGUMENT;
  of_pyramid_layout_t lay;
  of_status_t st = of_pyramid_layout(cam, ip->levels, &lay);
  if (st != OF_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  IcpWorkspace *ws = (IcpWorkspace *)d_ws;
  OF_CUDA_TRY(cudaMemsetAsync(&ws->ticket, 0, sizeof(unsigned int), s));
  of_camera_t cl = camera_level(*cam, level);
  Cam c = make_cam(cl);
  const float4 *fr = (const float4 *)((const char *)d_frame + lay.points_offset[level]);
  const float4 *md = (const float4 *)((const char *)d_model + lay.points_offset[level]);
  int g = icp_blocks(cl.width * cl.height);
  k_icp_iter<kModeSystem><<<g, kIcpThreads, 0, s>>>(md, cl.width, cl.height, fr, c,
                                                    ip->dist_thresh_mm, ip->normal_thresh,
                                                    (double *)pose, ws, nullptr, d_system);
  return of_launch_status();
}

namespace {
// One warp: the tracking kernels' FP64 solve and SE(3) update on a system of
// 29 sums, pose in place (unchanged when the system is singular).
__global__ void __launch_bounds__(32) k_icp_solve_step(const float *__restrict__ sys, double *pose,
                                                       of_icp_stats_t *stats) {
  __shared__ float s_tot[32];
  __shared__ double s_pose[16];
  const int lane = threadIdx.x;
  s_tot[lane] = lane < kVals ? sys[lane] : 0.f;
  if (lane < 16) s_pose[lane] = pose[lane];
  __syncwarp();
  double minpiv = 0.0;
  float inc_rot = 0.f, inc_trans = 0.f;
  const bool ok = warp_solve_update(s_tot, s_pose, &minpiv, &inc_rot, &inc_trans);
  if (ok && lane < 16) pose[lane] = s_pose[lane];
  if (lane == 0 && stats) {
    stats->status = ok ? 0 : 1;
    stats->inliers = (int)s_tot[28];
    stats->iterations = 1;
    stats->warm = 0;
    stats->residual_sq = (double)s_tot[27];
    stats->min_pivot = minpiv;
  }
}
}  // namespace

extern "C" of_status_t of_icp_solve_step(const float *d_system, double *d_pose,
                                         of_icp_stats_t *d_stats, of_stream_t stream) {
  if (!d_system || !d_pose) return OF_ERR_INVALID_ARGUMENT;
  k_icp_solve_step<<<1, 32, 0, (cudaStream_t)stream>>>(d_system, d_pose, d_stats);
  return of_launch_status();
}

// ---------------------------------------------------------------------------
// Tracking without a caller-provided workspace.
//
// For callers that cannot allocate device memory while they run (hosts that own
// every device allocation up front, such as plugin hosts with a fixed memory
// budget or real-time loops where cudaMalloc's implicit synchronisation and a
// possible failure mid-session are not acceptable), of_icp_track_static uses a
// workspace that lives in this file-scope array instead. Every GPU that loads
// the library holds it (sizeof(IcpWorkspace), about 186 KB) until the process
// exits. It holds the per-block partial sums of at most kFusedMaxBlocks
// cooperating blocks.
static __device__ __align__(256) unsigned char g_static_icp_ws[sizeof(IcpWorkspace)];

// Device address of the array in the current context. In host code the
// array's name is only a host-side stand-in, so the address is looked up with
// cudaGetSymbolAddress, which allocates nothing. It is looked up on every call
// rather than cached: after cudaDeviceReset, or in another context on the same
// device, the module is loaded again and the array may move. The array starts
// zeroed when the module loads, and k_icp_begin clears the partial-sum rows of
// a workspace that does not carry its magic word yet, so no clearing call is
// needed here (and nothing here blocks a stream or breaks a capture).
static of_status_t static_icp_workspace(void **out) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_static_icp_ws);
  if (e != cudaSuccess || !p) return of_set_cuda_error(e != cudaSuccess ? e : cudaErrorUnknown);
  *out = p;
  return OF_OK;
}

extern "C" of_status_t of_icp_track_static(const of_camera_t *cam, const of_icp_params_t *ip,
                                           const void *d_frame, const void *d_model,
                                           double *pose, of_icp_stats_t *stats,
                                           of_stream_t stream) {
  if (!of_camera_valid(cam) || !icp_params_ok(ip) || !d_frame || !d_model || !pose)
    return OF_ERR_INVALID_ARGUMENT;
  // the array holds partials for kFusedMaxBlocks blocks: a device whose
  // co-resident grid would need more is refused
  FusedShape fs;
  of_status_t sh = fused_shape(cam, &fs);
  if (sh != OF_OK) return sh;
  if (fs.grid > kFusedMaxBlocks) return OF_ERR_TOO_LARGE;
  void *ws = nullptr;
  of_status_t st = static_icp_workspace(&ws);
  if (st != OF_OK) return st;
  return of_icp_launch(cam, ip, d_frame, d_model, pose, ws, stats, (cudaStream_t)stream, nullptr,
                       nullptr, nullptr, 0);
}

// ------------------------------------------------------------ batched ICP --
//
// Multi-level ICP of many independent streams in one persistent launch: each
// thread-block cluster of kBatchCtas CTAs tracks one stream at a time and
// takes the next stream from an atomic ticket over a longest-first order.
// Per iteration every CTA associates its share of the level's model pixels
// (thread g of the cluster takes pixels g, g + kBatchCtas * kBatchThreads,
// ...), reduces its rows (warp recursive halving, then a tree over warps),
// and pushes its 30-value row into every CTA's shared memory
// (double-buffered by iteration parity); after one cluster barrier every CTA
// sums the kBatchCtas rows in the same order and solves the same 6x6 system,
// so all hold the same pose. The only waits are hardware cluster barriers.
// The per-pixel arithmetic (association, inlier tests, rows, FP64 solve and
// composition) is the single-stream kernel's; the summation order differs.
#include <cooperative_groups.h>

namespace {

namespace cg = cooperative_groups;

constexpr int kBatchCtas = 8;
constexpr int kBatchThreads = 512;
constexpr int kBatchWarps = kBatchThreads / 32;

struct IcpJob {
  IcpLevel lv[kMaxLevels];
  int levels;
  double *pose;
  of_icp_stats_t *stats;
};

__global__ void __cluster_dims__(kBatchCtas, 1, 1) __launch_bounds__(kBatchThreads, 1)
    k_icp_batch(const IcpJob *__restrict__ jobs, const int *__restrict__ order, int njobs,
                unsigned int *ticket, float dist_thresh, float normal_thresh, float stop_rot,
                float stop_trans) {
  __shared__ double s_pose[16], s_init[16];
  __shared__ Rigid s_c2w, s_w2c;
  __shared__ float s_red[kBatchWarps][32];
  __shared__ float s_part[2][kBatchCtas][32];
  __shared__ float s_tot[32];
  __shared__ int s_job, s_stop, s_conv, s_its, s_inl;
  __shared__ double s_res, s_piv;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float dist2 = dist_thresh * dist_thresh;
  for (;;) {
    if (rank == 0 && threadIdx.x == 0) {
      const unsigned t = atomicAdd(ticket, 1u);
      const int job = t < (unsigned)njobs ? __ldg(order + t) : -1;
      for (int r = 0; r < kBatchCtas; ++r) *cluster.map_shared_rank(&s_job, r) = job;
    }
    cluster.sync();
    const int job = s_job;
    // every CTA has read the job before CTA 0 may hand out the next one
    cluster.sync();
    if (job < 0) break;
    const IcpJob &J = jobs[job];
    if (threadIdx.x < 16) {
      s_pose[threadIdx.x] = J.pose[threadIdx.x];
      s_init[threadIdx.x] = J.pose[threadIdx.x];
    }
    if (threadIdx.x == 0) {
      s_stop = 0; s_conv = 0; s_its = 0; s_inl = 0; s_res = 0.0; s_piv = 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) pose_to_rigid(s_pose, &s_c2w, &s_w2c);
    __syncthreads();
    int iter = 0;
    for (int l = J.levels - 1; l >= 0 && !s_stop; --l) {
      const IcpLevel L = J.lv[l];
      const int npx = L.mw * L.mh;
      __syncthreads();  // every thread has read the previous level's exit flag
      if (threadIdx.x == 0) s_conv = 0;
      __syncthreads();
      for (int it = 0; it < L.iters; ++it) {
        float acc[kVals];
        float examined = 0.f;
#pragma unroll
        for (int v = 0; v < kVals; ++v) acc[v] = 0.f;
        constexpr int kStride = kBatchCtas * kBatchThreads;
        for (int p = rank * kBatchThreads + threadIdx.x; p < npx; p += 2 * kStride) {
          const int p2 = p + kStride;
          const float4 sA = __ldg(L.model + 2 * p), nA = __ldg(L.model + 2 * p + 1);
          float4 sB = make_float4(0.f, 0.f, 0.f, 0.f), nB = sB;
          if (p2 < npx) { sB = __ldg(L.model + 2 * p2); nB = __ldg(L.model + 2 * p2 + 1); }
          const int qA = (sA.w != 0.f && nA.w != 0.f) ? associate(s_w2c, L.cam, sA) : -1;
          const int qB = (sB.w != 0.f && nB.w != 0.f) ? associate(s_w2c, L.cam, sB) : -1;
          float4 dA = make_float4(0.f, 0.f, 0.f, 0.f), cA = dA, dB = dA, cB = dA;
          if (qA >= 0) { dA = __ldg(L.frame + 2 * qA); cA = __ldg(L.frame + 2 * qA + 1); }
          if (qB >= 0) { dB = __ldg(L.frame + 2 * qB); cB = __ldg(L.frame + 2 * qB + 1); }
          if (qA >= 0) {
            examined += 1.f;
            try_row(acc, s_c2w, sA, nA, dA, cA, dist2, normal_thresh);
          }
          if (qB >= 0) {
            examined += 1.f;
            try_row(acc, s_c2w, sB, nB, dB, cB, dist2, normal_thresh);
          }
        }
        // this CTA's row: recursive halving across the warp, a tree over warps
        {
          float r[32];
#pragma unroll
          for (int v = 0; v < 32; ++v) r[v] = v < kVals ? acc[v] : (v == kVals ? examined : 0.f);
#pragma unroll
          for (int sft = 16; sft >= 1; sft >>= 1) {
            const bool upper = (lane & sft) != 0;
#pragma unroll
            for (int i = 0; i < sft; ++i) {
              float send = upper ? r[i] : r[i + sft];
              float keep = upper ? r[i + sft] : r[i];
              r[i] = keep + __shfl_xor_sync(0xffffffffu, send, sft);
            }
          }
          s_red[warp][lane] = r[0];
        }
        __syncthreads();
        const int buf = iter & 1;
        if (warp == 0) {
          float y[kBatchWarps];
#pragma unroll
          for (int w = 0; w < kBatchWarps; ++w) y[w] = s_red[w][lane];
#pragma unroll
          for (int span = 1; span < kBatchWarps; span *= 2)
#pragma unroll
            for (int w = 0; w + span < kBatchWarps; w += 2 * span) y[w] += y[w + span];
#pragma unroll
          for (int r = 0; r < kBatchCtas; ++r) cluster.map_shared_rank(&s_part[buf][rank][0], r)[lane] = y[0];
        }
        cluster.sync();
        if (warp == 0) {
          float y[kBatchCtas];
#pragma unroll
          for (int r = 0; r < kBatchCtas; ++r) y[r] = s_part[buf][r][lane];
#pragma unroll
          for (int span = 1; span < kBatchCtas; span *= 2)
#pragma unroll
            for (int r = 0; r + span < kBatchCtas; r += 2 * span) y[r] += y[r + span];
          s_tot[lane] = y[0];
          __syncwarp();
          double minpiv = 0.0;
          float inc_rot = 0.f, inc_trans = 0.f;
          const bool ok = warp_solve_update(s_tot, s_pose, &minpiv, &inc_rot, &inc_trans);
          if (lane == 0) {
            s_its += 1;
            s_inl = (int)s_tot[28];
            s_res = (double)s_tot[27];
            s_piv = minpiv;
            if (!ok) {
              for (int i = 0; i < 16; ++i) s_pose[i] = s_init[i];
              s_stop = 1;
            } else if (stop_rot > 0.f && inc_rot < stop_rot && inc_trans < stop_trans) {
              s_conv = 1;
            }
            pose_to_rigid(s_pose, &s_c2w, &s_w2c);
          }
        }
        __syncthreads();
        ++iter;
        if (s_stop || s_conv) break;
      }
    }
    if (rank == 0 && threadIdx.x == 0) {
      for (int i = 0; i < 16; ++i) J.pose[i] = s_pose[i];
      if (J.stats) {
        J.stats->status = s_stop ? 1 : 0;
        J.stats->inliers = s_inl;
        J.stats->iterations = s_its;
        J.stats->warm = 0;
        J.stats->residual_sq = s_res;
        J.stats->min_pivot = s_piv;
      }
    }
  }
}

}  // namespace

namespace of {

struct IcpBatch {
  int n = 0;
  float dist, nthr, stop_rot, stop_trans;
  IcpJob *jobs = nullptr;
  int *order = nullptr;
  unsigned int *ticket = nullptr;
};

void icp_batch_destroy(IcpBatch *b) {
  if (!b) return;
  cudaFree(b->jobs);
  cudaFree(b->order);
  cudaFree(b->ticket);
  delete b;
}

// Clusters of the batched ICP that fit on the device at once.
int icp_batch_max_clusters() {
  static int cached = 0;
  if (cached > 0) return cached;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kBatchCtas * kSmCount / kBatchCtas);
  cfg.blockDim = dim3(kBatchThreads);
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = kBatchCtas;
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, (void *)k_icp_batch, &cfg) != cudaSuccess || n < 1) {
    cudaGetLastError();
    n = kSmCount / kBatchCtas;
  }
  cached = n;
  return n;
}

of_status_t icp_batch_create(const BatchStream *s, int n, const BatchParams &p, IcpBatch **out) {
  const of_icp_params_t *ip = &p.icp;
  if (n < 1 || !icp_params_ok(ip)) return OF_ERR_INVALID_ARGUMENT;
  IcpBatch *b = new IcpBatch();
  b->n = n;
  b->dist = ip->dist_thresh_mm;
  b->nthr = ip->normal_thresh;
  b->stop_rot = ip->stop_rot_rad;
  b->stop_trans = ip->stop_trans_mm;
  IcpJob *jobs = new IcpJob[n];
  int *order = new int[n + 1];
  double *cost = new double[n];
  of_status_t st = OF_OK;
  for (int i = 0; i < n && st == OF_OK; ++i) {
    of_pyramid_layout_t lay;
    st = of_pyramid_layout(&s[i].cam, ip->levels, &lay);
    memset(&jobs[i], 0, sizeof(IcpJob));
    jobs[i].levels = ip->levels;
    jobs[i].pose = s[i].pose;
    jobs[i].stats = s[i].stats;
    cost[i] = 0.0;
    for (int l = 0; l < ip->levels; ++l) {
      const of_camera_t cl = camera_level(s[i].cam, l);
      IcpLevel &L = jobs[i].lv[l];
      L.cam = make_cam(cl);
      L.frame = (const float4 *)((const char *)s[i].frame + lay.points_offset[l]);
      L.model = (const float4 *)((const char *)s[i].model + lay.points_offset[l]);
      L.mw = cl.width;
      L.mh = cl.height;
      L.iters = ip->iters[l];
      cost[i] += (double)cl.width * cl.height * ip->iters[l];
    }
  }
  // longest first (ties by index), so the last streams taken are the shortest
  for (int i = 0; i < n; ++i) order[i] = i;
  for (int i = 1; i < n; ++i)
    for (int k = i; k > 0 && (cost[order[k]] > cost[order[k - 1]] ||
                              (cost[order[k]] == cost[order[k - 1]] && order[k] < order[k - 1]));
         --k) {
      const int t = order[k]; order[k] = order[k - 1]; order[k - 1] = t;
    }
  order[n] = 0;
  if (st == OF_OK) st = upload_jobs(jobs, order, n, &b->jobs, &b->order);
  if (st == OF_OK) {
    cudaError_t e = cudaMalloc(&b->ticket, sizeof(unsigned int));
    if (e != cudaSuccess) st = of_set_cuda_error(e);
  }
  delete[] jobs;
  delete[] order;
  delete[] cost;
  if (st != OF_OK) {
    icp_batch_destroy(b);
    return st;
  }
  *out = b;
  return OF_OK;
}

of_status_t icp_batch_launch(const IcpBatch *b, const BatchKnobs &k, cudaStream_t s) {
  const int maxc = icp_batch_max_clusters();
  int clusters = k.icp_clusters > 0 ? k.icp_clusters : maxc;
  if (clusters > maxc) clusters = maxc;
  if (clusters > b->n) clusters = b->n;
  OF_CUDA_TRY(cudaMemsetAsync(b->ticket, 0, sizeof(unsigned int), s));
  k_icp_batch<<<clusters * kBatchCtas, kBatchThreads, 0, s>>>(b->jobs, b->order, b->n, b->ticket,
                                                            b->dist, b->nthr, b->stop_rot,
                                                            b->stop_trans);
  return of_launch_status();
}

}  // namespace of
