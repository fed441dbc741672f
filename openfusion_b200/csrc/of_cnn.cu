// of_cnn.cu -- the learned ICP warm start: a small BF16 CNN that maps a pair
// of 80x60 depth images (previous, current frame) to the 6-DoF motion between
// them, with its own forward, backward and Adam kernels.
//
// No reference counterpart (the reference tracks with plain ICP only,
// Source/src/ICP.cpp:84-182). Network (NCHW, batch b):
//   in  2 x 60 x 80   previous depth (m) minus its mean; current - previous
//   c1  conv 5x5 s2 p2  2 -> 16, ReLU    16 x 30 x 40
//   c2  conv 3x3 s2 p1 16 -> 32, ReLU    32 x 15 x 20
//   c3  conv 3x3 s2 p1 32 -> 64, ReLU    64 x  8 x 10
//   c4  conv 3x3 s2 p1 64 -> 128, ReLU  128 x  4 x  5
//   f1  2560 -> 160, ReLU
//   f2  160 -> 6   (rotation vector x 10 rad^-1, translation / 100 mm)
// 508,534 parameters. Mixed precision: weights and stored activations in
// BF16, every sum in FP32, gradients, master weights and Adam moments in
// FP32. Every reduction runs in a fixed order (no atomics), so a training run
// is reproducible bit for bit.
#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include "of_common.cuh"

namespace cg = cooperative_groups;

namespace {

using bf16 = __nv_bfloat16;

struct ConvSpec {
  int ci, co, k, s, p, hi, wi, ho, wo;
};
constexpr ConvSpec kConv[4] = {{2, 16, 5, 2, 2, 60, 80, 30, 40},
                               {16, 32, 3, 2, 1, 30, 40, 15, 20},
                               {32, 64, 3, 2, 1, 15, 20, 8, 10},
                               {64, 128, 3, 2, 1, 8, 10, 4, 5}};
constexpr int kF1In = 128 * 4 * 5, kF1Out = 160, kF2Out = 6;
constexpr int kInH = 60, kInW = 80;

constexpr long conv_w(int l) { return (long)kConv[l].co * kConv[l].ci * kConv[l].k * kConv[l].k; }
// parameter offsets (floats): [w0 b0 w1 b1 w2 b2 w3 b3 wf1 bf1 wf2 bf2]
constexpr long kOffW0 = 0, kOffB0 = kOffW0 + conv_w(0);
constexpr long kOffW1 = kOffB0 + 16, kOffB1 = kOffW1 + conv_w(1);
constexpr long kOffW2 = kOffB1 + 32, kOffB2 = kOffW2 + conv_w(2);
constexpr long kOffW3 = kOffB2 + 64, kOffB3 = kOffW3 + conv_w(3);
constexpr long kOffF1 = kOffB3 + 128, kOffBF1 = kOffF1 + (long)kF1In * kF1Out;
constexpr long kOffF2 = kOffBF1 + kF1Out, kOffBF2 = kOffF2 + (long)kF1Out * kF2Out;
constexpr long kParams = kOffBF2 + kF2Out;
static_assert(kParams == 508534, "parameter count");

// per-sample activation sizes: input, c1..c4, f1 (BF16) and the output (FP32)
constexpr long kActIn = 2L * kInH * kInW;
constexpr long kAct[4] = {16L * 30 * 40, 32L * 15 * 20, 64L * 8 * 10, 128L * 4 * 5};

// Workspace (per batch b): BF16 activations a1..a4, f1; FP32 output; FP32
// gradients g1..g4, gf1, gout (activation-sized).
struct CnnWs {
  bf16 *a[4];
  bf16 *f1;
  float *out;
  float *g[4];
  float *gf1;
  float *gout;
  float *loss;  // [b] per-sample losses, then their sum at [b]
  float *part;  // split-K partial tiles of the tensor-core GEMMs
  size_t total;
};
size_t mma_part_floats(int b);
inline size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }
CnnWs ws_layout(void *base, int b) {
  CnnWs w;
  char *p = (char *)base;
  size_t off = 0;
  auto take = [&](size_t bytes) { char *q = p ? p + off : nullptr; off += a256(bytes); return q; };
  for (int l = 0; l < 4; ++l) w.a[l] = (bf16 *)take((size_t)b * kAct[l] * sizeof(bf16));
  w.f1 = (bf16 *)take((size_t)b * kF1Out * sizeof(bf16));
  w.out = (float *)take((size_t)b * kF2Out * sizeof(float));
  for (int l = 0; l < 4; ++l) w.g[l] = (float *)take((size_t)b * kAct[l] * sizeof(float));
  w.gf1 = (float *)take((size_t)b * kF1Out * sizeof(float));
  w.gout = (float *)take((size_t)b * kF2Out * sizeof(float));
  w.loss = (float *)take((size_t)(b + 1) * sizeof(float));
  w.part = (float *)take(mma_part_floats(b) * sizeof(float));
  w.total = off;
  return w;
}

__device__ __forceinline__ float bf(bf16 x) { return __bfloat162float(x); }

// ---------------------------------------------------------------- input --

// Step 1 of the network input, one thread per (pair, frame, cell): the mean
// of the valid depths of the cell's k x k pixels (k = W / 80 = H / 60), in
// metres (0 for an empty cell).
__global__ void __launch_bounds__(256) k_cnn_cells(const uint16_t *__restrict__ prev,
                                                   const uint16_t *__restrict__ cur, int w,
                                                   int h, long pair_stride, int batch,
                                                   float *__restrict__ cells) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)batch * kActIn) return;
  const int c = (int)(i % (kInH * kInW)), f = (int)((i / (kInH * kInW)) % 2);
  const int b = (int)(i / kActIn);
  const int k = w / kInW;
  const int cy = c / kInW, cx = c % kInW;
  const uint16_t *src = (f ? cur : prev) + (size_t)b * pair_stride;
  float acc = 0.f;
  int n = 0;
  for (int y = 0; y < k; ++y)
    for (int x = 0; x < k; ++x) {
      const uint16_t d = __ldg(src + (size_t)(cy * k + y) * w + cx * k + x);
      if (d) { acc += (float)d; ++n; }
    }
  cells[i] = n ? acc / (1000.f * n) : 0.f;
}

// Step 2, one block per pair: channel 0 = previous cell minus the mean of
// the previous frame's non-empty cells (fixed-order tree), channel 1 =
// current cell minus previous cell (where both are non-empty); 0 elsewhere.
// Stored in BF16: the difference channel keeps the small motion signal at
// full relative precision (a depth near 2 m is only good to ~8 mm in BF16).
__global__ void __launch_bounds__(256) k_cnn_center(const float *__restrict__ cells,
                                                    bf16 *__restrict__ in) {
  __shared__ float s_sum[256];
  __shared__ int s_cnt[256];
  const int b = blockIdx.x;
  const float *cp = cells + (size_t)b * kActIn;
  float lsum = 0.f;
  int lcnt = 0;
  for (int c = threadIdx.x; c < kInH * kInW; c += blockDim.x) {
    const float v = cp[c];
    if (v > 0.f) { lsum += v; ++lcnt; }
  }
  s_sum[threadIdx.x] = lsum;
  s_cnt[threadIdx.x] = lcnt;
  __syncthreads();
  for (int span = blockDim.x / 2; span > 0; span >>= 1) {
    if ((int)threadIdx.x < span) {
      s_sum[threadIdx.x] += s_sum[threadIdx.x + span];
      s_cnt[threadIdx.x] += s_cnt[threadIdx.x + span];
    }
    __syncthreads();
  }
  const float mu = s_cnt[0] ? s_sum[0] / (float)s_cnt[0] : 0.f;
  for (int c = threadIdx.x; c < kInH * kInW; c += blockDim.x) {
    const float p = cp[c], q = cp[kInH * kInW + c];
    in[(size_t)b * kActIn + c] = __float2bfloat16_rn(p > 0.f ? p - mu : 0.f);
    in[(size_t)b * kActIn + kInH * kInW + c] = __float2bfloat16_rn(p > 0.f && q > 0.f ? q - p : 0.f);
  }
}

// ---------------------------------------------------------------- convs --

// out[b, co, oy, ox] = relu(bias[co] + sum_{ci, ky, kx} w[co, ci, ky, kx] in[b, ci, iy, ix])
// for small batches (inference): one warp per output,
// the ci x K x K taps dealt to the lanes in a fixed order, then a shuffle
// tree; enough parallelism for a single pair.
template <int K, int S, int P>
__global__ void __launch_bounds__(256) k_conv_fwd_warp(const bf16 *__restrict__ in,
                                                       const bf16 *__restrict__ wt,
                                                       const float *__restrict__ bias, ConvSpec c,
                                                       int batch, bf16 *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  const long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= (long)batch * c.co * c.ho * c.wo) return;  // warp-uniform
  const int ox = (int)(i % c.wo), oy = (int)((i / c.wo) % c.ho);
  const int co = (int)((i / ((long)c.wo * c.ho)) % c.co), b = (int)(i / ((long)c.wo * c.ho * c.co));
  const bf16 *ib = in + (size_t)b * c.ci * c.hi * c.wi;
  const bf16 *wb = wt + (size_t)co * c.ci * K * K;
  float acc = 0.f;
  for (int tap = lane; tap < c.ci * K * K; tap += 32) {
    const int ci = tap / (K * K), ky = (tap / K) % K, kx = tap % K;
    const int iy = oy * S - P + ky, ix = ox * S - P + kx;
    if ((unsigned)iy < (unsigned)c.hi && (unsigned)ix < (unsigned)c.wi)
      acc = fmaf(bf(wb[tap]), bf(ib[((size_t)ci * c.hi + iy) * c.wi + ix]), acc);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) out[i] = __float2bfloat16_rn(fmaxf(acc + bias[co], 0.f));
}

// ------------------------------------------------------------------- fc --

// out[b, j] = act(bias[j] + sum_i w[j, i] in[b, i]); one warp per (b, j).
template <bool RELU, typename TOut>
__global__ void __launch_bounds__(256) k_fc_fwd(const bf16 *__restrict__ in,
                                                const bf16 *__restrict__ wt,
                                                const float *__restrict__ bias, int nin, int nout,
                                                int batch, TOut *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= (long)batch * nout) return;  // warp-uniform
  const int j = (int)(warp % nout), b = (int)(warp / nout);
  float acc = 0.f;
  for (int i = lane; i < nin; i += 32)
    acc = fmaf(bf(wt[(size_t)j * nin + i]), bf(in[(size_t)b * nin + i]), acc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) {
    float v = acc + bias[j];
    if (RELU) v = fmaxf(v, 0.f);
    if constexpr (sizeof(TOut) == 2) out[warp] = __float2bfloat16_rn(v);
    else out[warp] = v;
  }
}

// ------------------------------------------------- tensor-core GEMMs --
//
// The training contractions as implicit GEMMs on the tensor cores:
// D[m, n] = sum_k A(m, k) B(k, n) with A and B read through a problem
// functor that gathers them from the layer's tensors (im2col on the fly, the
// padding and the ReLU masks included). One warp computes a 16 x 32 tile of
// D, four mma n8 subtiles sharing each A fragment, over a K range:
//   - forward (BF16 weights and activations): mma.sync m16n8k16 BF16 x BF16
//     with FP32 accumulation, the products the scalar kernels form, summed in
//     another fixed order;
//   - backward (FP32 gradients): mma.sync m16n8k8 TF32 x TF32 with FP32
//     accumulation; BF16 operands are exact in TF32, an FP32 gradient is
//     rounded to TF32 (cvt.rna, relative error below 2^-11).
// Large reductions (the weight gradients sum over batch x pixels) are split
// along K over blockIdx.y; each slice writes its partial tile and a second
// kernel sums the slices in index order, so every result is reproducible bit
// for bit. Fragment layouts (PTX ISA, mma.m16n8k16 / m16n8k8, g = lane / 4,
// t = lane % 4): A row-major, B column-major, accumulators c0..c3 at
// (g, 2t), (g, 2t + 1), (g + 8, 2t), (g + 8, 2t + 1).

constexpr int kMmaWarps = 4;      // warps per CTA, one 16 x 32 tile each
constexpr int kMmaNt = 4;         // n8 subtiles per warp tile
constexpr int kMmaTileN = 8 * kMmaNt;
constexpr long kMmaSliceK = 2048; // K per split slice of a long reduction
constexpr int kMmaMaxSlices = 256;

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}
__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void mma_bf16(float *c, const uint32_t *a, const uint32_t *b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
      "{%8, %9}, {%0, %1, %2, %3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ void mma_tf32(float *c, const uint32_t *a, const uint32_t *b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
      "{%8, %9}, {%0, %1, %2, %3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Warp tile (m0, n0) over k in [k0, k1): BF16 (KS = 16) or TF32 (KS = 8).
// Elements outside [0, M) x [0, Kd) or [0, Kd) x [0, N) read as 0 (Kd: the
// reduction length of the problem).
template <class P, bool BF16>
__device__ __forceinline__ void mma_tile(const P &p, int m0, int n0, long k0, long k1,
                                         float (&c)[kMmaNt][4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  constexpr int KS = BF16 ? 16 : 8;
  const int ma = m0 + g, mb = m0 + g + 8;
  for (long k = k0; k < k1; k += KS) {
    uint32_t a[4];
    if (BF16) {
      const long ka = k + 2 * t, kb = k + 2 * t + 8;
      a[0] = pack_bf16x2(p.a(ma, ka), p.a(ma, ka + 1));
      a[1] = pack_bf16x2(p.a(mb, ka), p.a(mb, ka + 1));
      a[2] = pack_bf16x2(p.a(ma, kb), p.a(ma, kb + 1));
      a[3] = pack_bf16x2(p.a(mb, kb), p.a(mb, kb + 1));
    } else {
      a[0] = to_tf32(p.a(ma, k + t));
      a[1] = to_tf32(p.a(mb, k + t));
      a[2] = to_tf32(p.a(ma, k + t + 4));
      a[3] = to_tf32(p.a(mb, k + t + 4));
    }
#pragma unroll
    for (int j = 0; j < kMmaNt; ++j) {
      const int n = n0 + 8 * j + g;
      uint32_t b[2];
      if (BF16) {
        b[0] = pack_bf16x2(p.b(k + 2 * t, n), p.b(k + 2 * t + 1, n));
        b[1] = pack_bf16x2(p.b(k + 2 * t + 8, n), p.b(k + 2 * t + 9, n));
        mma_bf16(c[j], a, b);
      } else {
        b[0] = to_tf32(p.b(k + t, n));
        b[1] = to_tf32(p.b(k + t + 4, n));
        mma_tf32(c[j], a, b);
      }
    }
  }
}

// Grid: x over the warp tiles (kMmaWarps per CTA), y over the K slices.
// With one slice the tile goes through p.store(m, n, value); with several,
// slice s writes part[(s * M + m) * N + n] and k_mma_reduce sums them.
template <class P, bool BF16>
__global__ void __launch_bounds__(32 * kMmaWarps) k_mma(P p, float *__restrict__ part) {
  const int tiles_n = (p.N + kMmaTileN - 1) / kMmaTileN;
  const int tiles = ((p.M + 15) / 16) * tiles_n;
  const int tile = blockIdx.x * kMmaWarps + (threadIdx.x >> 5);
  if (tile >= tiles) return;  // warp-uniform
  const int m0 = (tile / tiles_n) * 16, n0 = (tile % tiles_n) * kMmaTileN;
  const long slice = (p.Kd + gridDim.y - 1) / gridDim.y;
  const long KS = BF16 ? 16 : 8;
  const long k0 = ((long)blockIdx.y * slice) / KS * KS;
  const long k1 = blockIdx.y + 1 == gridDim.y ? p.Kd : (((long)blockIdx.y + 1) * slice) / KS * KS;
  float c[kMmaNt][4] = {};
  mma_tile<P, BF16>(p, m0, n0, k0, k1, c);
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int j = 0; j < kMmaNt; ++j)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int m = m0 + g + (r >= 2 ? 8 : 0), n = n0 + 8 * j + 2 * t + (r & 1);
      if (m >= p.M || n >= p.N) continue;
      if (gridDim.y == 1) p.store(m, n, c[j][r]);
      else part[((size_t)blockIdx.y * p.M + m) * p.N + n] = c[j][r];
    }
}

template <class P>
__global__ void __launch_bounds__(256) k_mma_reduce(P p, const float *__restrict__ part,
                                                    int slices) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)p.M * p.N) return;
  float acc = 0.f;
  for (int s = 0; s < slices; ++s) acc += part[(size_t)s * p.M * p.N + i];
  p.store((int)(i / p.N), (int)(i % p.N), acc);
}

// K slices of a reduction of length K (1 when it is short).
inline int mma_slices(long K) {
  const long s = (K + kMmaSliceK - 1) / kMmaSliceK;
  return (int)(s < 1 ? 1 : (s > kMmaMaxSlices ? kMmaMaxSlices : s));
}

// Launches D = A B of problem p; `part` holds slices x M x N floats when the
// reduction is split.
template <class P, bool BF16>
void mma_launch(const P &p, float *part, int slices, cudaStream_t s) {
  const long tiles = (long)((p.M + 15) / 16) * ((p.N + kMmaTileN - 1) / kMmaTileN);
  dim3 grid((unsigned)((tiles + kMmaWarps - 1) / kMmaWarps), (unsigned)slices);
  k_mma<P, BF16><<<grid, 32 * kMmaWarps, 0, s>>>(p, part);
  if (slices > 1)
    k_mma_reduce<P><<<(unsigned)(((long)p.M * p.N + 255) / 256), 256, 0, s>>>(p, part, slices);
}

// Convolution forward: m = co, k = (ci, ky, kx), n = (b, oy, ox);
// out = relu(bias + acc) in BF16.
template <int K, int S, int P>
struct ConvFwdProb {
  const bf16 *in, *wt;
  const float *bias;
  bf16 *out;
  ConvSpec c;
  int M, N;
  long Kd;
  __device__ float a(int m, long k) const {
    return (m < M && k < Kd) ? bf(wt[(size_t)m * Kd + k]) : 0.f;
  }
  __device__ float b(long k, int n) const {
    if (n >= N || k >= Kd) return 0.f;
    const int ci = (int)(k / (K * K)), ky = (int)((k / K) % K), kx = (int)(k % K);
    const int hw = c.ho * c.wo, bb = n / hw, p = n % hw, oy = p / c.wo, ox = p % c.wo;
    const int iy = oy * S - P + ky, ix = ox * S - P + kx;
    if ((unsigned)iy >= (unsigned)c.hi || (unsigned)ix >= (unsigned)c.wi) return 0.f;
    return bf(in[(((size_t)bb * c.ci + ci) * c.hi + iy) * c.wi + ix]);
  }
  __device__ void store(int m, int n, float v) const {
    const int hw = c.ho * c.wo, bb = n / hw, p = n % hw;
    out[((size_t)bb * c.co + m) * hw + p] = __float2bfloat16_rn(fmaxf(v + bias[m], 0.f));
  }
};

// The gradient at a ReLU layer's pre-activation: gpost where act > 0.
__device__ __forceinline__ float relu_grad(const float *gpost, const bf16 *act, size_t o) {
  return (!act || bf(act[o]) > 0.f) ? gpost[o] : 0.f;
}

// Convolution input gradient: m = ci, k = (co, ky, kx), n = (b, iy, ix).
template <int K, int S, int P>
struct ConvBwdDataProb {
  const float *gpost;
  const bf16 *act, *wt;
  float *gin;
  ConvSpec c;
  int M, N;
  long Kd;
  __device__ float a(int m, long k) const {
    if (m >= M || k >= Kd) return 0.f;
    const int co = (int)(k / (K * K)), tap = (int)(k % (K * K));
    return bf(wt[((size_t)co * c.ci + m) * K * K + tap]);
  }
  __device__ float b(long k, int n) const {
    if (n >= N || k >= Kd) return 0.f;
    const int co = (int)(k / (K * K)), ky = (int)((k / K) % K), kx = (int)(k % K);
    const int hw = c.hi * c.wi, bb = n / hw, q = n % hw, iy = q / c.wi, ix = q % c.wi;
    const int ny = iy + P - ky, nx = ix + P - kx;
    if (ny < 0 || nx < 0 || ny % S || nx % S) return 0.f;
    const int oy = ny / S, ox = nx / S;
    if (oy >= c.ho || ox >= c.wo) return 0.f;
    return relu_grad(gpost, act, (((size_t)bb * c.co + co) * c.ho + oy) * c.wo + ox);
  }
  __device__ void store(int m, int n, float v) const {
    const int hw = c.hi * c.wi, bb = n / hw, q = n % hw;
    gin[((size_t)bb * c.ci + m) * hw + q] = v;
  }
};

// Convolution weight (and bias) gradient: m = co, k = (b, oy, ox),
// n = (ci, ky, kx), and n = ci K K is the bias (B = 1).
template <int K, int S, int P>
struct ConvBwdWeightProb {
  const float *gpost;
  const bf16 *act, *in;
  float *gw, *gbias;
  ConvSpec c;
  int M, N;
  long Kd;
  __device__ float a(int m, long k) const {
    if (m >= M || k >= Kd) return 0.f;
    const int hw = c.ho * c.wo, bb = (int)(k / hw), p = (int)(k % hw);
    return relu_grad(gpost, act, ((size_t)bb * c.co + m) * hw + p);
  }
  __device__ float b(long k, int n) const {
    if (n >= N || k >= Kd) return 0.f;
    if (n == N - 1) return 1.f;
    const int ci = n / (K * K), ky = (n / K) % K, kx = n % K;
    const int hw = c.ho * c.wo, bb = (int)(k / hw), p = (int)(k % hw), oy = p / c.wo, ox = p % c.wo;
    const int iy = oy * S - P + ky, ix = ox * S - P + kx;
    if ((unsigned)iy >= (unsigned)c.hi || (unsigned)ix >= (unsigned)c.wi) return 0.f;
    return bf(in[(((size_t)bb * c.ci + ci) * c.hi + iy) * c.wi + ix]);
  }
  __device__ void store(int m, int n, float v) const {
    if (n == N - 1) gbias[m] = v;
    else gw[(size_t)m * (N - 1) + n] = v;
  }
};

// Fully connected forward: m = j, k = i, n = b; out = act(bias + acc).
template <bool RELU, typename TOut>
struct FcFwdProb {
  const bf16 *in, *wt;
  const float *bias;
  TOut *out;
  int M, N;
  long Kd;
  __device__ float a(int m, long k) const {
    return (m < M && k < Kd) ? bf(wt[(size_t)m * Kd + k]) : 0.f;
  }
  __device__ float b(long k, int n) const {
    return (n < N && k < Kd) ? bf(in[(size_t)n * Kd + k]) : 0.f;
  }
  __device__ void store(int m, int n, float v) const {
    v += bias[m];
    if (RELU) v = fmaxf(v, 0.f);
    if constexpr (sizeof(TOut) == 2) out[(size_t)n * M + m] = __float2bfloat16_rn(v);
    else out[(size_t)n * M + m] = v;
  }
};

// Fully connected input gradient: m = i, k = j, n = b.
struct FcBwdDataProb {
  const float *gpost;
  const bf16 *act, *wt;
  float *gin;
  int M, N;  // M = nin, N = batch
  long Kd;   // nout
  __device__ float a(int m, long k) const {
    return (m < M && k < Kd) ? bf(wt[(size_t)k * M + m]) : 0.f;
  }
  __device__ float b(long k, int n) const {
    return (n < N && k < Kd) ? relu_grad(gpost, act, (size_t)n * Kd + k) : 0.f;
  }
  __device__ void store(int m, int n, float v) const { gin[(size_t)n * M + m] = v; }
};

// Fully connected weight (and bias) gradient: m = j, k = b, n = i, and
// n = nin is the bias (B = 1).
struct FcBwdWeightProb {
  const float *gpost;
  const bf16 *act, *in;
  float *gw, *gbias;
  int M, N;  // M = nout, N = nin + 1
  long Kd;   // batch
  __device__ float a(int m, long k) const {
    return (m < M && k < Kd) ? relu_grad(gpost, act, (size_t)k * M + m) : 0.f;
  }
  __device__ float b(long k, int n) const {
    if (n >= N || k >= Kd) return 0.f;
    return n == N - 1 ? 1.f : bf(in[(size_t)k * (N - 1) + n]);
  }
  __device__ void store(int m, int n, float v) const {
    if (n == N - 1) gbias[m] = v;
    else gw[(size_t)m * (N - 1) + n] = v;
  }
};

// ----------------------------------------------------------------- loss --

// Mean over the batch of sum_k wk (out - target)^2; gout = d loss / d out.
// loss[b] per sample, loss[batch] the mean (fixed-order sum, one thread).
__global__ void k_loss(const float *__restrict__ out, const float *__restrict__ target,
                       const float *__restrict__ wk, int batch, float *__restrict__ gout,
                       float *__restrict__ loss) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < batch) {
    float l = 0.f;
    for (int k = 0; k < kF2Out; ++k) {
      const float e = out[b * kF2Out + k] - target[b * kF2Out + k];
      l = fmaf(wk[k] * e, e, l);
      gout[b * kF2Out + k] = 2.f * wk[k] * e / (float)batch;
    }
    loss[b] = l;
  }
}
__global__ void k_loss_sum(float *loss, int batch) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float s = 0.f;
  for (int b = 0; b < batch; ++b) s += loss[b];
  loss[batch] = s / (float)batch;
}

// ---------------------------------------------------------- init / adam --

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// He-uniform weights (bound sqrt(6 / fan_in)), zero biases.
__global__ void k_cnn_init(float *__restrict__ master, bf16 *__restrict__ mirror, uint64_t seed) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  long fan = 0;  // 0 for a bias
  if (i >= kOffW0 && i < kOffB0) fan = 2 * 5 * 5;
  else if (i >= kOffW1 && i < kOffB1) fan = 16 * 3 * 3;
  else if (i >= kOffW2 && i < kOffB2) fan = 32 * 3 * 3;
  else if (i >= kOffW3 && i < kOffB3) fan = 64 * 3 * 3;
  else if (i >= kOffF1 && i < kOffBF1) fan = kF1In;
  else if (i >= kOffF2 && i < kOffBF2) fan = kF1Out;
  const bool bias = fan == 0;
  float v = 0.f;
  if (!bias) {
    const double u = ((mix64(seed ^ mix64((uint64_t)i)) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    v = (float)((2.0 * u - 1.0) * sqrt(6.0 / (double)fan));
  }
  master[i] = v;
  mirror[i] = __float2bfloat16_rn(v);
}

__global__ void k_adam(float *__restrict__ master, bf16 *__restrict__ mirror,
                       const float *__restrict__ grad, float *__restrict__ m, float *__restrict__ v,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  const float g = grad[i];
  const float mi = fmaf(b1, m[i], (1.f - b1) * g);
  const float vi = fmaf(b2, v[i], (1.f - b2) * g * g);
  m[i] = mi;
  v[i] = vi;
  const float p = master[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  master[i] = p;
  mirror[i] = __float2bfloat16_rn(p);
}

unsigned blocks_for(long n) { return (unsigned)((n + 255) / 256 < 148L * 64 ? (n + 255) / 256 : 148L * 64); }

constexpr int kSmallBatch = 16;  // up to this batch, one warp per conv / fc output

// Partial-tile floats the split reductions of a batch need (the weight
// gradients, whose K = batch x output pixels).
size_t mma_part_floats(int b) {
  size_t m = 0;
  for (int l = 0; l < 4; ++l) {
    const ConvSpec &c = kConv[l];
    const int sl = mma_slices((long)b * c.ho * c.wo);
    const int taps = (l == 0 ? 25 : 9) * c.ci;
    if (sl > 1) m = m > (size_t)sl * c.co * (taps + 1) ? m : (size_t)sl * c.co * (taps + 1);
  }
  const int sl = mma_slices(b);
  if (sl > 1) {
    const size_t f1 = (size_t)sl * kF1Out * (kF1In + 1), f2 = (size_t)sl * kF2Out * (kF1Out + 1);
    m = m > f1 ? m : f1;
    m = m > f2 ? m : f2;
  }
  return m;
}

template <int K, int S, int P>
void conv_fwd(const bf16 *in, const bf16 *w, const float *b, const ConvSpec &c, int batch, bf16 *out,
              float *part, cudaStream_t s) {
  const long n = (long)batch * c.co * c.ho * c.wo;
  if (batch <= kSmallBatch) {
    k_conv_fwd_warp<K, S, P><<<(unsigned)((n * 32 + 255) / 256), 256, 0, s>>>(in, w, b, c, batch, out);
  } else {
    ConvFwdProb<K, S, P> p{in, w, b, out, c, c.co, batch * c.ho * c.wo, (long)c.ci * K * K};
    mma_launch<ConvFwdProb<K, S, P>, true>(p, part, 1, s);
  }
}

void forward(const bf16 *pw, const float *pm, const bf16 *in, int batch, const CnnWs &w,
             cudaStream_t s) {
  const bf16 *x = in;
  conv_fwd<5, 2, 2>(x, pw + kOffW0, pm + kOffB0, kConv[0], batch, w.a[0], w.part, s);
  conv_fwd<3, 2, 1>(w.a[0], pw + kOffW1, pm + kOffB1, kConv[1], batch, w.a[1], w.part, s);
  conv_fwd<3, 2, 1>(w.a[1], pw + kOffW2, pm + kOffB2, kConv[2], batch, w.a[2], w.part, s);
  conv_fwd<3, 2, 1>(w.a[2], pw + kOffW3, pm + kOffB3, kConv[3], batch, w.a[3], w.part, s);
  if (batch <= kSmallBatch) {
    const long w1 = (long)batch * kF1Out * 32, w2 = (long)batch * kF2Out * 32;
    k_fc_fwd<true, bf16><<<(unsigned)((w1 + 255) / 256), 256, 0, s>>>(
        w.a[3], pw + kOffF1, pm + kOffBF1, kF1In, kF1Out, batch, w.f1);
    k_fc_fwd<false, float><<<(unsigned)((w2 + 255) / 256), 256, 0, s>>>(
        w.f1, pw + kOffF2, pm + kOffBF2, kF1Out, kF2Out, batch, w.out);
  } else {
    FcFwdProb<true, bf16> f1{w.a[3], pw + kOffF1, pm + kOffBF1, w.f1, kF1Out, batch, kF1In};
    mma_launch<FcFwdProb<true, bf16>, true>(f1, w.part, 1, s);
    FcFwdProb<false, float> f2{w.f1, pw + kOffF2, pm + kOffBF2, w.out, kF2Out, batch, kF1Out};
    mma_launch<FcFwdProb<false, float>, true>(f2, w.part, 1, s);
  }
}

// A convolution's weight and bias gradients and, when gin is given, its
// input gradient, from the gradient at its output (masked by its ReLU).
template <int K, int S, int P>
void conv_bwd(const float *gpost, const bf16 *act, const bf16 *in, const bf16 *wt, const ConvSpec &c,
              int batch, float *gin, float *gw, float *gb, float *part, cudaStream_t s) {
  ConvBwdWeightProb<K, S, P> pw{gpost, act, in, gw, gb, c, c.co, c.ci * K * K + 1,
                                (long)batch * c.ho * c.wo};
  mma_launch<ConvBwdWeightProb<K, S, P>, false>(pw, part, mma_slices(pw.Kd), s);
  if (gin) {
    ConvBwdDataProb<K, S, P> pd{gpost, act, wt, gin, c, c.ci, batch * c.hi * c.wi,
                                (long)c.co * K * K};
    mma_launch<ConvBwdDataProb<K, S, P>, false>(pd, part, 1, s);
  }
}

// A fully connected layer's weight and bias gradients and its input gradient.
void fc_bwd(const float *gpost, const bf16 *act, const bf16 *in, const bf16 *wt, int nin, int nout,
            int batch, float *gin, float *gw, float *gb, float *part, cudaStream_t s) {
  FcBwdWeightProb pw{gpost, act, in, gw, gb, nout, nin + 1, batch};
  mma_launch<FcBwdWeightProb, false>(pw, part, mma_slices(batch), s);
  FcBwdDataProb pd{gpost, act, wt, gin, nin, batch, nout};
  mma_launch<FcBwdDataProb, false>(pd, part, 1, s);
}

}  // namespace

extern "C" of_status_t of_cnn_param_count(int64_t *count) {
  if (!count) return OF_ERR_INVALID_ARGUMENT;
  *count = kParams;
  return OF_OK;
}

extern "C" of_status_t of_cnn_workspace_bytes(int32_t batch, size_t *bytes) {
  if (batch < 1 || batch > 65536 || !bytes) return OF_ERR_INVALID_ARGUMENT;
  *bytes = ws_layout(nullptr, batch).total;
  return OF_OK;
}

extern "C" of_status_t of_cnn_init(float *d_master, uint16_t *d_params, uint64_t seed,
                                   of_stream_t s) {
  if (!d_master || !d_params) return OF_ERR_INVALID_ARGUMENT;
  k_cnn_init<<<(unsigned)((kParams + 255) / 256), 256, 0, (cudaStream_t)s>>>(d_master, (bf16 *)d_params, seed);
  return of_launch_status();
}

extern "C" of_status_t of_cnn_input(const uint16_t *d_prev, const uint16_t *d_cur, int32_t width,
                                    int32_t height, int32_t batch, int64_t pair_stride,
                                    float *d_cells, uint16_t *d_input, of_stream_t s) {
  if (!d_prev || !d_cur || !d_cells || !d_input || batch < 1 || batch > 65535 || width < kInW ||
      height < kInH || width % kInW || height % kInH || width / kInW != height / kInH ||
      (batch > 1 && pair_stride < (int64_t)width * height))
    return OF_ERR_INVALID_ARGUMENT;
  const long n = (long)batch * kActIn;
  k_cnn_cells<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)s>>>(
      d_prev, d_cur, width, height, (long)pair_stride, batch, d_cells);
  k_cnn_center<<<batch, 256, 0, (cudaStream_t)s>>>(d_cells, (bf16 *)d_input);
  return of_launch_status();
}

extern "C" of_status_t of_cnn_forward(const uint16_t *d_params, const float *d_master,
                                      const uint16_t *d_input, int32_t batch, void *d_ws,
                                      float *d_out, of_stream_t s) {
  if (!d_params || !d_master || !d_input || !d_ws || batch < 1 || batch > 65536)
    return OF_ERR_INVALID_ARGUMENT;
  CnnWs w = ws_layout(d_ws, batch);
  forward((const bf16 *)d_params, d_master, (const bf16 *)d_input, batch, w, (cudaStream_t)s);
  if (d_out)
    OF_CUDA_TRY(cudaMemcpyAsync(d_out, w.out, (size_t)batch * kF2Out * sizeof(float),
                                cudaMemcpyDeviceToDevice, (cudaStream_t)s));
  return of_launch_status();
}

extern "C" of_status_t of_cnn_backward(const uint16_t *d_params, const float *d_master,
                                       const uint16_t *d_input, int32_t batch,
                                       const float *d_target, const float *d_loss_weights,
                                       void *d_ws, float *d_grad, float *d_loss, of_stream_t st) {
  if (!d_params || !d_master || !d_input || !d_target || !d_loss_weights || !d_ws || !d_grad ||
      batch < 1 || batch > 65536)
    return OF_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)st;
  const bf16 *pw = (const bf16 *)d_params;
  const bf16 *in = (const bf16 *)d_input;
  CnnWs w = ws_layout(d_ws, batch);
  forward(pw, d_master, in, batch, w, s);
  k_loss<<<(batch + 255) / 256, 256, 0, s>>>(w.out, d_target, d_loss_weights, batch, w.gout, w.loss);
  k_loss_sum<<<1, 32, 0, s>>>(w.loss, batch);
  // f2 (linear): gradients of its weights and of f1's output
  fc_bwd(w.gout, nullptr, w.f1, pw + kOffF2, kF1Out, kF2Out, batch, w.gf1, d_grad + kOffF2,
         d_grad + kOffBF2, w.part, s);
  // f1 (ReLU)
  fc_bwd(w.gf1, w.f1, w.a[3], pw + kOffF1, kF1In, kF1Out, batch, w.g[3], d_grad + kOffF1,
         d_grad + kOffBF1, w.part, s);
  // convs (ReLU), last to first; the first has no input gradient
  conv_bwd<3, 2, 1>(w.g[3], w.a[3], w.a[2], pw + kOffW3, kConv[3], batch, w.g[2], d_grad + kOffW3,
                    d_grad + kOffB3, w.part, s);
  conv_bwd<3, 2, 1>(w.g[2], w.a[2], w.a[1], pw + kOffW2, kConv[2], batch, w.g[1], d_grad + kOffW2,
                    d_grad + kOffB2, w.part, s);
  conv_bwd<3, 2, 1>(w.g[1], w.a[1], w.a[0], pw + kOffW1, kConv[1], batch, w.g[0], d_grad + kOffW1,
                    d_grad + kOffB1, w.part, s);
  conv_bwd<5, 2, 2>(w.g[0], w.a[0], in, pw + kOffW0, kConv[0], batch, nullptr, d_grad + kOffW0,
                    d_grad + kOffB0, w.part, s);
  if (d_loss)
    OF_CUDA_TRY(cudaMemcpyAsync(d_loss, w.loss + batch, sizeof(float), cudaMemcpyDeviceToDevice, s));
  return of_launch_status();
}

extern "C" of_status_t of_cnn_adam(float *d_master, uint16_t *d_params, const float *d_grad,
                                   float *d_m, float *d_v, int32_t step, float lr,
                                   of_stream_t s) {
  if (!d_master || !d_params || !d_grad || !d_m || !d_v || step < 1 || !(lr > 0.f))
    return OF_ERR_INVALID_ARGUMENT;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = (float)(1.0 / (1.0 - pow((double)b1, step)));
  const float c2 = (float)(1.0 / (1.0 - pow((double)b2, step)));
  k_adam<<<(unsigned)((kParams + 255) / 256), 256, 0, (cudaStream_t)s>>>(
      d_master, (bf16 *)d_params, d_grad, d_m, d_v, lr, b1, b2, 1e-8f, c1, c2);
  return of_launch_status();
}

namespace {

__global__ void k_cnn_mirror(const float *__restrict__ master, bf16 *__restrict__ mirror) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kParams) mirror[i] = __float2bfloat16_rn(master[i]);
}

// warm = prev x [R | t] with R = exp(w) (Rodrigues; series for small angles),
// w = out[0..2] / 10 rad, t = 100 out[3..5] mm: the predicted motion applied
// in the previous camera's frame.
// D = [exp(w) | t] of a prediction (the motion in the previous camera's frame)
__device__ void motion_matrix(const float *out, double *D) {
  const double wx = out[0] * 0.1, wy = out[1] * 0.1, wz = out[2] * 0.1;
  const double th2 = wx * wx + wy * wy + wz * wz;
  double a, b;  // sin(th)/th, (1 - cos(th))/th^2
  if (th2 < 1e-8) {
    a = 1.0 - th2 / 6.0;
    b = 0.5 - th2 / 24.0;
  } else {
    const double th = sqrt(th2);
    a = sin(th) / th;
    b = (1.0 - cos(th)) / th2;
  }
  const double K[9] = {0.0, -wz, wy, wz, 0.0, -wx, -wy, wx, 0.0};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double k2 = 0.0;
      for (int m = 0; m < 3; ++m) k2 += K[3 * i + m] * K[3 * m + j];
      D[4 * i + j] = (i == j ? 1.0 : 0.0) + a * K[3 * i + j] + b * k2;
    }
  D[3] = out[3] * 100.0; D[7] = out[4] * 100.0; D[11] = out[5] * 100.0;
  D[12] = 0.0; D[13] = 0.0; D[14] = 0.0; D[15] = 1.0;
}

__device__ void warm_pose_of(const float *out, const double *prev, double *warm) {
  double D[16];
  motion_matrix(out, D);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0.0;
      for (int m = 0; m < 4; ++m) s += prev[4 * i + m] * D[4 * m + j];
      warm[4 * i + j] = s;
    }
}

__global__ void k_cnn_warm_pose(const float *__restrict__ out, const double *__restrict__ prev,
                                double *__restrict__ warm) {
  if (threadIdx.x == 0 && blockIdx.x == 0) warm_pose_of(out, prev, warm);
}

// ------------------------------------------- fused single-pair inference --
//
// The whole prediction for one (previous, current) pair in one launch: one
// cluster of kCluCtas CTAs, one per SM. CTA r owns 1/kCluCtas of the block
// means and of every layer's output channels, and holds a full copy of every
// activation in its shared memory. A layer runs in three steps: the CTA
// computes its channel slice from its local copy of the layer input, pushes
// the slice (a contiguous run of the NCHW activation) into the other CTAs'
// copies with 16-byte distributed-shared-memory stores, and one cluster
// barrier publishes every slice. The CTA's weight slice of every layer is
// staged into shared memory at launch, while the block means are summed:
// convolution weights converted to FP32 and stored tap-major
// ([ci][ky][kx][channel], one vector load feeds all of the CTA's channels),
// FC weights copied as BF16 with cp.async. Arithmetic is the batched
// kernels': BF16 weights and activations, FP32 sums (in another order), BF16
// storage.
constexpr int kCluCtas = 16;  // the non-portable cluster maximum (opted in at set-up)
constexpr int kInferThreads = 512;
constexpr int kInferWarps = kInferThreads / 32;
constexpr int kCellsPerCta = 2 * kInH * kInW / kCluCtas;
constexpr int kF1PerCta = kF1Out / kCluCtas;
constexpr int conv_per(int l) { return kConv[l].co / kCluCtas; }
constexpr int conv_taps(int l) { return kConv[l].ci * kConv[l].k * kConv[l].k; }
// bias slots in shared memory: b0..b3 (this CTA's channels), bf1 (its FC1
// outputs), bf2
constexpr int bias_at(int i) {
  return i == 0 ? 0 : i <= 4 ? bias_at(i - 1) + conv_per(i - 1) : bias_at(4) + kF1PerCta;
}
constexpr int kBiasN = bias_at(5) + kF2Out;
static_assert(kCellsPerCta * kCluCtas == 2 * kInH * kInW && kCellsPerCta % 4 == 0, "cell slices");
static_assert(kF1PerCta * kCluCtas == kF1Out && kF1PerCta <= kInferWarps, "FC1 slices");
static_assert(kBiasN <= 32 && conv_taps(0) * conv_per(0) <= kInferThreads, "staging");
// 16-byte vector staging of the conv1..3 and FC weight slices
static_assert(kOffW1 % 8 == 0 && kOffW2 % 8 == 0 && kOffW3 % 8 == 0 && kOffF1 % 8 == 0 &&
                  kOffF2 % 8 == 0, "16-byte aligned weight blocks");
static_assert((conv_taps(1) * conv_per(1)) % 8 == 0 && (conv_taps(2) * conv_per(2)) % 8 == 0 &&
                  (conv_taps(3) * conv_per(3)) % 8 == 0 && (kF1PerCta * kF1In) % 8 == 0 &&
                  (kF2Out * kF1Out) % 8 == 0, "16-byte weight slices");
// 16-byte slice pushes
static_assert((kAct[0] / kCluCtas) % 8 == 0 && (kAct[1] / kCluCtas) % 8 == 0 &&
                  (kAct[2] / kCluCtas) % 8 == 0 && (kAct[3] / kCluCtas) % 8 == 0,
              "16-byte activation slices");

constexpr int kV1 = conv_taps(1) * conv_per(1) / 8, kV2 = conv_taps(2) * conv_per(2) / 8,
              kV3 = conv_taps(3) * conv_per(3) / 8;
constexpr int kConvVecs = kV1 + kV2 + kV3;
constexpr int kConvVecRounds = (kConvVecs + kInferThreads - 1) / kInferThreads;

struct InferSmem {
  alignas(16) float cells[2 * kInH * kInW];
  alignas(16) bf16 in[kActIn];
  alignas(16) bf16 a1[kAct[0]];
  alignas(16) bf16 a2[kAct[1]];
  alignas(16) bf16 a3[kAct[2]];
  alignas(16) bf16 a4[kAct[3]];
  alignas(16) bf16 wf1[kF1PerCta * kF1In];
  alignas(16) bf16 wf2[kF2Out * kF1Out];
  alignas(16) float w0[conv_taps(0) * conv_per(0)];
  alignas(16) float w1[conv_taps(1) * conv_per(1)];
  alignas(16) float w2[conv_taps(2) * conv_per(2)];
  alignas(16) float w3[conv_taps(3) * conv_per(3)];
  float bias[32];
  alignas(16) bf16 f1[kF1Out];
  float out[8];
  float wsum[kInferWarps];
  int wcnt[kInferWarps];
  float psum[kCluCtas];
  int pcnt[kCluCtas];
};
static_assert(sizeof(InferSmem) <= 227 * 1024, "shared memory");

__device__ __forceinline__ float bf_bits(uint32_t b16) { return __uint_as_float(b16 << 16); }

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// source of staging vector v (8 BF16) of this CTA's conv1..3 weight slices
__device__ __forceinline__ const uint4 *conv_vec_src(const bf16 *pw, int rank, int v) {
  if (v < kV1) return reinterpret_cast<const uint4 *>(pw + kOffW1) + rank * kV1 + v;
  if (v < kV1 + kV2) return reinterpret_cast<const uint4 *>(pw + kOffW2) + rank * kV2 + (v - kV1);
  return reinterpret_cast<const uint4 *>(pw + kOffW3) + rank * kV3 + (v - kV1 - kV2);
}

// element e of a CTA's slice of conv layer L ([channel][tap], as in global
// memory) -> its tap-major FP32 place ([tap][channel])
template <int L>
__device__ __forceinline__ void put_tap_major(float *w, int e, float x) {
  constexpr int T = conv_taps(L), PER = conv_per(L);
  w[(e % T) * PER + e / T] = x;
}

__device__ __forceinline__ void store_conv_vec(InferSmem &S, int v, const uint4 q) {
  const uint32_t u[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float x = bf_bits(i & 1 ? u[i >> 1] >> 16 : u[i >> 1] & 0xffffu);
    if (v < kV1) put_tap_major<1>(S.w1, v * 8 + i, x);
    else if (v < kV1 + kV2) put_tap_major<2>(S.w2, (v - kV1) * 8 + i, x);
    else put_tap_major<3>(S.w3, (v - kV1 - kV2) * 8 + i, x);
  }
}

// bias slot s of this CTA (FP32 master values)
__device__ __forceinline__ float bias_of(const float *pm, int rank, int s) {
  if (s < bias_at(1)) return pm[kOffB0 + rank * conv_per(0) + s];
  if (s < bias_at(2)) return pm[kOffB1 + rank * conv_per(1) + s - bias_at(1)];
  if (s < bias_at(3)) return pm[kOffB2 + rank * conv_per(2) + s - bias_at(2)];
  if (s < bias_at(4)) return pm[kOffB3 + rank * conv_per(3) + s - bias_at(3)];
  if (s < bias_at(5)) return pm[kOffBF1 + rank * kF1PerCta + s - bias_at(4)];
  return pm[kOffBF2 + s - bias_at(5)];
}

// a row of K depth pixels as one load
template <int K> struct RowVec;
template <> struct RowVec<8> { using T = uint4; };
template <> struct RowVec<4> { using T = uint2; };
template <> struct RowVec<2> { using T = uint32_t; };
template <> struct RowVec<1> { using T = uint16_t; };

template <int K>
__device__ __forceinline__ void row_sum(const typename RowVec<K>::T &q, float &s, int &n) {
  uint32_t u[(K + 1) / 2];
  if constexpr (K == 8) { u[0] = q.x; u[1] = q.y; u[2] = q.z; u[3] = q.w; }
  else if constexpr (K == 4) { u[0] = q.x; u[1] = q.y; }
  else u[0] = q;
  s = 0.f;
  n = 0;
#pragma unroll
  for (int i = 0; i < K; ++i) {
    const uint32_t d = i & 1 ? u[i >> 1] >> 16 : u[i >> 1] & 0xffffu;
    if (d) { s += (float)d; ++n; }
  }
}

// This CTA's block means (cells rank * kCellsPerCta ..), K lanes per cell
// (one K-pixel row each, all loads in flight at once); sums of <= 64 uint16
// depths are exact in FP32, so the means equal the batched kernel's. Also
// returns this thread's share of the sum and count of the non-empty cells of
// the previous frame.
template <int K>
__device__ __forceinline__ void infer_cells(const uint16_t *prev, const uint16_t *cur, int w,
                                            InferSmem &S, int rank, float &psum, int &pcnt) {
  using V = typename RowVec<K>::T;
  constexpr int T = kCellsPerCta * K, R = (T + kInferThreads - 1) / kInferThreads;
  static_assert(kInferThreads % K == 0, "cell lanes");
  V q[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int t = r * kInferThreads + threadIdx.x;
    q[r] = V{};
    if (t < T) {
      const int c = rank * kCellsPerCta + t / K, y = t % K;
      const int f = c / (kInH * kInW), cy = (c / kInW) % kInH, cx = c % kInW;
      const uint16_t *row = (f ? cur : prev) + (size_t)(cy * K + y) * w + cx * K;
      q[r] = __ldg(reinterpret_cast<const V *>(row));
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    float s;
    int n;
    row_sum<K>(q[r], s, n);
#pragma unroll
    for (int o = 1; o < K; o <<= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      n += __shfl_xor_sync(0xffffffffu, n, o);
    }
    const int t = r * kInferThreads + threadIdx.x;
    if (t < T && t % K == 0) {
      const int c = rank * kCellsPerCta + t / K;
      const float v = n ? s / (1000.f * n) : 0.f;
      S.cells[c] = v;
      if (c < kInH * kInW && v > 0.f) { psum += v; ++pcnt; }
    }
  }
}

// copy this CTA's slice [off, off + bytes) of a shared buffer into the same
// place of every other CTA's copy (16-byte stores)
__device__ __forceinline__ void push_slice(cg::cluster_group &cluster, void *buf, int off, int bytes,
                                           int rank) {
  const int nv = bytes / 16;
  const uint4 *src = reinterpret_cast<const uint4 *>(static_cast<char *>(buf) + off);
  for (int i = threadIdx.x; i < nv * (kCluCtas - 1); i += kInferThreads) {
    const int p = i / nv, v = i - p * nv;
    const int r = p + (p >= rank);
    uint4 *dst = reinterpret_cast<uint4 *>(cluster.map_shared_rank(static_cast<char *>(buf), r) + off);
    dst[v] = src[v];
  }
}

// this CTA's channels of conv layer L from the local input copy into the
// local output copy: each thread one output pixel for all of the CTA's
// channels (register tile), the input channels split among G adjacent lanes
// (ci = g, g + G, ...) and summed by shuffles
template <int L, int G>
__device__ __forceinline__ void infer_conv(const bf16 *in, const float *w, const float *bias,
                                           bf16 *out, int rank) {
  constexpr int CI = kConv[L].ci, K = kConv[L].k, STR = kConv[L].s, P = kConv[L].p;
  constexpr int HI = kConv[L].hi, WI = kConv[L].wi, HO = kConv[L].ho, WO = kConv[L].wo;
  constexpr int PER = conv_per(L), T = HO * WO * G;
  static_assert(CI % G == 0 && 32 % G == 0 && (G == 1 || T % 32 == 0), "lane groups");
  for (int base = 0; base < T; base += kInferThreads) {
    if (base + (int)(threadIdx.x & ~31u) >= T) break;  // warp-uniform
    const int t = base + threadIdx.x;
    const bool live = t < T;
    const int p = live ? t / G : 0, g = t % G;
    const int oy = p / WO, ox = p % WO;
    float acc[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) acc[j] = 0.f;
#pragma unroll 2
    for (int ci = g; ci < CI; ci += G) {
#pragma unroll
      for (int ky = 0; ky < K; ++ky) {
        const int iy = oy * STR - P + ky;
        if ((unsigned)iy >= (unsigned)HI) continue;
#pragma unroll
        for (int kx = 0; kx < K; ++kx) {
          const int ix = ox * STR - P + kx;
          if ((unsigned)ix >= (unsigned)WI) continue;
          const float x = bf(in[(ci * HI + iy) * WI + ix]);
          const float *wp = w + ((ci * K + ky) * K + kx) * PER;
          if constexpr (PER % 4 == 0) {
#pragma unroll
            for (int j = 0; j < PER; j += 4) {
              const float4 q = *reinterpret_cast<const float4 *>(wp + j);
              acc[j] = fmaf(q.x, x, acc[j]);
              acc[j + 1] = fmaf(q.y, x, acc[j + 1]);
              acc[j + 2] = fmaf(q.z, x, acc[j + 2]);
              acc[j + 3] = fmaf(q.w, x, acc[j + 3]);
            }
          } else if constexpr (PER == 2) {
            const float2 q = *reinterpret_cast<const float2 *>(wp);
            acc[0] = fmaf(q.x, x, acc[0]);
            acc[1] = fmaf(q.y, x, acc[1]);
          } else {
#pragma unroll
            for (int j = 0; j < PER; ++j) acc[j] = fmaf(wp[j], x, acc[j]);
          }
        }
      }
    }
#pragma unroll
    for (int o = 1; o < G; o <<= 1)
#pragma unroll
      for (int j = 0; j < PER; ++j) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
    if (live) {
#pragma unroll
      for (int j = 0; j < PER; ++j)
        if (j % G == g)
          out[((rank * PER + j) * HO + oy) * WO + ox] = __float2bfloat16_rn(fmaxf(acc[j] + bias[j], 0.f));
    }
  }
}

// a conv layer's slice push: this CTA's PER channels of the NCHW output
template <int L>
__device__ __forceinline__ void push_conv(cg::cluster_group &cluster, bf16 *out, int rank) {
  constexpr int bytes = (int)(kAct[L] / kCluCtas * sizeof(bf16));
  push_slice(cluster, out, rank * bytes, bytes, rank);
}

// entry (i, j) of the warm start (the expression warm_pose_of evaluates)
__device__ double warm_pose_entry(const float *out, const double *prev, int i, int j) {
  double D[16];
  motion_matrix(out, D);
  double s = 0.0;
  for (int m = 0; m < 4; ++m) s += prev[4 * i + m] * D[4 * m + j];
  return s;
}

__global__ void __cluster_dims__(kCluCtas, 1, 1) __launch_bounds__(kInferThreads)
    k_cnn_infer(const bf16 *__restrict__ pw, const float *__restrict__ pm,
                const uint16_t *__restrict__ prev, const uint16_t *__restrict__ cur, int w,
                const double *__restrict__ prev_pose, float *__restrict__ out6,
                double *__restrict__ warm) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  InferSmem &S = *reinterpret_cast<InferSmem *>(s_raw);
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // every CTA of the cluster is running before any distributed store (the
  // matching wait comes before the first push)
  asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
  // weight staging: conv slices into registers, FC slices by cp.async
  uint4 wv[kConvVecRounds];
#pragma unroll
  for (int r = 0; r < kConvVecRounds; ++r) {
    const int v = r * kInferThreads + threadIdx.x;
    if (v < kConvVecs) wv[r] = __ldg(conv_vec_src(pw, rank, v));
  }
  float w0v = 0.f, bv = 0.f;
  if (threadIdx.x < conv_taps(0) * conv_per(0))
    w0v = bf(pw[kOffW0 + rank * conv_taps(0) * conv_per(0) + threadIdx.x]);
  if (threadIdx.x < kBiasN) bv = bias_of(pm, rank, threadIdx.x);
  {
    const uint4 *f1src = reinterpret_cast<const uint4 *>(pw + kOffF1) + rank * (kF1PerCta * kF1In / 8);
    for (int v = threadIdx.x; v < kF1PerCta * kF1In / 8; v += kInferThreads)
      cp_async16(reinterpret_cast<uint4 *>(S.wf1) + v, f1src + v);
    if (rank == 0)
      for (int v = threadIdx.x; v < kF2Out * kF1Out / 8; v += kInferThreads)
        cp_async16(reinterpret_cast<uint4 *>(S.wf2) + v, reinterpret_cast<const uint4 *>(pw + kOffF2) + v);
  }
  // block means of both frames (this CTA's cells)
  float psum = 0.f;
  int pcnt = 0;
  const int k = w / kInW;
  if (k == 8) infer_cells<8>(prev, cur, w, S, rank, psum, pcnt);
  else if (k == 4) infer_cells<4>(prev, cur, w, S, rank, psum, pcnt);
  else if (k == 2) infer_cells<2>(prev, cur, w, S, rank, psum, pcnt);
  else infer_cells<1>(prev, cur, w, S, rank, psum, pcnt);
  // staged conv weights and biases to shared memory
#pragma unroll
  for (int r = 0; r < kConvVecRounds; ++r) {
    const int v = r * kInferThreads + threadIdx.x;
    if (v < kConvVecs) store_conv_vec(S, v, wv[r]);
  }
  if (threadIdx.x < conv_taps(0) * conv_per(0)) put_tap_major<0>(S.w0, threadIdx.x, w0v);
  if (threadIdx.x < kBiasN) S.bias[threadIdx.x] = bv;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    psum += __shfl_xor_sync(0xffffffffu, psum, o);
    pcnt += __shfl_xor_sync(0xffffffffu, pcnt, o);
  }
  if (lane == 0) { S.wsum[warp] = psum; S.wcnt[warp] = pcnt; }
  __syncthreads();
  asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory");
  constexpr int kCellBytes = kCellsPerCta * (int)sizeof(float);
  push_slice(cluster, S.cells, rank * kCellBytes, kCellBytes, rank);
  if (warp == 0) {
    float s = 0.f;
    int n = 0;
    for (int i = 0; i < kInferWarps; ++i) { s += S.wsum[i]; n += S.wcnt[i]; }
    if (lane < kCluCtas) {
      cluster.map_shared_rank(S.psum, lane)[rank] = s;
      cluster.map_shared_rank(S.pcnt, lane)[rank] = n;
    }
  }
  cluster.sync();
  // network input, in every CTA: centred previous block means, difference
  {
    float s = 0.f;
    int n = 0;
#pragma unroll
    for (int r = 0; r < kCluCtas; ++r) { s += S.psum[r]; n += S.pcnt[r]; }
    const float mu = n ? s / (float)n : 0.f;
    for (int c = threadIdx.x; c < kInH * kInW; c += kInferThreads) {
      const float p = S.cells[c], q = S.cells[kInH * kInW + c];
      S.in[c] = __float2bfloat16_rn(p > 0.f ? p - mu : 0.f);
      S.in[kInH * kInW + c] = __float2bfloat16_rn(p > 0.f && q > 0.f ? q - p : 0.f);
    }
  }
  __syncthreads();
  infer_conv<0, 1>(S.in, S.w0, S.bias + bias_at(0), S.a1, rank);
  __syncthreads();
  push_conv<0>(cluster, S.a1, rank);
  cluster.sync();
  infer_conv<1, 1>(S.a1, S.w1, S.bias + bias_at(1), S.a2, rank);
  __syncthreads();
  push_conv<1>(cluster, S.a2, rank);
  cluster.sync();
  infer_conv<2, 4>(S.a2, S.w2, S.bias + bias_at(2), S.a3, rank);
  __syncthreads();
  push_conv<2>(cluster, S.a3, rank);
  cluster.sync();
  infer_conv<3, 16>(S.a3, S.w3, S.bias + bias_at(3), S.a4, rank);
  cp_async_wait_all();
  __syncthreads();
  push_conv<3>(cluster, S.a4, rank);
  cluster.sync();
  // f1: this CTA's outputs, one warp each, into CTA 0's copy
  if (warp < kF1PerCta) {
    const __nv_bfloat162 *wr = reinterpret_cast<const __nv_bfloat162 *>(S.wf1 + warp * kF1In);
    const __nv_bfloat162 *xa = reinterpret_cast<const __nv_bfloat162 *>(S.a4);
    float s0 = 0.f, s1 = 0.f;
#pragma unroll 4
    for (int i = lane; i < kF1In / 2; i += 32) {
      const float2 a = __bfloat1622float2(wr[i]), x = __bfloat1622float2(xa[i]);
      s0 = fmaf(a.x, x.x, s0);
      s1 = fmaf(a.y, x.y, s1);
    }
    float acc = s0 + s1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0)
      cluster.map_shared_rank(S.f1, 0)[rank * kF1PerCta + warp] =
          __float2bfloat16_rn(fmaxf(acc + S.bias[bias_at(4) + warp], 0.f));
  }
  cluster.sync();
  if (rank != 0) return;
  // f2 and the warm start, in CTA 0
  if (warp < kF2Out) {
    const __nv_bfloat162 *wr = reinterpret_cast<const __nv_bfloat162 *>(S.wf2 + warp * kF1Out);
    const __nv_bfloat162 *xa = reinterpret_cast<const __nv_bfloat162 *>(S.f1);
    float acc = 0.f;
    for (int i = lane; i < kF1Out / 2; i += 32) {
      const float2 a = __bfloat1622float2(wr[i]), x = __bfloat1622float2(xa[i]);
      acc = fmaf(a.x, x.x, acc);
      acc = fmaf(a.y, x.y, acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) S.out[warp] = acc + S.bias[bias_at(5) + warp];
  }
  __syncthreads();
  if (threadIdx.x < kF2Out && out6) out6[threadIdx.x] = S.out[threadIdx.x];
  if (threadIdx.x < 16 && warm)
    warm[threadIdx.x] = warm_pose_entry(S.out, prev_pose, threadIdx.x >> 2, threadIdx.x & 3);
}

}  // namespace

extern "C" of_status_t of_cnn_predict(const uint16_t *d_params, const float *d_master,
                                      const uint16_t *d_prev, const uint16_t *d_cur, int32_t width,
                                      int32_t height, const double *d_prev_pose, float *d_out,
                                      double *d_warm_pose, of_stream_t s) {
  OF_RANGE("of_cnn_predict");
  if (!d_params || !d_master || !d_prev || !d_cur || (d_warm_pose && !d_prev_pose) ||
      ((uintptr_t)d_params & 15u) || width % kInW || height % kInH || width / kInW != height / kInH ||
      (width / kInW != 1 && width / kInW != 2 && width / kInW != 4 && width / kInW != 8) ||
      ((uintptr_t)d_prev & 15u) || ((uintptr_t)d_cur & 15u))
    return OF_ERR_INVALID_ARGUMENT;
  static bool attr_set[64] = {};
  int dev = 0;
  OF_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    OF_CUDA_TRY(cudaFuncSetAttribute((const void *)k_cnn_infer,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(InferSmem)));
    OF_CUDA_TRY(cudaFuncSetAttribute((const void *)k_cnn_infer,
                                     cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    attr_set[dev] = true;
  }
  k_cnn_infer<<<kCluCtas, kInferThreads, sizeof(InferSmem), (cudaStream_t)s>>>(
      (const bf16 *)d_params, d_master, d_prev, d_cur, width, d_prev_pose, d_out, d_warm_pose);
  return of_launch_status();
}

extern "C" of_status_t of_cnn_load(const float *d_master, uint16_t *d_params, of_stream_t s) {
  if (!d_master || !d_params) return OF_ERR_INVALID_ARGUMENT;
  k_cnn_mirror<<<(unsigned)((kParams + 255) / 256), 256, 0, (cudaStream_t)s>>>(d_master, (bf16 *)d_params);
  return of_launch_status();
}

extern "C" of_status_t of_cnn_warm_pose(const float *d_out, const double *d_prev_pose,
                                        double *d_warm_pose, of_stream_t s) {
  if (!d_out || !d_prev_pose || !d_warm_pose) return OF_ERR_INVALID_ARGUMENT;
  k_cnn_warm_pose<<<1, 32, 0, (cudaStream_t)s>>>(d_out, d_prev_pose, d_warm_pose);
  return of_launch_status();
}
