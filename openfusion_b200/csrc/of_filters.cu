// of_filters.cu -- camera-side depth filters on raw uint16 depth: median
// 5x5, 8-neighbour average, Prewitt gradient, Brown undistortion
// (Source/src/CameraSupport/CameraAbstract.cu:9-229), and their chain.
//
// The equations are the reference's, with the intended border handling in
// place of its unsigned wrap-around indexing ((x + i) % width with x + i
// negative, :17, :42, :113): neighbours outside the image are left out
// (median, average) or clamped (gradient). Undistortion evaluates the y term
// of the Brown model from the undistorted x (the reference feeds it the
// already distorted x, :184-185), returns null for pixels whose source lies
// outside the image (the reference leaves them unwritten, :191-193) or whose
// bilinear taps include a null pixel (it would blend a null into the depth),
// and treats the last row like the last column (the reference compares the
// column with the height there, :207). Chained filters run back to back on
// one stream through a ping-pong buffer (the reference synchronises the
// device and copies the result back after every filter, :131-151).
#include "of_common.cuh"

using namespace of;

bool of_camera_valid(const of_camera_t *c);

namespace {

constexpr int kFx = 32, kFy = 8;

// Median of the window's non-null pixels by rank selection in registers:
// keys of null or outside pixels are 0x10000 (above every depth), so the
// valid values' ranks are their ranks among the valid ones.
__global__ void __launch_bounds__(kFx * kFy) k_median5(const uint16_t *__restrict__ in,
                                                       uint16_t *__restrict__ out, int w, int h,
                                                       uint32_t nullv) {
  const int x = blockIdx.x * kFx + threadIdx.x, y = blockIdx.y * kFy + threadIdx.y;
  if (x >= w || y >= h) return;
  uint32_t key[25];
  int n = 0, win = 0;
#pragma unroll
  for (int j = 0; j < 5; ++j)
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const int xx = x + i - 2, yy = y + j - 2;
      uint32_t k = 0x10000u;
      if ((unsigned)xx < (unsigned)w && (unsigned)yy < (unsigned)h) {
        ++win;
        const uint32_t d = __ldg(in + (size_t)yy * w + xx);
        if (d != nullv) { k = d; ++n; }
      }
      key[j * 5 + i] = k;
    }
  uint32_t r = nullv;
  if (n > win / 2) {
    // order statistics k0 = (n - 1) / 2 and k1 = n / 2 (equal for odd n)
    const int k0 = (n - 1) >> 1, k1 = n >> 1;
    uint32_t v0 = 0, v1 = 0;
#pragma unroll
    for (int a = 0; a < 25; ++a) {
      int less = 0, leq = 0;
#pragma unroll
      for (int b = 0; b < 25; ++b) {
        less += key[b] < key[a];
        leq += key[b] <= key[a];
      }
      if (key[a] < 0x10000u) {
        if (less <= k0 && k0 < leq) v0 = key[a];
        if (less <= k1 && k1 < leq) v1 = key[a];
      }
    }
    r = (n & 1) ? v1 : (v0 + v1) >> 1;
  }
  out[(size_t)y * w + x] = (uint16_t)r;
}

__global__ void __launch_bounds__(kFx * kFy) k_average(const uint16_t *__restrict__ in,
                                                       uint16_t *__restrict__ out, int w, int h,
                                                       uint32_t nullv, float thr) {
  const int x = blockIdx.x * kFx + threadIdx.x, y = blockIdx.y * kFy + threadIdx.y;
  if (x >= w || y >= h) return;
  float s = 0.f;
  int n = 0;
#pragma unroll
  for (int j = -1; j <= 1; ++j)
#pragma unroll
    for (int i = -1; i <= 1; ++i) {
      const int xx = x + i, yy = y + j;
      if ((i == 0 && j == 0) || (unsigned)xx >= (unsigned)w || (unsigned)yy >= (unsigned)h) continue;
      s += (float)__ldg(in + (size_t)yy * w + xx);
      ++n;
    }
  const float avg = s / (float)n;
  const float v = (float)__ldg(in + (size_t)y * w + x);
  out[(size_t)y * w + x] = fabsf(avg - v) > thr ? (uint16_t)nullv : (uint16_t)avg;
}

__global__ void __launch_bounds__(kFx * kFy) k_gradient(const uint16_t *__restrict__ in,
                                                        uint16_t *__restrict__ out, int w, int h,
                                                        double thr36) {
  const int x = blockIdx.x * kFx + threadIdx.x, y = blockIdx.y * kFy + threadIdx.y;
  if (x >= w || y >= h) return;
  const int xm = max(x - 1, 0), xp = min(x + 1, w - 1), ym = max(y - 1, 0), yp = min(y + 1, h - 1);
  const int cols[3] = {xm, x, xp}, rows[3] = {ym, y, yp};
  long long gx = 0, gy = 0;
#pragma unroll
  for (int j = 0; j < 3; ++j)
    gx += (long long)__ldg(in + (size_t)rows[j] * w + xp) - __ldg(in + (size_t)rows[j] * w + xm);
#pragma unroll
  for (int i = 0; i < 3; ++i)
    gy += (long long)__ldg(in + (size_t)yp * w + cols[i]) - __ldg(in + (size_t)ym * w + cols[i]);
  // (gx / 6)^2 + (gy / 6)^2 > thr^2, exactly: gx^2 + gy^2 > 36 thr^2
  const double g2 = (double)(gx * gx + gy * gy);
  out[(size_t)y * w + x] = g2 > thr36 ? (uint16_t)0 : __ldg(in + (size_t)y * w + x);
}

struct Brown {
  float fx, fy, cx, cy, k1, k2, p1, p2;
};

__global__ void __launch_bounds__(kFx * kFy) k_undistort(const uint16_t *__restrict__ in,
                                                         uint16_t *__restrict__ out, int w, int h,
                                                         Brown B, uint32_t nullv) {
  const int x = blockIdx.x * kFx + threadIdx.x, y = blockIdx.y * kFy + threadIdx.y;
  if (x >= w || y >= h) return;
  const float xn = ((float)x - B.cx) / B.fx, yn = ((float)y - B.cy) / B.fy;
  const float r2 = xn * xn + yn * yn, rad = 1.f + B.k1 * r2 + B.k2 * r2 * r2;
  const float xd = xn * rad + 2.f * B.p1 * xn * yn + B.p2 * (r2 + 2.f * xn * xn);
  const float yd = yn * rad + B.p1 * (r2 + 2.f * yn * yn) + 2.f * B.p2 * xn * yn;
  const float u = B.fx * xd + B.cx, v = B.fy * yd + B.cy;
  const float u0f = floorf(u), v0f = floorf(v);
  const size_t o = (size_t)y * w + x;
  if (!(u0f >= 0.f && u0f <= (float)(w - 1) && v0f >= 0.f && v0f <= (float)(h - 1))) {
    out[o] = (uint16_t)nullv;
    return;
  }
  const int u0 = (int)u0f, v0 = (int)v0f;
  const int u1 = u0 + 1 < w ? u0 + 1 : u0, v1 = v0 + 1 < h ? v0 + 1 : v0;
  const uint32_t a = __ldg(in + (size_t)v0 * w + u0), b = __ldg(in + (size_t)v0 * w + u1);
  const uint32_t c = __ldg(in + (size_t)v1 * w + u0), d = __ldg(in + (size_t)v1 * w + u1);
  if (a == nullv || b == nullv || c == nullv || d == nullv) {
    out[o] = (uint16_t)nullv;
    return;
  }
  const float fu = u - u0f, fv = v - v0f;
  const uint32_t f1 = u1 == u0 ? a : (uint32_t)((1.f - fu) * (float)a + fu * (float)b);
  const uint32_t f2 = v1 == v0 ? f1 : (u1 == u0 ? c : (uint32_t)((1.f - fu) * (float)c + fu * (float)d));
  out[o] = (uint16_t)(uint32_t)((1.f - fv) * (float)f1 + fv * (float)f2);
}

dim3 grid_of(int w, int h) { return dim3((w + kFx - 1) / kFx, (h + kFy - 1) / kFy); }

bool filter_params_ok(const of_depth_filter_params_t *p) {
  return p && (p->steps & ~0xF) == 0 && p->null_value >= 0 && p->null_value <= 0xFFFF &&
         p->average_passes >= 0 && p->average_passes <= 4 && p->average_threshold_mm >= 0.f &&
         p->gradient_threshold_mm >= 0.f;
}

// one filter step (kind = one OF_DEPTH_FILTER_* bit) from src to dst (distinct)
of_status_t launch_step(int kind, const of_camera_t *cam, const of_depth_filter_params_t *p,
                        const uint16_t *src, uint16_t *dst, cudaStream_t s) {
  const int w = cam->width, h = cam->height;
  const uint32_t nv = (uint32_t)p->null_value;
  switch (kind) {
    case OF_DEPTH_FILTER_UNDISTORT: {
      Brown B{cam->fx, cam->fy, cam->cx, cam->cy, p->k1, p->k2, p->p1, p->p2};
      k_undistort<<<grid_of(w, h), dim3(kFx, kFy), 0, s>>>(src, dst, w, h, B, nv);
      break;
    }
    case OF_DEPTH_FILTER_MEDIAN5:
      k_median5<<<grid_of(w, h), dim3(kFx, kFy), 0, s>>>(src, dst, w, h, nv);
      break;
    case OF_DEPTH_FILTER_GRADIENT:
      k_gradient<<<grid_of(w, h), dim3(kFx, kFy), 0, s>>>(
          src, dst, w, h, 36.0 * (double)p->gradient_threshold_mm * p->gradient_threshold_mm);
      break;
    case OF_DEPTH_FILTER_AVERAGE:
      k_average<<<grid_of(w, h), dim3(kFx, kFy), 0, s>>>(src, dst, w, h, nv, p->average_threshold_mm);
      break;
    default:
      return OF_ERR_INVALID_ARGUMENT;
  }
  return of_launch_status();
}

}  // namespace

extern "C" of_status_t of_depth_filter_step(const of_camera_t *cam, int32_t kind,
                                            const of_depth_filter_params_t *p, const uint16_t *d_in,
                                            uint16_t *d_out, of_stream_t stream) {
  if (!of_camera_valid(cam) || !filter_params_ok(p) || !d_in || !d_out || d_in == d_out ||
      (kind != OF_DEPTH_FILTER_UNDISTORT && kind != OF_DEPTH_FILTER_MEDIAN5 &&
       kind != OF_DEPTH_FILTER_GRADIENT && kind != OF_DEPTH_FILTER_AVERAGE))
    return OF_ERR_INVALID_ARGUMENT;
  return launch_step(kind, cam, p, d_in, d_out, (cudaStream_t)stream);
}

extern "C" of_status_t of_depth_filter(const of_camera_t *cam, const of_depth_filter_params_t *p,
                                       const uint16_t *d_in, uint16_t *d_out, uint16_t *d_scratch,
                                       of_stream_t stream) {
  OF_RANGE("of_depth_filter");
  if (!of_camera_valid(cam) || !filter_params_ok(p) || !d_in || !d_out) return OF_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t bytes = (size_t)cam->width * cam->height * sizeof(uint16_t);
  // the steps in the order the cameras apply them (SoftKineticCamera.cpp:424-430,
  // GIPCam.cpp:173-177): undistort, median, gradient, average (x passes)
  int steps[8], k = 0;
  if (p->steps & OF_DEPTH_FILTER_UNDISTORT) steps[k++] = OF_DEPTH_FILTER_UNDISTORT;
  if (p->steps & OF_DEPTH_FILTER_MEDIAN5) steps[k++] = OF_DEPTH_FILTER_MEDIAN5;
  if (p->steps & OF_DEPTH_FILTER_GRADIENT) steps[k++] = OF_DEPTH_FILTER_GRADIENT;
  if (p->steps & OF_DEPTH_FILTER_AVERAGE)
    for (int i = 0; i < (p->average_passes > 0 ? p->average_passes : 1); ++i)
      steps[k++] = OF_DEPTH_FILTER_AVERAGE;
  if (k == 0) {
    if (d_in != d_out) OF_CUDA_TRY(cudaMemcpyAsync(d_out, d_in, bytes, cudaMemcpyDeviceToDevice, s));
    return OF_OK;
  }
  if (k > 1 || d_in == d_out) {
    if (!d_scratch || d_scratch == d_in || d_scratch == d_out) return OF_ERR_INVALID_ARGUMENT;
  }
  // ping-pong between d_scratch and d_out so that the last step writes d_out;
  // an in-place chain starts from a copy of the input in d_scratch
  const uint16_t *src = d_in;
  if (d_in == d_out) {
    OF_CUDA_TRY(cudaMemcpyAsync(d_scratch, d_in, bytes, cudaMemcpyDeviceToDevice, s));
    src = d_scratch;
  }
  for (int i = 0; i < k; ++i) {
    const int left = k - 1 - i;  // steps after this one
    uint16_t *dst = (left % 2 == 0) ? d_out : d_scratch;
    if (dst == src) dst = (dst == d_out) ? d_scratch : d_out;
    of_status_t st = launch_step(steps[i], cam, p, src, dst, s);
    if (st != OF_OK) return st;
    src = dst;
  }
  if (src != d_out) OF_CUDA_TRY(cudaMemcpyAsync(d_out, src, bytes, cudaMemcpyDeviceToDevice, s));
  return OF_OK;
}

extern "C" void of_depth_filter_defaults(of_depth_filter_params_t *p) {
  if (!p) return;
  p->steps = 0;
  p->null_value = 0;
  p->average_passes = 1;
  p->average_threshold_mm = 15.f;   // CameraAbstract.cu:29
  p->gradient_threshold_mm = 10.f;  // CameraAbstract.cu:63 (threshold squared 100)
  p->k1 = p->k2 = p->p1 = p->p2 = 0.f;
}
