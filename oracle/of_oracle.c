/* of_oracle.c -- CPU restatement of the KinectFusion per-frame path.
 *
 * TEST INFRASTRUCTURE ONLY (see of_oracle.h): the checker of the CUDA path,
 * and, compiled with OF_REAL=float and OpenMP, the CPU baseline.
 * Reference citations are paths inside gilbs10/OpenFusion.
 */
#include "of_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef ora_real R;

#define EPS_REF 1e-6 /* _EPSILON_, Source/include/Constants.h:14 */

int32_t ora_real_bytes(void) { return (int32_t)sizeof(R); }

int32_t ora_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void ora_cam_level(const ora_cam *c, int32_t level, ora_cam *o) {
  *o = *c;
  for (int l = 0; l < level; ++l) {
    o->w = (o->w + 1) / 2;
    o->h = (o->h + 1) / 2;
    o->fx *= 0.5;
    o->fy *= 0.5;
    o->cx = (o->cx - 0.5) * 0.5;
    o->cy = (o->cy - 0.5) * 0.5;
  }
}

/* roundFloat: frac < 0.5 ? floor : ceil (Source/include/CudaUtilities.cuh:62-64) */
static inline int round_ref(R a) {
  R f = (R)floor(a);
  return (a - f) < (R)0.5 ? (int)f : (int)ceil(a);
}

static inline int near_half(double a, double margin) {
  double f = a - floor(a);
  return fabs(f - 0.5) < margin;
}


/* ---------------------------------------------------------------------------
 * Helpers shared by the main oracle and the reference-semantics functions
 * below (which are pinned against the reference's own kernels), so that the
 * pinning covers the arithmetic both use.
 * ------------------------------------------------------------------------ */

/* convertVoxelsToWorld (Source/src/VolumeIntegrator.cu:40-48): centre of
 * voxel i of n over a cube of edge `size` centred at 0. */
static inline double voxel_centre(double size, int n, int i) {
  double ratio = size / n;
  return i * ratio - 0.5 * size + 0.5 * ratio;
}

/* CameraToImage (Source/include/CudaUtilities.cuh:9-21): u = (fx X + cx Z) / Z. */
static inline void cam_project(double fx, double fy, double cx, double cy, double X, double Y,
                               double Z, double *u, double *v) {
  *u = (fx * X + cx * Z) / Z;
  *v = (fy * Y + cy * Z) / Z;
}

/* Truncation of VolumeIntegrator.cu:148-160: returns 0 when the voxel is not
 * updated (SDF < -trunc), else 1 with the truncated value in *t. */
static inline int tsdf_truncate(double sdf, double trunc, double *t) {
  if (sdf > 0.0) {
    *t = sdf < trunc ? sdf : trunc;
    return 1;
  }
  if (sdf >= -trunc) {
    *t = sdf;
    return 1;
  }
  return 0;
}

/* Running average with weight 1 (VolumeIntegrator.cu:165-166). */
static inline void tsdf_average(double prev, unsigned w, double t, unsigned max_w, double *out,
                                unsigned *w_out) {
  *out = (prev * (double)w + t) / (double)(w + 1);
  *w_out = w + 1 < max_w ? w + 1 : max_w;
}

/* Point-to-plane row of d_find_corresponding (Source/src/ICP.cu:186-201):
 * A = [n_s x d, n_s], b = n_s . (s - d). */
static inline void icp_row_terms(const double *ns, const double *d, const double *s, double *a,
                                 double *b) {
  a[0] = ns[1] * d[2] - ns[2] * d[1];
  a[1] = ns[2] * d[0] - ns[0] * d[2];
  a[2] = ns[0] * d[1] - ns[1] * d[0];
  a[3] = ns[0]; a[4] = ns[1]; a[5] = ns[2];
  *b = ns[0] * (s[0] - d[0]) + ns[1] * (s[1] - d[1]) + ns[2] * (s[2] - d[2]);
}

/* Incremental transform of Cpu_buildNewTransformMatrix (Source/src/ICP.cu:266-290):
 * R = Rz(g) Ry(b) Rx(a), t = (tx, ty, tz), from xo = (a, b, g, tx, ty, tz). */
static void euler_increment(const double *xo, double *D) {
  double al = xo[0], be = xo[1], ga = xo[2];
  double ca = cos(al), sa = sin(al), cb = cos(be), sb = sin(be), cg = cos(ga), sg = sin(ga);
  double M[16] = {cg * cb, -sg * ca + cg * sb * sa, sg * sa + cg * sb * ca, xo[3],
                  sg * cb, cg * ca + sg * sb * sa,  -cg * sa + sg * sb * ca, xo[4],
                  -sb,     cb * sa,                 cb * ca,                 xo[5],
                  0.0,     0.0,                     0.0,                     1.0};
  memcpy(D, M, sizeof(M));
}

static void matmul4(const double *A, const double *B, double *C) {
  double T[16];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double a = 0.0;
      for (int k = 0; k < 4; ++k) a += A[4 * i + k] * B[4 * k + j];
      T[4 * i + j] = a;
    }
  memcpy(C, T, sizeof(T));
}

/* ------------------------------------------------------------------------
 * Bilateral filter: Tomasi & Manduchi (ICCV 1998) on the raw depth, square
 * window of half-width `radius`, Gaussian spatial (sigma_s px) and range
 * (sigma_r mm) weights; invalid depths (outside [dmin, dmax] or 0) take no
 * part and an invalid centre stays 0 -- the pre-filter of KinectFusion
 * (Newcombe et al., ISMAR 2011, s3.2). No reference counterpart.
 * ---------------------------------------------------------------------- */
static inline int depth_ok(double d, const ora_cam *c) {
  return d > 0.0 && d >= c->dmin && d <= c->dmax;
}

void ora_bilateral(const ora_cam *c, const uint16_t *depth, double ss, double sr, int32_t rad,
                   R *out) {
  const int w = c->w, h = c->h;
  const double ks = 1.0 / (2.0 * ss * ss), kr = 1.0 / (2.0 * sr * sr);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < h; ++y) {
    for (int x = 0; x < w; ++x) {
      double cd = depth[(size_t)y * w + x];
      R res = 0;
      if (depth_ok(cd, c)) {
        R sw = 0, sd = 0;
        for (int dy = -rad; dy <= rad; ++dy) {
          int yy = y + dy;
          if (yy < 0 || yy >= h) continue;
          for (int dx = -rad; dx <= rad; ++dx) {
            int xx = x + dx;
            if (xx < 0 || xx >= w) continue;
            double q = depth[(size_t)yy * w + xx];
            if (!depth_ok(q, c)) continue;
            double del = q - cd;
            R wt = (R)exp(-((double)(dx * dx + dy * dy) * ks + del * del * kr));
            sw += wt;
            sd += wt * (R)q;
          }
        }
        res = sd / sw;
      }
      out[(size_t)y * w + x] = res;
    }
  }
}

/* Depth pyramid: block averaging of KinectFusion s3.2 with its 3 sigma_r
 * guard; a 2x2 block is averaged over its valid depths within `guard` of the
 * block's first valid depth (row-major). No reference counterpart. */
void ora_pyr_down(const R *src, int32_t sw, int32_t sh, R *dst, int32_t dw, int32_t dh,
                  double guard) {
#pragma omp parallel for schedule(static)
  for (int y = 0; y < dh; ++y)
    for (int x = 0; x < dw; ++x) {
      R ref = 0, sum = 0;
      int cnt = 0;
      for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) {
          int sx = 2 * x + i, sy = 2 * y + j;
          if (sx >= sw || sy >= sh) continue;
          R d = src[(size_t)sy * sw + sx];
          if (d > 0) {
            if (cnt == 0) ref = d;
            if (fabs((double)(d - ref)) <= guard) {
              sum += d;
              ++cnt;
            }
          }
        }
      dst[(size_t)y * dw + x] = cnt ? sum / (R)cnt : (R)0;
    }
}

/* Vertex map: d_convertDepthToWorldVertices (CameraHandler.cu:65-89) in
 * camera space: v = (-d (u-cx)/fx, -d (v-cy)/fy, -d) (CudaUtilities.cuh:24-33
 * with depth -d). Normal map: d_convertDepthToWorldNormals
 * (CameraHandler.cu:91-132): normalize((v(x+1,y)-v) x (v(x,y+1)-v)), invalid
 * on the last row/column or next to an invalid vertex; a zero cross product
 * stays invalid (cutil_math.h:1131-1137 returns the zero vector). */
void ora_vertex_normal(const ora_cam *c, const R *depth, R *pts) {
  const int w = c->w, h = c->h;
#pragma omp parallel for schedule(static)
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      size_t p = (size_t)y * w + x;
      R *o = pts + 8 * p;
      for (int i = 0; i < 8; ++i) o[i] = 0;
      R d = depth[p];
      if (!(d > 0)) continue;
      R ax = (R)((double)x - c->cx), ay = (R)((double)y - c->cy);
      R vx = -d * ax / (R)c->fx, vy = -d * ay / (R)c->fy, vz = -d;
      o[0] = vx; o[1] = vy; o[2] = vz; o[3] = 1;
      if (x + 1 >= w || y + 1 >= h) continue;
      R d10 = depth[p + 1], d01 = depth[p + w];
      if (!(d10 > 0 && d01 > 0)) continue;
      R a0 = -d10 * (ax + 1) / (R)c->fx - vx, a1 = -d10 * ay / (R)c->fy - vy, a2 = -d10 - vz;
      R b0 = -d01 * ax / (R)c->fx - vx, b1 = -d01 * (ay + 1) / (R)c->fy - vy, b2 = -d01 - vz;
      R n0 = a1 * b2 - a2 * b1, n1 = a2 * b0 - a0 * b2, n2 = a0 * b1 - a1 * b0;
      R l2 = n0 * n0 + n1 * n1 + n2 * n2;
      if (!(l2 > 0)) continue;
      R il = (R)(1.0 / sqrt((double)l2));
      o[4] = n0 * il; o[5] = n1 * il; o[6] = n2 * il; o[7] = 1;
    }
}

int64_t ora_pyramid_elems(const ora_cam *c, int32_t levels) {
  int64_t n = 0;
  for (int l = 0; l < levels; ++l) {
    ora_cam lc;
    ora_cam_level(c, l, &lc);
    n += (int64_t)lc.w * lc.h * 9;
  }
  return n;
}

void ora_preprocess(const ora_cam *c, const ora_params *p, const uint16_t *depth, R *out) {
  int rad = p->radius > 0 ? p->radius : (int)ceil(2.0 * p->sigma_s);
  R *lvl_depth[4];
  R *lvl_pts[4];
  ora_cam lc[4];
  R *q = out;
  for (int l = 0; l < p->levels; ++l) {
    ora_cam_level(c, l, &lc[l]);
    lvl_depth[l] = q;
    q += (size_t)lc[l].w * lc[l].h;
    lvl_pts[l] = q;
    q += (size_t)lc[l].w * lc[l].h * 8;
  }
  if (p->radius == -1) {
    /* no filter: the raw depth (CameraHandler.cu:65-89 converts it unfiltered) */
    for (size_t i = 0; i < (size_t)c->w * c->h; ++i)
      lvl_depth[0][i] = depth_ok(depth[i], c) ? (R)depth[i] : (R)0;
  } else {
    ora_bilateral(c, depth, p->sigma_s, p->sigma_r, rad, lvl_depth[0]);
  }
  for (int l = 1; l < p->levels; ++l)
    ora_pyr_down(lvl_depth[l - 1], lc[l - 1].w, lc[l - 1].h, lvl_depth[l], lc[l].w, lc[l].h,
                 3.0 * p->sigma_r);
  for (int l = 0; l < p->levels; ++l) ora_vertex_normal(&lc[l], lvl_depth[l], lvl_pts[l]);
}

/* ------------------------------------------------------------------ voxels */

static inline float half_to_float(uint16_t h) {
  _Float16 v;
  memcpy(&v, &h, 2);
  return (float)v;
}
static inline uint16_t float_to_half(double x) {
  _Float16 v = (_Float16)(float)x;
  uint16_t h;
  memcpy(&h, &v, 2);
  return h;
}

/* normalised tsdf; weight 0 reads +1 (d_initVoxelArray sets +TRUNCATION,
 * Source/src/General.cu:27-50) */
static inline R vox_value(uint32_t w, int storage) {
  if ((w >> 16) == 0) return 1;
  uint16_t lo = (uint16_t)(w & 0xffffu);
  if (storage == 0) return (R)(int16_t)lo / (R)32767.0;
  return (R)half_to_float(lo);
}

static inline uint32_t vox_pack(R t, uint32_t weight, int storage) {
  if (storage == 0) {
    double q = nearbyint((double)t * 32767.0);
    if (q > 32767.0) q = 32767.0;
    if (q < -32767.0) q = -32767.0;
    return (uint32_t)(uint16_t)(int16_t)q | (weight << 16);
  }
  double tc = t > 1 ? 1.0 : (t < -1 ? -1.0 : (double)t);
  return (uint32_t)float_to_half(tc) | (weight << 16);
}

/* Integration: d_integrateVolume (Source/src/VolumeIntegrator.cu:86-187) with
 * voxel x stored in slab x (the reference increments `offset` before its
 * first use, :115-123, so its voxel x lands in slab x+1):
 *   centre p_w = -size/2 + (i + 0.5) size/n (convertVoxelsToWorld, :40-48)
 *   p_c = T^-1 p_w (:126); skip unless -z in [dmin, dmax] and z < 0 (:12-16;
 *   the z < 0 test keeps voxels behind the camera out, which the reference's
 *   fabs(z) test lets through); pixel = roundFloat(project) (:127-129); skip
 *   inside the 2-pixel border (:14-15) or on invalid depth (:136-140);
 *   SDF = |v_depth - c| - |p_w - c| (:146) with |v_depth - c| = lambda D;
 *   skip SDF < -trunc, tsdf' = min(SDF, trunc) (:148-160);
 *   tsdf = (tsdf w + tsdf') / (w + 1), w = min(max_w, w + 1) (:165-166). */
int64_t ora_integrate(const ora_vol *v, uint32_t *words, const ora_cam *c, const uint16_t *depth,
                      const double *P, uint8_t *ambig) {
  const int n = v->n;
  const double T = v->trunc;
  const double cpos[3] = {P[3], P[7], P[11]};
  int64_t updated = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : updated)
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      for (int k = 0; k < n; ++k) {
        size_t idx = ((size_t)i * n + j) * n + k;
        int amb = 0;
        R pw[3] = {(R)voxel_centre(v->size, n, i), (R)voxel_centre(v->size, n, j),
                   (R)voxel_centre(v->size, n, k)};
        R dlt[3] = {pw[0] - (R)cpos[0], pw[1] - (R)cpos[1], pw[2] - (R)cpos[2]};
        R X = (R)P[0] * dlt[0] + (R)P[4] * dlt[1] + (R)P[8] * dlt[2];
        R Y = (R)P[1] * dlt[0] + (R)P[5] * dlt[1] + (R)P[9] * dlt[2];
        R Z = (R)P[2] * dlt[0] + (R)P[6] * dlt[1] + (R)P[10] * dlt[2];
        if (ambig) {
          if (fabs(-(double)Z - c->dmin) < 2e-3 || fabs(-(double)Z - c->dmax) < 2e-3) amb = 1;
        }
        int upd = 0;
        R sn = 0;
        if (Z < 0 && -Z >= (R)c->dmin && -Z <= (R)c->dmax) {
          double ud, vd;
          cam_project(c->fx, c->fy, c->cx, c->cy, X, Y, Z, &ud, &vd);
          R uf = (R)ud, vf = (R)vd;
          if (ambig && (near_half(uf, 1e-3) || near_half(vf, 1e-3))) amb = 1;
          int pu = round_ref(uf), pv = round_ref(vf);
          if (!(pu < 2 || pu >= c->w - 2 || pv < 2 || pv >= c->h - 2)) {
            double D = depth[(size_t)pv * c->w + pu];
            if (depth_ok(D, c)) {
              R a = (R)(((double)pu - c->cx) / c->fx), b = (R)(((double)pv - c->cy) / c->fy);
              R lam = (R)sqrt((double)(1 + a * a + b * b));
              R rr = (R)sqrt((double)(dlt[0] * dlt[0] + dlt[1] * dlt[1] + dlt[2] * dlt[2]));
              R sdf = lam * (R)D - rr;
              if (ambig && fabs((double)sdf + T) < 1e-3) amb = 1;
              double tt;
              if (tsdf_truncate((double)sdf, T, &tt)) {
                upd = 1;
                sn = (R)(tt / T);
              }
            }
          }
        }
        if (ambig) ambig[idx] = (uint8_t)amb;
        if (!upd) continue;
        ++updated;
        uint32_t word = words[idx];
        uint32_t wt = word >> 16;
        R told = wt ? vox_value(word, v->storage) : 0;
        double tnd;
        unsigned wn;
        tsdf_average((double)told, wt, (double)sn, (unsigned)v->max_w, &tnd, &wn);
        R tn = (R)tnd;
        words[idx] = vox_pack(tn, wn, v->storage);
      }
    }
  }
  return updated;
}

/* ---------------------------------------------------------------- raycast */

typedef struct {
  const uint32_t *w;
  int n, storage;
  double org, inv_vs;
} vol_view;

static R trilinear(const vol_view *V, R px, R py, R pz) {
  R g[3] = {(R)(((double)px - V->org) * V->inv_vs - 0.5), (R)(((double)py - V->org) * V->inv_vs - 0.5),
            (R)(((double)pz - V->org) * V->inv_vs - 0.5)};
  int i0[3];
  R f[3];
  for (int a = 0; a < 3; ++a) {
    int q = (int)floor(g[a]);
    if (q < 0) q = 0;
    if (q > V->n - 2) q = V->n - 2;
    i0[a] = q;
    f[a] = g[a] - (R)q;
  }
  R cval[8];
  for (int q = 0; q < 8; ++q) {
    int a = (q >> 2) & 1, b = (q >> 1) & 1, d = q & 1;
    size_t idx = ((size_t)(i0[0] + a) * V->n + (i0[1] + b)) * V->n + (i0[2] + d);
    cval[q] = vox_value(V->w[idx], V->storage);
  }
  R c00 = cval[0] + f[2] * (cval[1] - cval[0]);
  R c01 = cval[2] + f[2] * (cval[3] - cval[2]);
  R c10 = cval[4] + f[2] * (cval[5] - cval[4]);
  R c11 = cval[6] + f[2] * (cval[7] - cval[6]);
  R c0 = c00 + f[1] * (c01 - c00);
  R c1 = c10 + f[1] * (c11 - c10);
  return c0 + f[0] * (c1 - c0);
}

/* The surface of a + -> - bracket [t, tn] (f(t) = fp > 0 >= f(tn) = fn) along
 * o + t dir: the bracket is narrowed to one min_step by stepping from its
 * positive end, then `iters` Illinois regula-falsi steps (Dowell & Jarratt
 * 1971) refine it; returns the final secant point. */
static R refine_root(const vol_view *V, const R *o, const R *dir, R t, R fp, R tn, R fn,
                     R min_step, int iters) {
  R ta = t, fa = fp, tb = tn, fb = fn;
  while (tb - ta > min_step * (R)1.0001) {
    R tm = ta + min_step;
    R fm = trilinear(V, o[0] + tm * dir[0], o[1] + tm * dir[1], o[2] + tm * dir[2]);
    if (fm > 0) { ta = tm; fa = fm; } else { tb = tm; fb = fm; break; }
  }
  int side = 0;
  for (int r = 0; r < iters; ++r) {
    R tm = ta + (tb - ta) * (fa / (fa - fb));
    R fm = trilinear(V, o[0] + tm * dir[0], o[1] + tm * dir[1], o[2] + tm * dir[2]);
    if (fm > 0) {
      ta = tm; fa = fm;
      if (side == 1) fb *= (R)0.5;
      side = 1;
    } else {
      tb = tm; fb = fm;
      if (side == -1) fa *= (R)0.5;
      side = -1;
    }
  }
  return ta + (tb - ta) * (fa / (fa - fb));
}

/* Whether a refined surface depends on where rounding puts the march: the
 * bracket moved by +-shift (FP32 rounding of a metre-long march reaches a
 * few micrometres and the tsdf-scaled steps can carry it on) must keep its
 * sign change and give a surface within `tol` of `ts`. A bracket that holds a
 * non-monotonic stretch of the field (a ray clipping a thin negative dip, with
 * its negative end near the dip's far zero crossing) leaves the few Illinois
 * steps far from converged, and their result then moves with the bracket. */
static int refine_is_sensitive(const vol_view *V, const R *o, const R *dir, R t, R tn, R ts,
                               R min_step, int iters, R shift, R tol) {
  for (int k = -1; k <= 1; k += 2) {
    const R a = t + (R)k * shift, b = tn + (R)k * shift;
    const R fa = trilinear(V, o[0] + a * dir[0], o[1] + a * dir[1], o[2] + a * dir[2]);
    const R fb = trilinear(V, o[0] + b * dir[0], o[1] + b * dir[1], o[2] + b * dir[2]);
    if (!(fa > 0) || !(fb <= 0)) return 1;
    const R tp = refine_root(V, o, dir, a, fa, b, fb, min_step, iters);
    if (fabs((double)(tp - ts)) > (double)tol) return 1;
  }
  return 0;
}

/* What a ray's march needs besides the ray. */
typedef struct {
  const vol_view *V;
  const uint8_t *flags, *sflags;  /* brick / super-brick flags (NULL: no skipping) */
  int n, nbk, ns;
  double vs;
  R min_step, far_k;
  int refine_iters;
} march_ctx;

/* The march of one ray over [t0, t1] (see ora_raycast); returns whether it
 * hit, with the refined surface in *ts. `pert` is added to every position
 * update (each step's end and each skip's landing): 0 for the method itself,
 * a small shift to test whether the result depends on rounding. With `amb`,
 * decisions within rounding of a boundary set *amb. */
static int march_ray(const march_ctx *M, const R *o, const R *dir, R t0, R t1, R pert, R *ts,
                     int *amb) {
  const vol_view *V = M->V;
  const int n = M->n, nbk = M->nbk, ns = M->ns;
  const double vs = M->vs;
  const R min_step = M->min_step, far_k = M->far_k;
  if (!(t0 < t1)) return 0;
  R t = t0;
  R fp = 1;
  int sampled = 0;
  for (int it = 0; it < (1 << 16); ++it) {
    R px = o[0] + t * dir[0], py = o[1] + t * dir[1], pz = o[2] + t * dir[2];
    if (M->flags) {
      /* empty-space skip: a brick whose flag is clear holds, with its 26
       * neighbours, only +1 voxels; every sample whose cell base is in it
       * reads +1, so the march jumps past its region (past the region of the
       * whole super-brick when its flag is clear) */
      int bi[3];
      R pp[3] = {px, py, pz};
      for (int a = 0; a < 3; ++a) {
        int q = (int)floor(((double)pp[a] - V->org) * V->inv_vs - 0.5);
        if (q < 0) q = 0;
        if (q > n - 2) q = n - 2;
        bi[a] = q >> 3;
      }
      const int super_clear = !M->sflags[((size_t)(bi[0] / 4) * ns + bi[1] / 4) * ns + bi[2] / 4];
      if (super_clear || !M->flags[((size_t)bi[0] * nbk + bi[1]) * nbk + bi[2]]) {
        const int span = super_clear ? 32 : 8;
        R te = (R)1e30;
        for (int a = 0; a < 3; ++a) {
          if (fabs((double)dir[a]) <= 1e-12) continue;
          const int ci = super_clear ? bi[a] / 4 : bi[a];
          double edge = dir[a] > 0 ? V->org + vs * ((double)span * (ci + 1) + 0.5)
                                   : V->org + vs * ((double)span * ci + 0.5);
          R ta = (R)((edge - (double)o[a]) / (double)dir[a]);
          if (ta < te) te = ta;
        }
        t = (te > t ? te : t) + (R)(0.01 * vs) + pert;
        fp = 1;
        sampled = 1;
        if (amb && fabs((double)(t - t1)) < 0.05) *amb = 1;
        if (t > t1) return 0;
        continue;
      }
    }
    if (!sampled) {
      fp = trilinear(V, px, py, pz);
      sampled = 1;
    }
    R step = fp > 0 ? (far_k * fp > min_step ? far_k * fp : min_step) : min_step;
    R tn = t + step + pert;
    if (amb && fabs((double)(tn - t1)) < 0.05) *amb = 1;
    if (tn > t1) return 0;
    R fn = trilinear(V, o[0] + tn * dir[0], o[1] + tn * dir[1], o[2] + tn * dir[2]);
    if (amb && fabs((double)fn) < 2e-4) *amb = 1;
    if (fp > 0 && fn <= 0) {
      *ts = refine_root(V, o, dir, t, fp, tn, fn, min_step, M->refine_iters);
      if (amb && refine_is_sensitive(V, o, dir, t, tn, *ts, min_step, M->refine_iters, (R)0.01,
                                     (R)0.02))
        *amb = 1;
      return 1;
    }
    if (fp < 0 && fn > 0) return 0;
    t = tn;
    fp = fn;
  }
  return 0;
}

/* Raycast: d_raycast (Source/src/Raycaster.cu:97-230) -- ray from the camera
 * position through the pixel's point at z = -1 (:117-125), slab clip
 * (:35-55) to the box of voxel centres, march to the first surface. The
 * sampling follows KinectFusion s3.4 (the trilinear zero-crossing the
 * reference left disabled, :170-187, :246-351): trilinear tsdf samples, step
 * max(min_step, far_frac * f * trunc) for f > 0 else min_step, surface at a
 * + -> - crossing whose bracket is narrowed to one min_step by stepping from
 * its positive end, then refined by `refine_iters` Illinois regula-falsi
 * steps, - -> + ends
 * the ray; normal = normalised central differences of trilinear samples one
 * voxel apart; the march is limited to [dmin, dmax] depth. With `flags` (one
 * byte per 8^3 brick, clear = the brick and its 26 neighbours hold only +1
 * voxels) the march jumps over clear bricks: empty-space skipping, as the
 * CUDA kernel does. Every skipped sample would have read +1, but the samples
 * after a jump fall elsewhere than a plain march's, so a negative stretch
 * thinner than one step can be found by one march and stepped over by the
 * other. `ambig` flags a ray whose skip landing or step ends
 * within 0.05 mm of the range end, whose march sample lies within 2e-4 of
 * zero, whose normal's samples touch the box within 0.05 mm, whose refined
 * surface is sensitive to rounding (refine_is_sensitive), or whose march finds
 * another hit or miss, or a surface more than 0.05 mm away, when every
 * position update moves by +-2e-3 mm: where the field is steep (noise),
 * tsdf-scaled steps amplify position differences, and a negative stretch
 * thinner than a step is caught by one march and stepped over by another. */
void ora_raycast(const ora_vol *v, const uint32_t *words, const uint8_t *flags, const ora_cam *c,
                 const ora_params *p, const double *P, R *pts, uint8_t *ambig) {
  const int n = v->n;
  const double vs = v->size / n;
  vol_view V = {words, n, v->storage, -0.5 * v->size, 1.0 / vs};
  const R lo = (R)(-0.5 * v->size + 0.5 * vs + 1e-3), hi = (R)(0.5 * v->size - 0.5 * vs - 1e-3);
  const R min_step = (R)(p->min_step_vox * vs), far_k = (R)(p->far_step_frac * v->trunc);
  const R o[3] = {(R)P[3], (R)P[7], (R)P[11]};
  const R rvs = (R)vs;
  /* super-brick flags (4^3 bricks): the OR of their bricks' flags, as the
   * volume keeps them beside the brick flags */
  const int nbk = n / 8, ns = (nbk + 3) / 4;
  uint8_t *sflags = NULL;
  if (flags) {
    sflags = (uint8_t *)calloc((size_t)ns * ns * ns, 1);
    for (int i = 0; i < nbk; ++i)
      for (int j = 0; j < nbk; ++j)
        for (int k = 0; k < nbk; ++k)
          if (flags[((size_t)i * nbk + j) * nbk + k]) sflags[((size_t)(i / 4) * ns + j / 4) * ns + k / 4] = 1;
  }
  const march_ctx M = {&V, flags, sflags, n, nbk, ns, vs, min_step, far_k, p->refine_iters};
#pragma omp parallel for schedule(dynamic, 4)
  for (int y = 0; y < c->h; ++y) {
    for (int x = 0; x < c->w; ++x) {
      size_t pix = (size_t)y * c->w + x;
      int amb = 0;
      R dc[3] = {(R)(-((double)x - c->cx) / c->fx), (R)(-((double)y - c->cy) / c->fy), -1};
      R lam = (R)sqrt((double)(dc[0] * dc[0] + dc[1] * dc[1] + 1));
      R dir[3];
      for (int a = 0; a < 3; ++a)
        dir[a] = ((R)P[4 * a] * dc[0] + (R)P[4 * a + 1] * dc[1] + (R)P[4 * a + 2] * dc[2]) / lam;
      R tnear = (R)-1e30, tfar = (R)1e30;
      for (int a = 0; a < 3; ++a) {
        if (fabs((double)dir[a]) < 1e-12) {
          if (o[a] < lo || o[a] > hi) { tnear = (R)1e30; tfar = (R)-1e30; }
        } else {
          R t0 = (lo - o[a]) / dir[a], t1 = (hi - o[a]) / dir[a];
          R mn = t0 < t1 ? t0 : t1, mx = t0 < t1 ? t1 : t0;
          if (mn > tnear) tnear = mn;
          if (mx < tfar) tfar = mx;
        }
      }
      R t0 = tnear > (R)c->dmin * lam ? tnear : (R)c->dmin * lam;
      R t1 = tfar < (R)c->dmax * lam ? tfar : (R)c->dmax * lam;
      R ts = 0;
      const int hit = march_ray(&M, o, dir, t0, t1, 0, &ts, ambig ? &amb : NULL);
      if (ambig && !amb && t0 < t1) {
        /* the found surface must not depend on where rounding puts the
         * march: every position update moved by +-2e-3 mm (FP32 rounding
         * of one update of a metre-long march is ~1e-4 mm) must find the
         * same hit or miss, and a surface within 0.05 mm */
        for (int k = -1; k <= 1 && !amb; k += 2) {
          R tp = 0;
          const int hp = march_ray(&M, o, dir, t0, t1, (R)(2e-3 * k), &tp, NULL);
          if (hp != hit || (hit && fabs((double)(tp - ts)) > 0.05)) amb = 1;
        }
      }
      R *out = pts + 8 * pix;
      for (int i = 0; i < 8; ++i) out[i] = 0;
      if (hit) {
        R px = o[0] + ts * dir[0], py = o[1] + ts * dir[1], pz = o[2] + ts * dir[2];
        out[0] = px; out[1] = py; out[2] = pz; out[3] = 1;
        if (px - rvs >= lo && px + rvs <= hi && py - rvs >= lo && py + rvs <= hi &&
            pz - rvs >= lo && pz + rvs <= hi) {
          R gx = trilinear(&V, px + rvs, py, pz) - trilinear(&V, px - rvs, py, pz);
          R gy = trilinear(&V, px, py + rvs, pz) - trilinear(&V, px, py - rvs, pz);
          R gz = trilinear(&V, px, py, pz + rvs) - trilinear(&V, px, py, pz - rvs);
          R l2 = gx * gx + gy * gy + gz * gz;
          if (l2 > 0) {
            R il = (R)(1.0 / sqrt((double)l2));
            out[4] = gx * il; out[5] = gy * il; out[6] = gz * il; out[7] = 1;
          }
          if (ambig && (fabs((double)px - rvs - lo) < 0.05 || fabs((double)hi - px - rvs) < 0.05 ||
                        fabs((double)py - rvs - lo) < 0.05 || fabs((double)hi - py - rvs) < 0.05 ||
                        fabs((double)pz - rvs - lo) < 0.05 || fabs((double)hi - pz - rvs) < 0.05))
            amb = 1;
        }
      }
      if (ambig) ambig[pix] = (uint8_t)amb;
    }
  }
  free(sflags);
}

/* The march of chosen pixels with every position update moved by each of
 * `npert` perturbations (mm): out[(i * npert + k) * 4] = hit vertex (x, y, z,
 * 1) or zeros, for pixel (xy[2 i], xy[2 i + 1]). Explains a disagreement with
 * another arithmetic: the surface a march finds when its positions move by a
 * bounded amount. */
void ora_raycast_pixels(const ora_vol *v, const uint32_t *words, const uint8_t *flags,
                        const ora_cam *c, const ora_params *p, const double *P, int32_t npix,
                        const int32_t *xy, int32_t npert, const double *perts, R *out) {
  const int n = v->n;
  const double vs = v->size / n;
  vol_view V = {words, n, v->storage, -0.5 * v->size, 1.0 / vs};
  const R lo = (R)(-0.5 * v->size + 0.5 * vs + 1e-3), hi = (R)(0.5 * v->size - 0.5 * vs - 1e-3);
  const R o[3] = {(R)P[3], (R)P[7], (R)P[11]};
  const int nbk = n / 8, ns = (nbk + 3) / 4;
  uint8_t *sflags = NULL;
  if (flags) {
    sflags = (uint8_t *)calloc((size_t)ns * ns * ns, 1);
    for (int i = 0; i < nbk; ++i)
      for (int j = 0; j < nbk; ++j)
        for (int k = 0; k < nbk; ++k)
          if (flags[((size_t)i * nbk + j) * nbk + k]) sflags[((size_t)(i / 4) * ns + j / 4) * ns + k / 4] = 1;
  }
  const march_ctx M = {&V, flags, sflags, n, nbk, ns, vs, (R)(p->min_step_vox * vs),
                       (R)(p->far_step_frac * v->trunc), p->refine_iters};
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < npix * npert; ++i) {
    const int q = i / npert, k = i % npert;
    const int x = xy[2 * q], y = xy[2 * q + 1];
    R dc[3] = {(R)(-((double)x - c->cx) / c->fx), (R)(-((double)y - c->cy) / c->fy), -1};
    R lam = (R)sqrt((double)(dc[0] * dc[0] + dc[1] * dc[1] + 1));
    R dir[3];
    for (int a = 0; a < 3; ++a)
      dir[a] = ((R)P[4 * a] * dc[0] + (R)P[4 * a + 1] * dc[1] + (R)P[4 * a + 2] * dc[2]) / lam;
    R tnear = (R)-1e30, tfar = (R)1e30;
    for (int a = 0; a < 3; ++a) {
      if (fabs((double)dir[a]) < 1e-12) {
        if (o[a] < lo || o[a] > hi) { tnear = (R)1e30; tfar = (R)-1e30; }
      } else {
        R t0 = (lo - o[a]) / dir[a], t1 = (hi - o[a]) / dir[a];
        R mn = t0 < t1 ? t0 : t1, mx = t0 < t1 ? t1 : t0;
        if (mn > tnear) tnear = mn;
        if (mx < tfar) tfar = mx;
      }
    }
    R t0 = tnear > (R)c->dmin * lam ? tnear : (R)c->dmin * lam;
    R t1 = tfar < (R)c->dmax * lam ? tfar : (R)c->dmax * lam;
    R ts = 0;
    const int hit = march_ray(&M, o, dir, t0, t1, (R)perts[k], &ts, NULL);
    R *dst = out + 4 * (size_t)i;
    for (int a = 0; a < 3; ++a) dst[a] = hit ? o[a] + ts * dir[a] : 0;
    dst[3] = hit ? 1 : 0;
  }
  free(sflags);
}

/* The trilinear tsdf (tsdf / trunc) at world points xyz[3 i .. 3 i + 2]: the
 * field the raycast marches (cell corners clamped as in `trilinear`). */
void ora_tsdf_at(const ora_vol *v, const uint32_t *words, int64_t npts, const double *xyz,
                 R *out) {
  const int n = v->n;
  const double vs = v->size / n;
  vol_view V = {words, n, v->storage, -0.5 * v->size, 1.0 / vs};
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < npts; ++i)
    out[i] = trilinear(&V, (R)xyz[3 * i], (R)xyz[3 * i + 1], (R)xyz[3 * i + 2]);
}

void ora_model_down(const R *src, int32_t sw, R *dst, int32_t dw, int32_t dh) {
  for (int y = 0; y < dh; ++y)
    for (int x = 0; x < dw; ++x)
      memcpy(dst + 8 * ((size_t)y * dw + x), src + 8 * ((size_t)(2 * y) * sw + 2 * x),
             8 * sizeof(R));
}

/* -------------------------------------------------------------------- ICP */

/* Correspondence + point-to-plane row of one model pixel:
 * d_find_corresponding (Source/src/ICP.cu:116-251). Returns 1 and fills
 * a[6], b when the pixel is an inlier. With `alt` != 0 the other rounding of
 * the projected coordinate is used on the axes whose bit is set. */
static int icp_row(const ora_cam *lc, const R *frame, const R *s, const R *ns, const double *P,
                   const double *W, double dist, double nthr, int alt, R *a, R *b, int *gate_amb,
                   int *round_amb, int *projected) {
  R sc[3];
  for (int r = 0; r < 3; ++r)
    sc[r] = (R)W[4 * r] * s[0] + (R)W[4 * r + 1] * s[1] + (R)W[4 * r + 2] * s[2] + (R)W[4 * r + 3];
  if (sc[2] >= (R)-EPS_REF) return 0;
  R uf = (R)lc->fx * sc[0] / sc[2] + (R)lc->cx;
  R vf = (R)lc->fy * sc[1] / sc[2] + (R)lc->cy;
  if (round_amb) *round_amb = (near_half(uf, 1e-3) ? 1 : 0) | (near_half(vf, 1e-3) ? 2 : 0);
  int pu = round_ref(uf), pv = round_ref(vf);
  if (alt & 1) pu = (uf - floor(uf) < 0.5) ? pu + 1 : pu - 1;
  if (alt & 2) pv = (vf - floor(vf) < 0.5) ? pv + 1 : pv - 1;
  if (pu < 0 || pu >= lc->w || pv < 0 || pv >= lc->h) return 0;
  if (projected) *projected = 1;  /* the model point lands in the frame: examined */
  const R *f = frame + 8 * ((size_t)pv * lc->w + pu);
  if (f[3] == 0 || f[7] == 0) return 0;
  R d[3], nd[3];
  for (int r = 0; r < 3; ++r) {
    d[r] = (R)P[4 * r] * f[0] + (R)P[4 * r + 1] * f[1] + (R)P[4 * r + 2] * f[2] + (R)P[4 * r + 3];
    nd[r] = (R)P[4 * r] * f[4] + (R)P[4 * r + 1] * f[5] + (R)P[4 * r + 2] * f[6];
  }
  R e[3] = {d[0] - s[0], d[1] - s[1], d[2] - s[2]};
  R len = (R)sqrt((double)(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]));
  R dn = nd[0] * ns[0] + nd[1] * ns[1] + nd[2] * ns[2];
  if (gate_amb)
    *gate_amb = fabs((double)len - dist) < 1e-3 || fabs((double)dn - nthr) < 1e-5 ||
                fabs((double)dn - (1.0 + EPS_REF)) < 1e-6;
  {
    double nsd[3] = {ns[0], ns[1], ns[2]}, dd[3] = {d[0], d[1], d[2]}, sd[3] = {s[0], s[1], s[2]};
    double ad[6], bd;
    icp_row_terms(nsd, dd, sd, ad, &bd);
    for (int q = 0; q < 6; ++q) a[q] = (R)ad[q];
    *b = (R)bd;
  }
  if (!(len < (R)dist)) return gate_amb && *gate_amb ? 2 : 0;
  if (!(dn > (R)nthr && dn < (R)(1.0 + EPS_REF))) return gate_amb && *gate_amb ? 2 : 0;
  return 1;
}

static void row_products(const R *a, R b, double *v) {
  int k = 0;
  for (int i = 0; i < 6; ++i)
    for (int j = i; j < 6; ++j) v[k++] = (double)a[i] * (double)a[j];
  for (int i = 0; i < 6; ++i) v[21 + i] = (double)a[i] * (double)b;
  v[27] = (double)b * (double)b;
  v[28] = 1.0;
}

static void rigid_inverse(const double *P, double *W) {
  for (int i = 0; i < 3; ++i) {
    double acc = 0.0;
    for (int j = 0; j < 3; ++j) {
      W[4 * i + j] = P[4 * j + i];
      acc -= P[4 * j + i] * P[4 * j + 3];
    }
    W[4 * i + 3] = acc;
  }
  W[12] = W[13] = W[14] = 0.0;
  W[15] = 1.0;
}

/* One correspondence pass (see ora_icp_system); `examined` (may be NULL)
 * gets the number of model points that project into the frame. */
static void icp_system_impl(const ora_cam *lc, const R *frame, int32_t mw, int32_t mh,
                            const R *model, const double *P, double dist, double nthr,
                            double *out, double *amb, double *examined) {
  double W[16];
  rigid_inverse(P, W);
  const int npx = mw * mh;
  double acc[29] = {0}, am[29] = {0}, ex = 0.0;
  /* rows accumulate per image row, rows combine in order: deterministic */
  double *rows = (double *)calloc((size_t)mh * 59, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int y = 0; y < mh; ++y) {
    double *ra = rows + (size_t)y * 59, *rm = ra + 29;
    for (int x = 0; x < mw; ++x) {
      size_t p = (size_t)y * mw + x;
      const R *s = model + 8 * p;
      if (s[3] == 0 || s[7] == 0) continue;
      R a[6], b;
      int gamb = 0, ramb = 0, proj = 0;
      double v[29];
      int ok = icp_row(lc, frame, s, s + 4, P, W, dist, nthr, 0, a, &b, &gamb, &ramb, &proj);
      ra[58] += proj;
      if (ok) row_products(a, b, v);
      if (ok == 1)
        for (int q = 0; q < 29; ++q) ra[q] += v[q];
      if (amb && (gamb || ramb)) {
        if (ok)
          for (int q = 0; q < 29; ++q) rm[q] += fabs(v[q]);
        for (int alt = 1; alt < 4; ++alt) {
          if ((alt & ramb) != alt) continue;
          R a2[6], b2;
          if (icp_row(lc, frame, s, s + 4, P, W, dist, nthr, alt, a2, &b2, NULL, NULL, NULL) ==
              1) {
            row_products(a2, b2, v);
            for (int q = 0; q < 29; ++q) rm[q] += fabs(v[q]);
          }
        }
      }
    }
  }
  (void)npx;
  for (int y = 0; y < mh; ++y) {
    for (int q = 0; q < 29; ++q) {
      acc[q] += rows[(size_t)y * 59 + q];
      am[q] += rows[(size_t)y * 59 + 29 + q];
    }
    ex += rows[(size_t)y * 59 + 58];
  }
  free(rows);
  for (int q = 0; q < 29; ++q) out[q] = acc[q];
  if (amb)
    for (int q = 0; q < 29; ++q) amb[q] = am[q];
  if (examined) *examined = ex;
}

void ora_icp_system(const ora_cam *lc, const R *frame, int32_t mw, int32_t mh, const R *model,
                    const double *P, double dist, double nthr, double *out, double *amb) {
  icp_system_impl(lc, frame, mw, mh, model, P, dist, nthr, out, amb, NULL);
}

/* FP64 Cholesky solve of the 6x6 normal equations and the SE(3) update:
 * ICP::Iterate_ICP (Source/src/ICP.cpp:142-168: symmetrise, singularity test,
 * llt().solve, rotation part negated) and Cpu_buildNewTransformMatrix
 * (Source/src/ICP.cu:266-305: dT = [Rz(g) Ry(b) Rx(a) | t], T <- dT T). The
 * singularity test is a pivot below 1e-12 x the largest diagonal entry or
 * fewer than 6 inliers, in place of |det| < 1e-6 in FP32. */
static int32_t icp_solve_step(const double *sys, double *P, double *minpiv, double *x_out);

int32_t ora_icp_step(const double *sys, double *P, double *minpiv) {
  return icp_solve_step(sys, P, minpiv, NULL);
}

/* as ora_icp_step; x_out (may be NULL) gets the solution x of H x = g before
 * the rotation part is negated */
static int32_t icp_solve_step(const double *sys, double *P, double *minpiv, double *x_out) {
  double H[6][6], L[6][6] = {{0}}, g[6], y[6], x[6];
  int q = 0;
  for (int i = 0; i < 6; ++i)
    for (int j = i; j < 6; ++j) { H[i][j] = H[j][i] = sys[q++]; }
  for (int i = 0; i < 6; ++i) g[i] = sys[21 + i];
  double dmax = 0.0;
  for (int i = 0; i < 6; ++i) dmax = fmax(dmax, H[i][i]);
  double mp = 1e300;
  int ok = sys[28] >= 6.0 && dmax > 0.0 && isfinite(dmax);
  for (int j = 0; j < 6 && ok; ++j) {
    double s = H[j][j];
    for (int k = 0; k < j; ++k) s -= L[j][k] * L[j][k];
    mp = fmin(mp, s / dmax);
    if (!(s > 1e-12 * dmax) || !isfinite(s)) { ok = 0; break; }
    L[j][j] = sqrt(s);
    for (int i = j + 1; i < 6; ++i) {
      double t = H[i][j];
      for (int k = 0; k < j; ++k) t -= L[i][k] * L[j][k];
      L[i][j] = t / L[j][j];
    }
  }
  if (minpiv) *minpiv = ok ? mp : fmin(mp, 0.0);
  if (!ok) return 1;
  for (int i = 0; i < 6; ++i) {
    double t = g[i];
    for (int k = 0; k < i; ++k) t -= L[i][k] * y[k];
    y[i] = t / L[i][i];
  }
  for (int i = 5; i >= 0; --i) {
    double t = y[i];
    for (int k = i + 1; k < 6; ++k) t -= L[k][i] * x[k];
    x[i] = t / L[i][i];
  }
  if (x_out)
    for (int i = 0; i < 6; ++i) x_out[i] = x[i];
  double xo[6] = {-x[0], -x[1], -x[2], x[3], x[4], x[5]};
  double D[16];
  euler_increment(xo, D);
  matmul4(D, P, P);
  return 0;
}

static void pyramid_levels(const ora_cam *c, int levels, const R *base, const R **dep,
                           const R **pts, ora_cam *lc) {
  const R *q = base;
  for (int l = 0; l < levels; ++l) {
    ora_cam_level(c, l, &lc[l]);
    dep[l] = q;
    q += (size_t)lc[l].w * lc[l].h;
    pts[l] = q;
    q += (size_t)lc[l].w * lc[l].h * 8;
  }
}

/* Multi-level ICP, coarse to fine, fixed iteration counts (the reference runs
 * ICP_ITERATIONS = 15 at one level, Source/include/Constants.h:50). A
 * singular system restores the starting pose and stops (ICP.cpp:152-158). */
int32_t ora_icp_track(const ora_cam *c, const ora_params *p, const R *frame, const R *model,
                      double *P, int32_t *iterations) {
  const R *fd[4], *fp[4], *md[4], *mp[4];
  ora_cam lc[4];
  pyramid_levels(c, p->levels, frame, fd, fp, lc);
  pyramid_levels(c, p->levels, model, md, mp, lc);
  double P0[16];
  memcpy(P0, P, sizeof(P0));
  int its = 0;
  for (int l = p->levels - 1; l >= 0; --l) {
    for (int it = 0; it < p->iters[l]; ++it) {
      double sys[29];
      ora_icp_system(&lc[l], fp[l], lc[l].w, lc[l].h, mp[l], P, p->dist_thresh, p->normal_thresh,
                     sys, NULL);
      ++its;
      if (ora_icp_step(sys, P, NULL) != 0) {
        memcpy(P, P0, sizeof(P0));
        if (iterations) *iterations = its;
        return 1;
      }
    }
  }
  if (iterations) *iterations = its;
  return 0;
}

/* Multi-level ICP with the device path's options, in FP64: the early exit, a
 * warm-started first pass and the judge that keeps or replaces its result.
 * Neither has a reference counterpart (the reference starts from the
 * previous pose and runs every iteration, Source/src/ICP.cpp:84-182); this
 * restates the project's own method so the device kernel can be checked
 * against it step by step:
 *   - a level ends early once the increment's rotation components are all
 *     below stop_rot (rad) and its translation components all below
 *     stop_trans (mm), when stop_rot > 0;
 *   - with a warm start W, pass 0 starts from W and runs only the
 *     warm_levels finest levels; its result is kept when the system did not
 *     become singular, the last iteration's RMS point-to-plane residual is at
 *     most judge_rms, its inliers are at least judge_frac of the model points
 *     that landed in the frame, and the result lies within judge_rot (rad,
 *     angle of W^T P) and judge_trans (mm) of W; otherwise pass 1 runs plain
 *     ICP from the starting pose over every level;
 *   - a singular system restores the starting pose and ends the pass
 *     (ICP.cpp:152-158).
 * res->decisions_near counts exit and judge decisions whose quantity lies
 * within 1 % of its threshold (where FP32 and FP64 may decide differently). */
static int near_threshold(double q, double thr) { return fabs(q - thr) <= 0.01 * fabs(thr); }

int32_t ora_icp_track_ex(const ora_cam *c, const ora_params *p, const ora_icp_opts *o,
                         const R *frame, const R *model, double *P, const double *warm,
                         ora_icp_result *res) {
  const R *fd[4], *fp[4], *md[4], *mp[4];
  ora_cam lc[4];
  pyramid_levels(c, p->levels, frame, fd, fp, lc);
  pyramid_levels(c, p->levels, model, md, mp, lc);
  double P0[16];
  memcpy(P0, P, sizeof(P0));
  const int warm_levels = (o->warm_levels > 0 && o->warm_levels < p->levels) ? o->warm_levels
                                                                             : p->levels;
  int its = 0, stop = 0, warm_status = 0, near = 0, inl = 0, examined = 0;
  double res_sq = 0.0;
  if (warm) memcpy(P, warm, 16 * sizeof(double));
  for (int pass = 0; pass < 2; ++pass) {
    const int top = (pass == 0 && warm) ? warm_levels - 1 : p->levels - 1;
    for (int l = top; l >= 0 && !stop; --l) {
      for (int it = 0; it < p->iters[l]; ++it) {
        double sys[29], ex = 0.0, x[6], mp_ = 0.0;
        icp_system_impl(&lc[l], fp[l], lc[l].w, lc[l].h, mp[l], P, p->dist_thresh,
                        p->normal_thresh, sys, NULL, &ex);
        ++its;
        inl = (int)sys[28];
        examined = (int)ex;
        res_sq = sys[27];
        if (icp_solve_step(sys, P, &mp_, x) != 0) {
          memcpy(P, P0, sizeof(P0));
          stop = 1;
          break;
        }
        if (o->stop_rot > 0.0) {
          const double ir = fmax(fabs(x[0]), fmax(fabs(x[1]), fabs(x[2])));
          const double it_ = fmax(fabs(x[3]), fmax(fabs(x[4]), fabs(x[5])));
          near += near_threshold(ir, o->stop_rot) || near_threshold(it_, o->stop_trans);
          if (ir < o->stop_rot && it_ < o->stop_trans) break;
        }
      }
    }
    if (pass == 1 || !warm) break;
    int keep = !stop;
    if (keep) {
      double tr = 0.0, dt2 = 0.0;
      for (int i = 0; i < 3; ++i) {
        for (int k = 0; k < 3; ++k) tr += warm[4 * k + i] * P[4 * k + i];
        const double d = P[4 * i + 3] - warm[4 * i + 3];
        dt2 += d * d;
      }
      const double rot = acos(fmin(1.0, fmax(-1.0, 0.5 * (tr - 1.0))));
      const double rms = sqrt(res_sq / (double)(inl > 1 ? inl : 1));
      const double frac = (double)inl / (double)(examined > 1 ? examined : 1);
      near += near_threshold(rms, o->judge_rms) || near_threshold(frac, o->judge_frac) ||
              near_threshold(rot, o->judge_rot) || near_threshold(sqrt(dt2), o->judge_trans);
      keep = rms <= o->judge_rms && frac >= o->judge_frac && rot <= o->judge_rot &&
             sqrt(dt2) <= o->judge_trans;
    }
    warm_status = keep ? 1 : 2;
    if (keep) break;
    stop = 0;
    memcpy(P, P0, sizeof(P0));
  }
  if (res) {
    res->status = stop ? 1 : 0;
    res->iterations = its;
    res->warm = warm ? warm_status : 0;
    res->inliers = inl;
    res->examined = examined;
    res->decisions_near = near;
    res->residual_sq = res_sq;
  }
  return stop ? 1 : 0;
}

/* ------------------------------------------------------------ CPU tracker */

struct ora_tracker {
  ora_cam cam;
  ora_vol vol;
  ora_params par;
  double pose[16];
  uint32_t *words;
  R *frame, *model;
  int64_t frames;
};

ora_tracker *ora_tracker_create(const ora_cam *c, const ora_vol *v, const ora_params *p,
                                const double *pose0) {
  ora_tracker *t = (ora_tracker *)calloc(1, sizeof(ora_tracker));
  if (!t) return NULL;
  t->cam = *c;
  t->vol = *v;
  t->par = *p;
  memcpy(t->pose, pose0, sizeof(t->pose));
  size_t nv = (size_t)v->n * v->n * v->n;
  int64_t pe = ora_pyramid_elems(c, p->levels);
  t->words = (uint32_t *)calloc(nv, sizeof(uint32_t));
  t->frame = (R *)calloc((size_t)pe, sizeof(R));
  t->model = (R *)calloc((size_t)pe, sizeof(R));
  if (!t->words || !t->frame || !t->model) {
    ora_tracker_destroy(t);
    return NULL;
  }
  return t;
}

void ora_tracker_destroy(ora_tracker *t) {
  if (!t) return;
  free(t->words);
  free(t->frame);
  free(t->model);
  free(t);
}

/* RunApp::display (Source/src/MainApp.cpp:786-964) in the order
 * pre-process -> ICP -> integrate -> raycast. */
int32_t ora_tracker_process(ora_tracker *t, const uint16_t *depth) {
  int32_t status = 0;
  if (t->frames > 0) {
    ora_preprocess(&t->cam, &t->par, depth, t->frame);
    status = ora_icp_track(&t->cam, &t->par, t->frame, t->model, t->pose, NULL);
  }
  ora_integrate(&t->vol, t->words, &t->cam, depth, t->pose, NULL);
  const R *md[4], *mp[4];
  ora_cam lc[4];
  pyramid_levels(&t->cam, t->par.levels, t->model, md, mp, lc);
  ora_raycast(&t->vol, t->words, NULL, &t->cam, &t->par, t->pose, (R *)mp[0], NULL);
  for (int l = 1; l < t->par.levels; ++l)
    ora_model_down(mp[l - 1], lc[l - 1].w, (R *)mp[l], lc[l].w, lc[l].h);
  t->frames += 1;
  return status;
}

void ora_tracker_pose(const ora_tracker *t, double *pose) { memcpy(pose, t->pose, sizeof(t->pose)); }

uint32_t *ora_tracker_volume(ora_tracker *t) { return t->words; }

/* ===========================================================================
 * Reference semantics. These restate the reference's kernels as they are
 * (float storage, uint8 weights, nearest-voxel raycast, single-pass
 * correspondences), in FP64, for comparison with the reference's own kernels
 * run on the same inputs (tests/golden/ref_*.npz). They share the helpers
 * above with the main oracle.
 * ======================================================================== */

#define REF_BAD 3.4028234663852886e38 /* BAD_VERTEX = FLT_MAX (Constants.h:36) */

static inline int ref_bad(const double *v) {
  return v[0] == REF_BAD || v[1] == REF_BAD || v[2] == REF_BAD;
}

/* d_convertDepthToWorldVertices + d_convertDepthToWorldNormals
 * (Source/src/CameraSupport/CameraHandler.cu:65-132) with the inverse
 * intrinsics the caller passes (m_invIntrinsic). */
void ora_ref_convert(const ora_refcam *c, const uint16_t *depth, const double *T, double *vertex,
                     double *normal) {
  const int w = c->w, h = c->h;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      size_t p = (size_t)y * w + x;
      double D = depth[p];
      double *v = vertex + 3 * p;
      if (fabs(D) < c->dmin || fabs(D) > c->dmax) {
        v[0] = v[1] = v[2] = REF_BAD;
        continue;
      }
      double d = -D;  /* ImageToCamera with depth -newDepth (CameraHandler.cu:87) */
      double cam[3] = {d * (c->ifx * x + c->icx), d * (c->ify * y + c->icy), d};
      for (int r = 0; r < 3; ++r)
        v[r] = T[4 * r] * cam[0] + T[4 * r + 1] * cam[1] + T[4 * r + 2] * cam[2] + T[4 * r + 3];
    }
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      size_t p = (size_t)y * w + x;
      double *n = normal + 3 * p;
      n[0] = n[1] = n[2] = 0.0;
      const double *v = vertex + 3 * p;
      if (ref_bad(v) || x + 1 >= w || y + 1 >= h) continue;
      const double *a = vertex + 3 * (p + 1), *b = vertex + 3 * (p + w);
      if (ref_bad(a) || ref_bad(b)) continue;
      double e1[3] = {a[0] - v[0], a[1] - v[1], a[2] - v[2]};
      double e2[3] = {b[0] - v[0], b[1] - v[1], b[2] - v[2]};
      double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                      e1[0] * e2[1] - e1[1] * e2[0]};
      double l2 = cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2];
      if (l2 == 0.0) continue;  /* normalize keeps the zero vector (cutil_math.h:1131-1137) */
      double il = 1.0 / sqrt(l2);
      n[0] = cr[0] * il; n[1] = cr[1] * il; n[2] = cr[2] * il;
    }
}

/* One voxel of d_integrateVolume (VolumeIntegrator.cu:119-166) against a world
 * vertex map: returns 1 and the truncated SDF when the voxel is updated. */
static int ref_voxel_sdf(const ora_refvol *v, const ora_refcam *c, const double *vertex,
                         const double *invT, const double *cpos, int x, int y, int z, double *t,
                         int *amb) {
  double p[3] = {voxel_centre(v->world, v->n, x), voxel_centre(v->world, v->n, y),
                 voxel_centre(v->world, v->n, z)};
  double cam[3];
  for (int r = 0; r < 3; ++r)
    cam[r] = invT[4 * r] * p[0] + invT[4 * r + 1] * p[1] + invT[4 * r + 2] * p[2] + invT[4 * r + 3];
  if (fabs(cam[2]) < 1e-6) return 0; /* CameraToImage returns BAD_VERTEX; the frustum test rejects it */
  double u, w_;
  cam_project(c->fx, c->fy, c->cx, c->cy, cam[0], cam[1], cam[2], &u, &w_);
  if (amb && (near_half(u, 1e-3) || near_half(w_, 1e-3) || fabs(fabs(cam[2]) - c->dmin) < 1e-2 ||
              fabs(fabs(cam[2]) - c->dmax) < 1e-2))
    *amb = 1;
  int pu = round_ref((R)u), pv = round_ref((R)w_);
  /* notInFrustum (VolumeIntegrator.cu:12-16) */
  if (pu < 2 || pu >= c->w - 2 || pv < 2 || pv >= c->h - 2 || fabs(cam[2]) > c->dmax ||
      fabs(cam[2]) < c->dmin)
    return 0;
  const double *dv = vertex + 3 * ((size_t)pv * c->w + pu);
  if (ref_bad(dv)) return 0;
  double a2 = 0.0, b2 = 0.0;
  for (int r = 0; r < 3; ++r) {
    a2 += (dv[r] - cpos[r]) * (dv[r] - cpos[r]);
    b2 += (p[r] - cpos[r]) * (p[r] - cpos[r]);
  }
  double sdf = sqrt(a2) - sqrt(b2); /* VolumeIntegrator.cu:146 */
  if (amb && fabs(sdf + v->trunc) < 1e-3) *amb = 1;
  return tsdf_truncate(sdf, v->trunc, t);
}

/* d_integrateVolume at the given storage indices (x*n*n + y*n + z, x up to
 * n): with v->b1 the kernel's storage shift applies (voxel x lives in slab
 * x + 1, VolumeIntegrator.cu:115-123). prev_* are the stored values before the
 * call; out_* after. */
void ora_ref_integrate_voxels(const ora_refvol *v, const ora_refcam *c, const double *vertex,
                              const double *invT, const double *cpos, const int64_t *storage,
                              int64_t count, const double *prev_tsdf, const int32_t *prev_w,
                              double *out_tsdf, int32_t *out_w, uint8_t *ambig) {
  const int64_t n = v->n;
#pragma omp parallel for schedule(static)
  for (int64_t q = 0; q < count; ++q) {
    int64_t s = storage[q];
    int sx = (int)(s / (n * n)), sy = (int)((s / n) % n), sz = (int)(s % n);
    int x = v->b1 ? sx - 1 : sx;
    out_tsdf[q] = prev_tsdf[q];
    out_w[q] = prev_w[q];
    int amb = 0;
    double t;
    if (x >= 0 && x < n && ref_voxel_sdf(v, c, vertex, invT, cpos, x, sy, sz, &t, &amb)) {
      double o;
      unsigned wo;
      tsdf_average(prev_tsdf[q], (unsigned)prev_w[q], t, (unsigned)v->max_w, &o, &wo);
      out_tsdf[q] = (double)(float)o; /* the reference stores float */
      out_w[q] = (int32_t)wo;
    }
    if (ambig) ambig[q] = (uint8_t)amb;
  }
}

/* The whole float volume (storage of (n + 1) n^2 elements), for the raycast. */
void ora_ref_integrate_full(const ora_refvol *v, const ora_refcam *c, const double *vertex,
                            const double *invT, const double *cpos, float *tsdf, uint8_t *w) {
  const int n = v->n;
#pragma omp parallel for schedule(dynamic, 1)
  for (int x = 0; x < n; ++x)
    for (int y = 0; y < n; ++y)
      for (int z = 0; z < n; ++z) {
        double t;
        if (!ref_voxel_sdf(v, c, vertex, invT, cpos, x, y, z, &t, NULL)) continue;
        size_t s = ((size_t)(v->b1 ? x + 1 : x) * n + y) * n + z;
        double o;
        unsigned wo;
        tsdf_average(tsdf[s], w[s], t, (unsigned)v->max_w, &o, &wo);
        tsdf[s] = (float)o;
        w[s] = (uint8_t)wo;
      }
}

/* d_raycast (Source/src/Raycaster.cu:97-230) with its fixed constants
 * (maxSteps 850, tstep 1.5 mm, zPlane -1, stop at tfar - 2): nearest-voxel
 * samples, the first tsdf <= 0 is the surface, central-difference normal at
 * that voxel (zero on the volume faces). `tsdf` is the storage array read by
 * slab floor(position). */
void ora_ref_raycast(const ora_refvol *v, const float *tsdf, const ora_refcam *c, const double *T,
                     const double *cpos, double *vertex, double *normal, uint8_t *ambig) {
  const int n = v->n;
  const double half = 0.5 * v->world;
#pragma omp parallel for schedule(dynamic, 4)
  for (int y = 0; y < c->h; ++y)
    for (int x = 0; x < c->w; ++x) {
      size_t p = (size_t)y * c->w + x;
      double *vo = vertex + 3 * p, *no = normal + 3 * p;
      int amb = 0;
      /* ray: pixel at z = -1 in camera space, to world, minus the origin (:117-125) */
      double cc[3] = {-(c->ifx * x + c->icx), -(c->ify * y + c->icy), -1.0};
      double d[3];
      for (int r = 0; r < 3; ++r)
        d[r] = T[4 * r] * cc[0] + T[4 * r + 1] * cc[1] + T[4 * r + 2] * cc[2] + T[4 * r + 3] - cpos[r];
      double dl = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      for (int r = 0; r < 3; ++r) d[r] /= dl;
      /* intersectBox (:35-55) */
      double tmin[3], tmax[3];
      for (int r = 0; r < 3; ++r) {
        double inv = 1.0 / d[r];
        double tb = inv * (-half - cpos[r]), tt = inv * (half - cpos[r]);
        tmin[r] = tt < tb ? tt : tb;
        tmax[r] = tt < tb ? tb : tt;
      }
      double tnear = fmax(fmax(tmin[0], tmin[1]), fmax(tmin[0], tmin[2]));
      double tfar = fmin(fmin(tmax[0], tmax[1]), fmin(tmax[0], tmax[2]));
      no[0] = no[1] = no[2] = 0.0;
      if (!(tfar > tnear)) {
        vo[0] = vo[1] = vo[2] = REF_BAD;
        if (ambig) ambig[p] = (uint8_t)(fabs(tfar - tnear) < 1e-3);
        continue;
      }
      if (tnear < 0.0) tnear = 0.0;
      double t = tnear;
      double start[3] = {cpos[0] + d[0] * tnear, cpos[1] + d[1] * tnear, cpos[2] + d[2] * tnear};
      double surf[3] = {REF_BAD, REF_BAD, REF_BAD};
      int flag = 0, cur[3] = {-1, -1, -1};
      for (int s = 1; s < 850; ++s) {
        double pos[3];
        for (int r = 0; r < 3; ++r) pos[r] = start[r] + s * (d[r] * 1.5);
        double gg[3];
        for (int r = 0; r < 3; ++r) {
          gg[r] = (pos[r] / v->world + 0.5) * n;
          cur[r] = (int)floor(gg[r]);
        }
        if (cur[0] < 0 || cur[0] >= n || cur[1] < 0 || cur[1] >= n || cur[2] < 0 || cur[2] >= n)
          break;
        float val = tsdf[((size_t)cur[0] * n + cur[1]) * n + cur[2]];
        if (ambig) {
          if (fabs(val) < 1e-4) amb = 1;
          /* a sample within FP32 rounding of a voxel face matters only when
           * the voxel across the face would flip the surface decision */
          for (int r = 0; r < 3; ++r) {
            double fr = gg[r] - floor(gg[r]);
            int alt = fr < 1e-4 ? -1 : (fr > 1.0 - 1e-4 ? 1 : 0);
            if (!alt) continue;
            int q[3] = {cur[0], cur[1], cur[2]};
            q[r] += alt;
            if (q[r] < 0 || q[r] >= n) { amb = 1; continue; }
            float va = tsdf[((size_t)q[0] * n + q[1]) * n + q[2]];
            if ((va <= 0.f) != (val <= 0.f)) amb = 1;
          }
        }
        if (val <= 0.f) {
          for (int r = 0; r < 3; ++r) surf[r] = pos[r];
          flag = 1;
          break;
        }
        t += 1.5;
        if (ambig && fabs(t - (tfar - 2.0)) < 1e-3) amb = 1;
        if (t > tfar - 2.0) break;
      }
      for (int r = 0; r < 3; ++r) vo[r] = surf[r];
      if (flag) {
        int X = cur[0], Y = cur[1], Z = cur[2];
        if (!(X <= 0 || X + 1 >= n || Y <= 0 || Y + 1 >= n || Z <= 0 || Z + 1 >= n)) {
#define RV(a, b, e) ((double)tsdf[((size_t)(a) * n + (b)) * n + (e)])
          double g[3] = {RV(X + 1, Y, Z) - RV(X - 1, Y, Z), RV(X, Y + 1, Z) - RV(X, Y - 1, Z),
                         RV(X, Y, Z + 1) - RV(X, Y, Z - 1)};
#undef RV
          double l2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
          if (l2 > 0.0) {
            double il = 1.0 / sqrt(l2);
            no[0] = g[0] * il; no[1] = g[1] * il; no[2] = g[2] * il;
          }
        }
      }
      if (ambig) ambig[p] = (uint8_t)amb;
    }
}

/* d_find_corresponding (Source/src/ICP.cu:116-251) over the whole image:
 * new depth tested at the model pixel's own offset (:139-149), projection of
 * the model point with the current world-to-camera transform, rejection
 * outside the image or at z >= -eps (:90-95), distance and normal gates
 * (:179-181), row terms (:186-201). out36: AtA as the reference stores it
 * (upper entries i <= j at [6 i + j]); out6: Atb; amb36/amb6 (may be NULL):
 * sums of |terms| of pixels within rounding of a decision. */
void ora_ref_icp_system(const ora_refcam *c, const uint16_t *new_depth, const double *new_vertex,
                        const double *new_normal, const double *model_vertex,
                        const double *model_normal, const double *invT, double *out36,
                        double *out6, double *amb36, double *amb6) {
  for (int q = 0; q < 36; ++q) { out36[q] = 0.0; if (amb36) amb36[q] = 0.0; }
  for (int q = 0; q < 6; ++q) { out6[q] = 0.0; if (amb6) amb6[q] = 0.0; }
  for (int y = 0; y < c->h; ++y)
    for (int x = 0; x < c->w; ++x) {
      size_t p = (size_t)y * c->w + x;
      double nd0 = new_depth[p];
      const double *s = model_vertex + 3 * p, *ns = model_normal + 3 * p;
      if (fabs(nd0) < c->dmin || fabs(nd0) > c->dmax || ref_bad(s)) continue;
      double sc[3];
      for (int r = 0; r < 3; ++r)
        sc[r] = invT[4 * r] * s[0] + invT[4 * r + 1] * s[1] + invT[4 * r + 2] * s[2] + invT[4 * r + 3];
      if (fabs(sc[2]) < 1e-6) continue;
      double u, w_;
      cam_project(c->fx, c->fy, c->cx, c->cy, sc[0], sc[1], sc[2], &u, &w_);
      int amb = near_half(u, 1e-3) || near_half(w_, 1e-3);
      int col = round_ref((R)u), row = round_ref((R)w_);
      if (col < 0 || col >= c->w || row < 0 || row >= c->h || sc[2] >= -1e-6) continue;
      size_t o = (size_t)row * c->w + col;
      const double *dv = new_vertex + 3 * o, *dn = new_normal + 3 * o;
      double e[3] = {dv[0] - s[0], dv[1] - s[1], dv[2] - s[2]};
      double len = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
      double dot = dn[0] * ns[0] + dn[1] * ns[1] + dn[2] * ns[2];
      amb |= fabs(len - 25.0) < 1e-3 || fabs(dot - 0.65) < 1e-5;
      if (!(len < 25.0 && dot > 0.65 && dot < 1.0 + 1e-6)) {
        if (amb && amb36 && len < 1e30) {
          double a[6], b;
          icp_row_terms(ns, dv, s, a, &b);
          for (int i = 0; i < 6; ++i) {
            for (int j = i; j < 6; ++j) amb36[6 * i + j] += fabs(a[i] * a[j]);
            amb6[i] += fabs(a[i] * b);
          }
        }
        continue;
      }
      double a[6], b;
      icp_row_terms(ns, dv, s, a, &b);
      for (int i = 0; i < 6; ++i) {
        for (int j = i; j < 6; ++j) out36[6 * i + j] += a[i] * a[j];
        out6[i] += a[i] * b;
      }
      if (amb && amb36) {
        for (int i = 0; i < 6; ++i) {
          for (int j = i; j < 6; ++j) amb36[6 * i + j] += fabs(a[i] * a[j]);
          amb6[i] += fabs(a[i] * b);
        }
      }
    }
}

/* Cpu_buildNewTransformMatrix (Source/src/ICP.cu:266-321) in FP64:
 * T <- dT T, full <- full dT. */
void ora_ref_compose(const double *xopt, double *T, double *full) {
  double D[16];
  euler_increment(xopt, D);
  matmul4(D, T, T);
  matmul4(full, D, full);
}

/* ------------------------------------------------------------------ mesh */

/* Marching tetrahedra (Doi & Koide 1991; Bloomenthal's tetrahedral
 * polygonizer) over Kuhn's split of each cell into the 6 tetrahedra around
 * its main diagonal: corners 0, e_a, e_a + e_b, 7 (corner index dx | dy << 1 |
 * dz << 2) for each axis order. A corner with tsdf < 0 is inside; one corner
 * against three gives the triangle on its three edges, two against two the
 * quadrilateral e(p,r) e(q,r) e(q,s) e(p,s) as (epr, eqr, eqs) + (epr, eqs,
 * eps). Vertex = linear zero crossing, interpolated from the edge's voxel of
 * lower brick-major address. Triangles face from the inside corners to the
 * outside ones. Only cells whose 8 voxels are observed produce triangles. */
static const int ora_tets[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7},
                                   {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};

static uint64_t brick_address(int n, int i, int j, int k) {
  const uint64_t nb = (uint64_t)(n / 8);
  const uint64_t b = ((uint64_t)(i >> 3) * nb + (uint64_t)(j >> 3)) * nb + (uint64_t)(k >> 3);
  return (b << 9) | (uint64_t)(((i & 7) << 6) | ((j & 7) << 3) | (k & 7));
}

typedef struct {
  R v, p[3];
  uint64_t a;
} mesh_corner;

static void mesh_edge(const mesh_corner *x, const mesh_corner *y, R *out) {
  const mesh_corner *lo = x->a < y->a ? x : y, *hi = x->a < y->a ? y : x;
  const R t = lo->v / (lo->v - hi->v);
  for (int d = 0; d < 3; ++d) out[d] = lo->p[d] + t * (hi->p[d] - lo->p[d]);
}

static void mesh_put(R *out, const R *a, const R *b, const R *c, const R *dir) {
  R u[3], w[3];
  for (int d = 0; d < 3; ++d) { u[d] = b[d] - a[d]; w[d] = c[d] - a[d]; }
  const R nx = u[1] * w[2] - u[2] * w[1], ny = u[2] * w[0] - u[0] * w[2], nz = u[0] * w[1] - u[1] * w[0];
  const int flip = nx * dir[0] + ny * dir[1] + nz * dir[2] < 0;
  for (int d = 0; d < 3; ++d) {
    out[d] = a[d];
    out[3 + d] = flip ? c[d] : b[d];
    out[6 + d] = flip ? b[d] : c[d];
  }
}

int64_t ora_mesh(const ora_vol *v, const uint32_t *words, R *tris, uint64_t *ids, int64_t max_tris) {
  const int n = v->n;
  int64_t cnt = 0;
  for (int i = 0; i < n - 1; ++i)
    for (int j = 0; j < n - 1; ++j)
      for (int k = 0; k < n - 1; ++k) {
        mesh_corner C[8];
        int live = 1;
        for (int c = 0; c < 8 && live; ++c) {
          const int ci = i + (c & 1), cj = j + ((c >> 1) & 1), ck = k + (c >> 2);
          const uint32_t w = words[((size_t)ci * n + cj) * n + ck];
          if ((w >> 16) == 0) live = 0;
          C[c].v = vox_value(w, v->storage);
          C[c].p[0] = (R)voxel_centre(v->size, n, ci);
          C[c].p[1] = (R)voxel_centre(v->size, n, cj);
          C[c].p[2] = (R)voxel_centre(v->size, n, ck);
          C[c].a = brick_address(n, ci, cj, ck);
        }
        if (!live) continue;
        const uint64_t cell = ((uint64_t)i * n + j) * n + k;
        for (int q = 0; q < 6; ++q) {
          int in[4], outc[4], ni = 0, no = 0;
          for (int r = 0; r < 4; ++r) {
            const int t = ora_tets[q][r];
            if (C[t].v < 0) in[ni++] = t;
            else outc[no++] = t;
          }
          if (ni == 0 || ni == 4) continue;
          R dir[3] = {0, 0, 0};
          for (int r = 0; r < no; ++r)
            for (int d = 0; d < 3; ++d) dir[d] += C[outc[r]].p[d] * ni;
          for (int r = 0; r < ni; ++r)
            for (int d = 0; d < 3; ++d) dir[d] -= C[in[r]].p[d] * no;
          if (ni == 2) {
            R epr[3], eqr[3], eqs[3], eps[3];
            mesh_edge(&C[in[0]], &C[outc[0]], epr);
            mesh_edge(&C[in[1]], &C[outc[0]], eqr);
            mesh_edge(&C[in[1]], &C[outc[1]], eqs);
            mesh_edge(&C[in[0]], &C[outc[1]], eps);
            if (cnt < max_tris) { mesh_put(tris + 9 * cnt, epr, eqr, eqs, dir); ids[cnt] = cell * 12 + 2 * q; }
            ++cnt;
            if (cnt < max_tris) { mesh_put(tris + 9 * cnt, epr, eqs, eps, dir); ids[cnt] = cell * 12 + 2 * q + 1; }
            ++cnt;
          } else {
            const int s = ni == 1 ? in[0] : outc[0];
            const int *rest = ni == 1 ? outc : in;
            R a[3], b[3], c[3];
            mesh_edge(&C[s], &C[rest[0]], a);
            mesh_edge(&C[s], &C[rest[1]], b);
            mesh_edge(&C[s], &C[rest[2]], c);
            if (cnt < max_tris) { mesh_put(tris + 9 * cnt, a, b, c, dir); ids[cnt] = cell * 12 + 2 * q; }
            ++cnt;
          }
        }
      }
  return cnt;
}

/* -------------------------------------------------------- depth filters */

static int cmp_u16(const void *a, const void *b) {
  return (int)*(const uint16_t *)a - (int)*(const uint16_t *)b;
}

/* d_MedianFilter (CameraAbstract.cu:103-124) with in-image windows */
void ora_depth_median5(int32_t w, int32_t h, int32_t null_value, const uint16_t *in, uint16_t *out) {
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      uint16_t v[25];
      int n = 0, win = 0;
      for (int j = -2; j <= 2; ++j)
        for (int i = -2; i <= 2; ++i) {
          const int xx = x + i, yy = y + j;
          if (xx < 0 || xx >= w || yy < 0 || yy >= h) continue;
          ++win;
          const uint16_t d = in[(size_t)yy * w + xx];
          if (d != (uint16_t)null_value) v[n++] = d;
        }
      uint16_t r = (uint16_t)null_value;
      if (n > win / 2) {
        qsort(v, (size_t)n, sizeof(uint16_t), cmp_u16);
        r = (n & 1) ? v[n / 2] : (uint16_t)(((int)v[n / 2 - 1] + (int)v[n / 2]) / 2);
      }
      out[(size_t)y * w + x] = r;
    }
}

/* d_AverageFilter (CameraAbstract.cu:9-34): mean of the 8-neighbours (the
 * in-image ones), compared with the pixel */
void ora_depth_average(int32_t w, int32_t h, int32_t null_value, double thr, const uint16_t *in,
                       uint16_t *out) {
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      double s = 0;
      int n = 0;
      for (int j = -1; j <= 1; ++j)
        for (int i = -1; i <= 1; ++i) {
          const int xx = x + i, yy = y + j;
          if ((i == 0 && j == 0) || xx < 0 || xx >= w || yy < 0 || yy >= h) continue;
          s += in[(size_t)yy * w + xx];
          ++n;
        }
      const double avg = s / n;
      const double v = in[(size_t)y * w + x];
      out[(size_t)y * w + x] = fabs(avg - v) > thr ? (uint16_t)null_value : (uint16_t)avg;
    }
}

/* d_GradientFilter (CameraAbstract.cu:36-71): Prewitt sums with clamped
 * coordinates; gradient / 6 against the threshold */
void ora_depth_gradient(int32_t w, int32_t h, double thr, const uint16_t *in, uint16_t *out,
                        uint8_t *ambig) {
#define CL(a, m) ((a) < 0 ? 0 : ((a) >= (m) ? (m) - 1 : (a)))
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      long gx = 0, gy = 0;
      for (int j = -1; j <= 1; ++j)
        gx += (long)in[(size_t)CL(y + j, h) * w + CL(x + 1, w)] - in[(size_t)CL(y + j, h) * w + CL(x - 1, w)];
      for (int i = -1; i <= 1; ++i)
        gy += (long)in[(size_t)CL(y + 1, h) * w + CL(x + i, w)] - in[(size_t)CL(y - 1, h) * w + CL(x + i, w)];
      const double g2 = (double)(gx * gx + gy * gy), t2 = 36.0 * thr * thr;
      out[(size_t)y * w + x] = g2 > t2 ? 0 : in[(size_t)y * w + x];
      if (ambig) ambig[(size_t)y * w + x] = fabs(g2 - t2) <= 1e-3 * t2;
    }
#undef CL
}

/* d_undistort (CameraAbstract.cu:170-221): the Brown model of the raw image
 * evaluated at the ideal pixel's normalised coordinates (the y term from the
 * undistorted x), bilinear sample of the raw depth */
void ora_depth_undistort(int32_t w, int32_t h, double fx, double fy, double cx, double cy,
                         double k1, double k2, double p1, double p2, int32_t null_value,
                         const uint16_t *in, uint16_t *out, uint8_t *ambig) {
  const uint16_t nv = (uint16_t)null_value;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const double xn = (x - cx) / fx, yn = (y - cy) / fy;
      const double r2 = xn * xn + yn * yn, rad = 1 + k1 * r2 + k2 * r2 * r2;
      const double xd = xn * rad + 2 * p1 * xn * yn + p2 * (r2 + 2 * xn * xn);
      const double yd = yn * rad + p1 * (r2 + 2 * yn * yn) + 2 * p2 * xn * yn;
      const double u = fx * xd + cx, v = fy * yd + cy;
      const double u0f = floor(u), v0f = floor(v);
      const size_t o = (size_t)y * w + x;
      if (ambig) {
        const double fu = u - u0f, fv = v - v0f;
        ambig[o] = fu < 1e-4 || fu > 1 - 1e-4 || fv < 1e-4 || fv > 1 - 1e-4;
      }
      if (u0f < 0 || u0f > w - 1 || v0f < 0 || v0f > h - 1) { out[o] = nv; continue; }
      const int u0 = (int)u0f, v0 = (int)v0f;
      const int u1 = u0 + 1 < w ? u0 + 1 : u0, v1 = v0 + 1 < h ? v0 + 1 : v0;
      const uint16_t a = in[(size_t)v0 * w + u0], b = in[(size_t)v0 * w + u1];
      const uint16_t c = in[(size_t)v1 * w + u0], d = in[(size_t)v1 * w + u1];
      if (a == nv || b == nv || c == nv || d == nv) { out[o] = nv; continue; }
      const double fu = u - u0f, fv = v - v0f;
      const uint16_t f1 = u1 == u0 ? a : (uint16_t)((1 - fu) * a + fu * b);
      const uint16_t f2 = v1 == v0 ? f1 : (u1 == u0 ? c : (uint16_t)((1 - fu) * c + fu * d));
      out[o] = (uint16_t)((1 - fv) * f1 + fv * f2);
    }
}

