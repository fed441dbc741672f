/* of_oracle.h -- CPU restatement of the KinectFusion per-frame path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the CUDA path is compared
 * against; it is never linked into, called by or shipped with the product
 * (openfusion_b200/). Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.
 *
 * The same source builds twice:
 *   liboracle_f64.so   -- OF_REAL = double: the FP64 oracle (parity checker)
 *   libcpu_f32_omp.so  -- OF_REAL = float:  a straightforward FP32 OpenMP CPU
 *                         implementation of the same equations (CPU baseline)
 *
 * Pinning: the reference (gilbs10/OpenFusion) ships no tests, golden vectors or
 * recordings. The stages with a reference counterpart are pinned against the
 * reference's own kernel sources compiled for the host and run here
 * (oracle/ref_harness, fixtures in tests/golden/). The stages the reference
 * does not have (bilateral filter, pyramid, trilinear raycast, FP64 Cholesky)
 * restate the published methods cited at each function.
 */
#ifndef OF_ORACLE_H_
#define OF_ORACLE_H_

#include <stdint.h>

#ifndef OF_REAL
#define OF_REAL double
#endif
typedef OF_REAL ora_real;

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_cam {
  int32_t w, h;
  double fx, fy, cx, cy;
  double dmin, dmax;
} ora_cam;

typedef struct ora_vol {
  int32_t n;        /* voxels per edge */
  int32_t storage;  /* 0 = int16, 1 = fp16 */
  double size;      /* mm */
  double trunc;     /* mm */
  int32_t max_w;
  int32_t pad;
} ora_vol;

typedef struct ora_params {
  double sigma_s, sigma_r;
  int32_t radius, levels;
  int32_t iters[4];
  double dist_thresh, normal_thresh;
  double min_step_vox, far_step_frac;
  int32_t refine_iters;
  int32_t pad;
} ora_params;

int32_t ora_real_bytes(void);
void ora_cam_level(const ora_cam *c, int32_t level, ora_cam *out);

/* pre-processing; pts is [h*w][8]: vertex xyz valid, normal xyz valid */
void ora_bilateral(const ora_cam *c, const uint16_t *depth, double sigma_s, double sigma_r,
                   int32_t radius, ora_real *out);
void ora_pyr_down(const ora_real *src, int32_t sw, int32_t sh, ora_real *dst, int32_t dw,
                  int32_t dh, double guard);
void ora_vertex_normal(const ora_cam *c, const ora_real *depth, ora_real *pts);
/* whole pyramid: for level l, depth_l and pts_l are laid out one after the
 * other: [depth_0 | pts_0 | depth_1 | pts_1 ...] (sizes w_l*h_l and 8*w_l*h_l) */
void ora_preprocess(const ora_cam *c, const ora_params *p, const uint16_t *depth, ora_real *out);
int64_t ora_pyramid_elems(const ora_cam *c, int32_t levels);

/* integration into linear-layout voxel words (index (i*n + j)*n + k); returns
 * the number of voxels updated. ambig (may be NULL, n^3 bytes) flags voxels
 * whose decisions lie within FP32 rounding of a boundary. */
int64_t ora_integrate(const ora_vol *v, uint32_t *words, const ora_cam *c, const uint16_t *depth,
                      const double *pose, uint8_t *ambig);

/* raycast; pts is [h*w][8] world vertex/normal; flags (may be NULL): one
 * byte per brick for empty-space skipping; ambig (may be NULL) flags pixels
 * whose sign or range decisions are within rounding of a boundary, hits
 * whose refined surface moves by more than 0.02 mm when the bracket moves by
 * 0.01 mm (unconverged refinement), and rays whose hit or surface changes when
 * every march position moves by 2e-3 mm (the result depends on FP rounding). */
void ora_raycast(const ora_vol *v, const uint32_t *words, const uint8_t *flags, const ora_cam *c,
                 const ora_params *p, const double *pose, ora_real *pts, uint8_t *ambig);
/* the march of chosen pixels (xy[2 i], xy[2 i + 1]) under each position
 * perturbation perts[k] (mm per update): out[(i npert + k) 4] = vertex, 1 or
 * zeros on a miss */
void ora_raycast_pixels(const ora_vol *v, const uint32_t *words, const uint8_t *flags,
                        const ora_cam *c, const ora_params *p, const double *pose, int32_t npix,
                        const int32_t *xy, int32_t npert, const double *perts, ora_real *out);
/* the trilinear tsdf / trunc at world points xyz[3 i .. 3 i + 2] */
void ora_tsdf_at(const ora_vol *v, const uint32_t *words, int64_t npts, const double *xyz,
                 ora_real *out);
/* model level l+1 from level l by subsampling (2x, 2y) */
void ora_model_down(const ora_real *src, int32_t sw, ora_real *dst, int32_t dw, int32_t dh);

/* one correspondence pass at one level: out[29] = 21 upper A^T A, 6 A^T b,
 * sum b^2, inliers; amb[29] (may be NULL) = sum of |contribution| of pixels
 * whose association or gates lie within rounding of a boundary. */
void ora_icp_system(const ora_cam *lc, const ora_real *frame_pts, int32_t mw, int32_t mh,
                    const ora_real *model_pts, const double *pose, double dist_thresh,
                    double normal_thresh, double *out, double *amb);
/* solve + compose; returns 0 ok, 1 singular (pose untouched) */
int32_t ora_icp_step(const double *sys, double *pose, double *min_pivot);
/* multi-level ICP from pyramids laid out as ora_preprocess writes them (the
 * model uses the same layout; its depth planes are ignored). Returns status. */
int32_t ora_icp_track(const ora_cam *c, const ora_params *p, const ora_real *frame,
                      const ora_real *model, double *pose, int32_t *iterations);

/* options and result of ora_icp_track_ex: early exit, warm start, judge */
typedef struct ora_icp_opts {
  double stop_rot, stop_trans;  /* early exit thresholds (rad, mm); stop_rot 0 = off */
  int32_t warm_levels;          /* finest levels of a warm-started pass (0 = all) */
  int32_t pad;
  double judge_rms, judge_frac, judge_rot, judge_trans;
} ora_icp_opts;
typedef struct ora_icp_result {
  int32_t status;          /* 0 tracked, 1 singular (starting pose restored) */
  int32_t iterations;      /* both passes */
  int32_t warm;            /* 0 no warm start, 1 kept, 2 replaced by plain ICP */
  int32_t inliers;         /* last iteration */
  int32_t examined;        /* model points of the last iteration that landed in the frame */
  int32_t decisions_near;  /* exit/judge decisions within 1 % of a threshold */
  double residual_sq;      /* last iteration */
} ora_icp_result;
/* ora_icp_track with the early exit and an optional warm start (`warm`, FP64
 * 4x4, or NULL) judged as the device path judges it. Returns status. */
int32_t ora_icp_track_ex(const ora_cam *c, const ora_params *p, const ora_icp_opts *o,
                         const ora_real *frame, const ora_real *model, double *pose,
                         const double *warm, ora_icp_result *res);

/* ---- reference semantics (pinned against the reference's own kernels) ---- */
typedef struct ora_refcam {
  int32_t w, h;
  double fx, fy, cx, cy;      /* m_intrinsic */
  double ifx, ify, icx, icy;  /* m_invIntrinsic */
  double dmin, dmax;
} ora_refcam;

typedef struct ora_refvol {
  int32_t n;       /* VOLUME_SIZE */
  int32_t b1;      /* 1: the kernel's storage shift (voxel x in slab x + 1) */
  double world;    /* worldVolume, mm */
  double trunc;    /* TRUNCATION, mm */
  int32_t max_w;   /* MAX_WEIGHT */
  int32_t pad;
} ora_refvol;

void ora_ref_convert(const ora_refcam *c, const uint16_t *depth, const double *T, double *vertex,
                     double *normal);
void ora_ref_integrate_voxels(const ora_refvol *v, const ora_refcam *c, const double *vertex,
                              const double *invT, const double *cpos, const int64_t *storage,
                              int64_t count, const double *prev_tsdf, const int32_t *prev_w,
                              double *out_tsdf, int32_t *out_w, uint8_t *ambig);
void ora_ref_integrate_full(const ora_refvol *v, const ora_refcam *c, const double *vertex,
                            const double *invT, const double *cpos, float *tsdf, uint8_t *w);
void ora_ref_raycast(const ora_refvol *v, const float *tsdf, const ora_refcam *c, const double *T,
                     const double *cpos, double *vertex, double *normal, uint8_t *ambig);
void ora_ref_icp_system(const ora_refcam *c, const uint16_t *new_depth, const double *new_vertex,
                        const double *new_normal, const double *model_vertex,
                        const double *model_normal, const double *invT, double *out36,
                        double *out6, double *amb36, double *amb6);
void ora_ref_compose(const double *xopt, double *T, double *full);

/* Mesh of the tsdf = 0 surface by marching tetrahedra (Kuhn's 6 tetrahedra
 * per cell, cells of 8 observed voxels), linear-layout words. Writes up to
 * `max_tris` triangles (9 reals each) and their ids (cell * 12 + 2 tet + k,
 * cell = (i n + j) n + k), in id order; returns the number of triangles. */
int64_t ora_mesh(const ora_vol *v, const uint32_t *words, ora_real *tris, uint64_t *ids,
                 int64_t max_tris);

/* Camera-side depth filters (Source/src/CameraSupport/CameraAbstract.cu:9-229)
 * on uint16 depth, with the intended border handling: neighbours outside the
 * image are left out (median, average) or clamped (gradient).
 *   median5:  median of the window's non-null pixels (mean of the middle two,
 *             truncated, for an even count); null unless more than half of the
 *             window's in-image pixels are non-null
 *   average:  mean of the in-image 8-neighbours; null when it differs from the
 *             pixel by more than `thr`, else the mean truncated
 *   gradient: Prewitt sums gx, gy; 0 where (gx/6)^2 + (gy/6)^2 > thr^2
 *   undistort: Brown model (k1, k2 radial, p1, p2 tangential) from the ideal
 *             pixel to the raw image, bilinear with truncated row values;
 *             null outside the image or where a tap is null. `ambig` flags
 *             pixels whose source lies within 1e-4 px of a tap boundary. */
void ora_depth_median5(int32_t w, int32_t h, int32_t null_value, const uint16_t *in, uint16_t *out);
void ora_depth_average(int32_t w, int32_t h, int32_t null_value, double thr, const uint16_t *in,
                       uint16_t *out);
void ora_depth_gradient(int32_t w, int32_t h, double thr, const uint16_t *in, uint16_t *out,
                        uint8_t *ambig);
void ora_depth_undistort(int32_t w, int32_t h, double fx, double fy, double cx, double cy,
                         double k1, double k2, double p1, double p2, int32_t null_value,
                         const uint16_t *in, uint16_t *out, uint8_t *ambig);

/* CPU tracker: the whole frame loop (used as the CPU baseline) */
typedef struct ora_tracker ora_tracker;
ora_tracker *ora_tracker_create(const ora_cam *c, const ora_vol *v, const ora_params *p,
                                const double *pose0);
void ora_tracker_destroy(ora_tracker *t);
int32_t ora_tracker_process(ora_tracker *t, const uint16_t *depth);
void ora_tracker_pose(const ora_tracker *t, double *pose);
uint32_t *ora_tracker_volume(ora_tracker *t);
int32_t ora_threads(void);

#ifdef __cplusplus
}
#endif

#endif
