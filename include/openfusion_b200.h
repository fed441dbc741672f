/*
 * openfusion_b200.h -- C-ABI of the B200 (sm_100a) KinectFusion per-frame path.
 *
 * Plain C: no CUDA or torch types. Every device pointer is a plain pointer
 * into CUDA device memory of the current device; every stream argument is a
 * cudaStream_t passed as `of_stream_t` (NULL = legacy default stream). Every
 * entry point returns an `of_status_t`; none of them exits the process.
 *
 * Conventions (kept from the reference so that its callers see the same
 * numbers):
 *   - units are millimetres;
 *   - camera space is the reference's: a pixel (u, v) with depth D > 0 (mm)
 *     back-projects to X = -D (u - cx) / fx, Y = -D (v - cy) / fy, Z = -D
 *     (Source/include/CudaUtilities.cuh:24-33, CameraHandler.cu:87), and
 *     projects as u = fx X / Z + cx (CudaUtilities.cuh:9-21);
 *   - a pose is a row-major 4x4 camera-to-world matrix, kept in FP64 on the
 *     device (the reference keeps it as float[16], Source/src/MainApp.cpp:613);
 *   - the TSDF cube of edge `size_mm` is centred at the world origin and voxel
 *     (i, j, k) has its centre at -size/2 + (i + 0.5) size/N
 *     (Source/src/VolumeIntegrator.cu:40-48).
 *
 * Memory is owned by the caller, as in the reference, where RunApp allocates
 * every shared buffer (Source/src/MainApp.cpp:591-647): `*_bytes` queries give
 * the sizes. The tracker object (of_tracker_*) is the exception: it owns the
 * whole per-frame state, like RunApp, and replays the frame as a CUDA graph.
 */
#ifndef OPENFUSION_B200_H_
#define OPENFUSION_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OF_ABI_VERSION 4

typedef int32_t of_status_t;
#define OF_OK 0
#define OF_ERR_INVALID_ARGUMENT 1 /* a size, pointer or parameter is out of range */
#define OF_ERR_CUDA 2             /* a CUDA runtime call failed */
#define OF_ERR_OUT_OF_MEMORY 3    /* the tracker could not allocate device memory */
#define OF_ERR_NOT_READY 4        /* called in the wrong order (e.g. track before the first frame) */
#define OF_ERR_TOO_LARGE 5        /* a size beyond a fixed maximum of the entry point */
#define OF_ERR_IO 6               /* a file could not be opened, read or written */
#define OF_END_OF_SEQUENCE 7      /* a recorded sequence has no more frames */

typedef void *of_stream_t; /* cudaStream_t */

/* TSDF storage of one voxel: one 32-bit word, low half tsdf, high half weight. */
#define OF_TSDF_I16 0 /* int16 tsdf/trunc * 32767 + uint16 weight */
#define OF_TSDF_F16 1 /* IEEE half tsdf/trunc + uint16 weight */

/* Replaces CameraParams (Source/include/BasicTypes.h:88-103); only the fields
 * the fusion path reads (CameraHandler.cu:80-87, VolumeIntegrator.cu:131). */
typedef struct of_camera {
  int32_t width;
  int32_t height;
  float fx, fy, cx, cy;  /* m_intrinsic, pixels */
  float min_depth_mm;    /* m_min_depth */
  float max_depth_mm;    /* m_max_depth */
} of_camera_t;

/* Replaces the compile-time worldVolume / VOLUME_SIZE / TRUNCATION /
 * MAX_WEIGHT constants (Source/include/Constants.h:23-55). */
typedef struct of_volume_desc {
  int32_t resolution; /* N voxels per edge; multiple of 8, 8..1024 */
  int32_t storage;    /* OF_TSDF_I16 or OF_TSDF_F16 */
  float size_mm;      /* cube edge */
  float trunc_mm;     /* truncation distance */
  int32_t max_weight; /* running-average weight cap, 1..65535 */
  int32_t reserved;
} of_volume_desc_t;

/* Depth pre-processing (no reference counterpart: bilateral filter of
 * Tomasi & Manduchi 1998 and the KinectFusion depth pyramid). */
typedef struct of_filter_params {
  float sigma_space_px; /* 4.5 */
  float sigma_range_mm; /* 30 */
  int32_t radius_px;    /* window half-width; 0 = ceil(2 sigma_space); -1 = no filter
                           (raw depth, as CameraHandler.cu:65-89 converts it) */
  int32_t levels;       /* pyramid levels, 1..4 */
} of_filter_params_t;

/* Ray marching (replaces the fixed constants of Source/src/Raycaster.cu:109-112). */
typedef struct of_raycast_params {
  float min_step_vox;    /* smallest march step, voxels (0.75) */
  float far_step_frac;   /* step as a fraction of tsdf*trunc when far from the surface (0.8) */
  int32_t refine_iters;  /* regula-falsi refinements of the zero crossing (3) */
  int32_t tile;          /* pixel block of one CTA (no result depends on it):
                            0 = 16x16, 1 = 32x8, 2 = 8x32, 3 = 32x4, 4 = 16x8,
                            5 = 8x16, 6 = 8x8 */
} of_raycast_params_t;

/* ICP (replaces ICP_ITERATIONS, DISTANCE_THRESHOLD, NORMAL_THRESHOLD,
 * Source/include/Constants.h:48-50). */
typedef struct of_icp_params {
  int32_t levels;          /* 1..4 */
  int32_t iters[4];        /* iterations per level, finest level first: {10, 5, 4} */
  float dist_thresh_mm;    /* 25 */
  float normal_thresh;     /* cosine, 0.65 */
  /* Early exit (no reference counterpart; 0 = always run every iteration):
   * a level ends after an iteration whose increment rotates by less than
   * stop_rot_rad about every axis and translates by less than stop_trans_mm
   * along every axis. */
  float stop_rot_rad;
  float stop_trans_mm;
  /* Judge of a warm-started result (of_icp_track_warm; no reference
   * counterpart): it is replaced by plain ICP from the previous pose when the
   * last iteration's RMS point-to-plane residual exceeds judge_max_rms_mm, its
   * inliers are fewer than judge_min_inlier_frac of the examined model points,
   * or it lies farther than judge_max_rot_rad / judge_max_trans_mm from the
   * warm start (the disagreement with the prediction). */
  float judge_max_rms_mm;
  float judge_min_inlier_frac;
  float judge_max_rot_rad;
  float judge_max_trans_mm;
  /* Pyramid levels a warm-started pass uses, finest first (0 = all): the
   * coarse levels exist to pull in a large initial misalignment, which a
   * good warm start does not have; the judge still guards the result. */
  int32_t warm_levels;
} of_icp_params_t;

/* Per-frame ICP result, written by the device. */
typedef struct of_icp_stats {
  int32_t status;        /* 0 = tracked; 1 = singular system, pose restored (ICP.cpp:152-158);
                            2 = a device-side wait gave up, pose restored */
  int32_t inliers;       /* correspondences of the last iteration run */
  int32_t iterations;    /* iterations run (both passes of a replaced warm start) */
  int32_t warm;          /* 0 = no warm start, 1 = warm start kept, 2 = replaced */
  double residual_sq;    /* sum of squared point-to-plane residuals, mm^2, last iteration */
  double min_pivot;      /* smallest Cholesky pivot / largest diagonal, last iteration */
} of_icp_stats_t;

/* Device layout of a pre-processed frame and of a raycast model: per pyramid
 * level l (0 = finest, W_l = ceil(W / 2^l)), a 256-byte aligned block. */
typedef struct of_pyramid_layout {
  int32_t levels;
  int32_t width[4];
  int32_t height[4];
  size_t depth_offset[4];  /* float depth, mm (frame only; 0 = invalid) */
  size_t points_offset[4]; /* float4 [2 * W_l * H_l]: vertex (x, y, z, valid), normal (x, y, z, valid) */
  size_t total_bytes;
} of_pyramid_layout_t;

/* ---- library --------------------------------------------------------- */

int32_t of_abi_version(void);
const char *of_status_string(of_status_t status);
/* Fills defaults for every parameter block (the values of the full-size
 * 640x480 / 512^3 configuration). Any pointer may be NULL. */
void of_default_params(of_filter_params_t *filter, of_raycast_params_t *raycast,
                       of_icp_params_t *icp);
/* Intrinsics of pyramid level `level` (fx/2^l, cx_{l+1} = (cx_l - 0.5) / 2). */
of_status_t of_camera_level(const of_camera_t *cam, int32_t level, of_camera_t *out);

/* ---- volume (replaces General::InitVoxelArray, General.cpp:42-49) ----- */

/* Bytes of a volume: N^3 x 4 (8^3-voxel bricks, brick-major) followed by one
 * flag byte per brick (brick or a neighbour near a surface), padded to 256. */
of_status_t of_volume_bytes(const of_volume_desc_t *desc, size_t *bytes);
/* Resets every voxel to weight 0 (tsdf reads as +trunc), replacing
 * d_initVoxelArray (Source/src/General.cu:27-50). An unobserved voxel's word
 * holds the +1 tsdf pattern with weight 0. */
of_status_t of_volume_reset(const of_volume_desc_t *desc, void *d_volume, of_stream_t stream);
/* Writes the volume in the reference's layout: float tsdf in mm and the
 * weight, index x*N*N + y*N + z (Source/src/MainApp.cpp:181-276 dumps the
 * same float array). Either output may be NULL. */
of_status_t of_volume_export(const of_volume_desc_t *desc, const void *d_volume,
                             float *d_tsdf_mm, uint16_t *d_weight, of_stream_t stream);
/* Overwrites the volume from the reference layout (for resume / import). */
of_status_t of_volume_import(const of_volume_desc_t *desc, void *d_volume,
                             const float *d_tsdf_mm, const uint16_t *d_weight,
                             of_stream_t stream);

/* ---- pre-processing (replaces CameraHandler::updateCameraData,
 *      Source/src/CameraSupport/CameraHandler.cu:134-143) ----------------- */

of_status_t of_pyramid_layout(const of_camera_t *cam, int32_t levels, of_pyramid_layout_t *out);
/* uint16 depth (mm, row pitch `pitch_px` pixels) -> bilateral-filtered depth
 * pyramid + camera-space vertex and normal maps at every level, into
 * `d_frame` (of_pyramid_layout). Invalid depth (outside [min, max]) is 0. */
of_status_t of_preprocess(const of_camera_t *cam, const of_filter_params_t *filter,
                          const uint16_t *d_depth, int32_t pitch_px, void *d_frame,
                          of_stream_t stream);

/* ---- integration (replaces VolumeIntegrator::Integrate,
 *      Source/src/VolumeIntegrator.cu:86-201) ---------------------------- */

/* Fuses the raw depth frame into the volume at pose `d_pose` (device,
 * FP64 4x4 camera-to-world). `d_lambda` is the per-pixel ray-length table
 * of of_lambda_table (device, float2 [W * H]). */
of_status_t of_integrate(const of_volume_desc_t *desc, void *d_volume, const of_camera_t *cam,
                         const uint16_t *d_depth, int32_t pitch_px, const double *d_pose,
                         const float *d_lambda, of_stream_t stream);
/* Bytes of the ray-length table (W * H * 8). */
of_status_t of_lambda_bytes(const of_camera_t *cam, size_t *bytes);
/* Fills the table: for every pixel, sqrt(1 + ((u-cx)/fx)^2 + ((v-cy)/fy)^2)
 * as an unevaluated float pair (hi, lo), computed in FP64. */
of_status_t of_lambda_table(const of_camera_t *cam, float *d_lambda, of_stream_t stream);
/* The same integration with whole-brick decisions: the call first bounds
 * lambda * D over every 8x8 pixel tile of the frame, then lists the bricks
 * in the frustum, skipping those entirely behind the surface beyond the
 * truncation band and marking those entirely in free space (updated without
 * per-voxel projection), then integrates the listed bricks. `d_scratch` is
 * device scratch of of_integrate_scratch_bytes, 256-byte aligned; two calls
 * in flight must not share it. The volume written is bit-identical to
 * of_integrate's. Also replaces VolumeIntegrator::Integrate. */
of_status_t of_integrate_tiled(const of_volume_desc_t *desc, void *d_volume,
                               const of_camera_t *cam, const uint16_t *d_depth, int32_t pitch_px,
                               const double *d_pose, const float *d_lambda, void *d_scratch,
                               of_stream_t stream);
/* Bytes of of_integrate_tiled's scratch: 768 + 8 B per 8x8 pixel tile + 16 B
 * per 8^3 brick + 8 B per pixel (the frame's lambda * D map), each part
 * rounded up to 256. */
of_status_t of_integrate_scratch_bytes(const of_volume_desc_t *desc, const of_camera_t *cam,
                                       size_t *bytes);
/* Counts the voxels one of_integrate call would update (same decisions, no
 * volume write). `d_count` is one device uint64. */
of_status_t of_integrate_census(const of_volume_desc_t *desc, const void *d_volume,
                                const of_camera_t *cam, const uint16_t *d_depth,
                                int32_t pitch_px, const double *d_pose, const float *d_lambda,
                                unsigned long long *d_count, of_stream_t stream);
/* Counts the voxels in view at `d_pose`: those whose centre projects inside the
 * 2-pixel image border with a depth in [min, max] (the frustum test of
 * VolumeIntegrator.cu:12-16, :131), adding to the device uint64 `d_count`. */
of_status_t of_integrate_visible_census(const of_volume_desc_t *desc, const void *d_volume,
                                        const of_camera_t *cam, const uint16_t *d_depth,
                                        int32_t pitch_px, const double *d_pose,
                                        const float *d_lambda, unsigned long long *d_count,
                                        of_stream_t stream);

/* ---- raycast (replaces Raycaster::Raycast, Source/src/Raycaster.cu:97-242) */

/* Casts one ray per pixel of level 0 from pose `d_pose` and writes world-space
 * vertex/normal maps into `d_model` (of_pyramid_layout; only points_offset
 * is used); pixel (x, y) of level l = 1 .. levels-1 is the ray of level-0
 * pixel (2^l x, 2^l y), written by the same launch. `d_rgba` (may be NULL)
 * receives the reference's shaded image (Raycaster.cu:214-228). */
of_status_t of_raycast(const of_volume_desc_t *desc, const void *d_volume, const of_camera_t *cam,
                       const of_raycast_params_t *params, int32_t levels, const double *d_pose,
                       void *d_model, uint32_t *d_rgba, of_stream_t stream);

/* ---- ICP (replaces ICP::Iterate_ICP, Source/src/ICP.cpp:84-182, with the
 *      correspondence kernel of Source/src/ICP.cu:116-251) --------------- */

of_status_t of_icp_workspace_bytes(const of_camera_t *cam, size_t *bytes);
/* Refines `d_pose` (device FP64 4x4, in/out) of the frame in `d_frame`
 * against the model `d_model`, coarse to fine, all on the device: fused
 * association + point-to-plane rows + compensated 27-value reduction, then
 * an FP64 6x6 Cholesky solve and SE(3) composition by the last block of
 * every iteration. `d_stats` (device, may be NULL) gets of_icp_stats_t. */
of_status_t of_icp_track(const of_camera_t *cam, const of_icp_params_t *params,
                         const void *d_frame, const void *d_model, double *d_pose,
                         void *d_workspace, of_icp_stats_t *d_stats, of_stream_t stream);
/* of_icp_track starting from a warm start (`d_warm_pose`, device FP64 4x4;
 * e.g. of_cnn_warm_pose's). The result is judged (of_icp_params_t judge_*);
 * a rejected one is replaced by plain ICP from `pose`. stats->warm tells
 * which (1 kept, 2 replaced). No reference counterpart. */
of_status_t of_icp_track_warm(const of_camera_t *cam, const of_icp_params_t *params,
                              const void *d_frame, const void *d_model, double *d_pose,
                              const double *d_warm_pose, void *d_workspace,
                              of_icp_stats_t *d_stats, of_stream_t stream);
/* of_icp_track without a workspace argument (no counterpart in the
 * reference): for callers that cannot allocate device memory once they run --
 * hosts that own every device allocation up front, such as plugin hosts with
 * a fixed memory budget, or real-time loops where cudaMalloc's implicit
 * synchronisation and a possible failure mid-session are not acceptable. It
 * allocates nothing: its scratch is one file-scope device array of about
 * 186 KB (per-block partial sums for at most 296 cooperating blocks) that every
 * GPU loading the library holds until the process exits; a device that would
 * need more blocks gets OF_ERR_TOO_LARGE. Every call looks up the array's
 * device address in the current context with cudaGetSymbolAddress (no
 * allocation, no synchronisation); on a device's first call that lookup may
 * load the library's device code, so make that first call before any stream
 * capture. The array starts zeroed when the device code loads. All calls
 * share the one array and each starts by clearing the state it needs
 * cleared; calls whose executions overlap on the GPU race with each other --
 * order them on one stream. Results equal of_icp_track's bit for bit. */
of_status_t of_icp_track_static(const of_camera_t *cam, const of_icp_params_t *params,
                                const void *d_frame, const void *d_model, double *d_pose,
                                of_icp_stats_t *d_stats, of_stream_t stream);
/* Fault injection for failure-detection tests (no reference counterpart):
 * every grid barrier of later of_icp_track calls on this workspace waits for
 * `extra` block arrivals that never come. Each such wait gives up after about
 * 0.15 s; the call then stops, restores the starting pose and reports status 2
 * in of_icp_stats_t. `extra` = 0 restores normal operation. */
of_status_t of_icp_workspace_hold_barrier(void *d_workspace, int32_t extra, of_stream_t stream);
/* One FindCorresponding pass (ICP.cu:116-262) at `level`: the 21 upper
 * J^T J entries (row-major i<=j), 6 J^T r entries, sum r^2 and the inlier
 * count as 29 floats into `d_system`, for the pose `d_pose`. */
of_status_t of_icp_system(const of_camera_t *cam, const of_icp_params_t *params, int32_t level,
                          const void *d_frame, const void *d_model, const double *d_pose,
                          void *d_workspace, float *d_system, of_stream_t stream);
/* One solve-and-compose step on a system of_icp_system wrote: replaces the
 * host half of an ICP::Iterate_ICP iteration (ICP.cpp:142-168: symmetrise,
 * singularity test, LLT solve, rotation part negated) and
 * ICP::BuildNewTransformMatrix (ICP.cu:320-340: dT = [Rz Ry Rx | t],
 * T <- dT T), in FP64 on the device with the tracking kernels' own solve.
 * A singular system (a pivot not above 1e-12 x the largest diagonal entry, or
 * fewer than 6 inliers) leaves `d_pose` unchanged and reports status 1 in
 * `d_stats` (device, may be NULL; iterations = 1). */
of_status_t of_icp_solve_step(const float *d_system, double *d_pose, of_icp_stats_t *d_stats,
                              of_stream_t stream);

/* ---- camera-side depth filters ---------------------------------------- */

/* The filters the reference's cameras run on raw depth
 * (Source/src/CameraSupport/CameraAbstract.cu:9-229; chained by
 * GIPCam.cpp:173-177 and SoftKineticCamera.cpp:424-430), with the intended
 * border handling (neighbours outside the image left out or clamped, not
 * wrapped around). */
#define OF_DEPTH_FILTER_MEDIAN5 1   /* median of the 5x5 window's non-null pixels */
#define OF_DEPTH_FILTER_GRADIENT 2  /* Prewitt: 0 where |gradient| / 6 > threshold */
#define OF_DEPTH_FILTER_AVERAGE 4   /* 8-neighbour mean; null where it differs from the pixel by more than the threshold */
#define OF_DEPTH_FILTER_UNDISTORT 8 /* Brown k1, k2, p1, p2 from the camera's intrinsics */
typedef struct of_depth_filter_params {
  int32_t steps;           /* OF_DEPTH_FILTER_* bits; applied as undistort, median, gradient, average */
  int32_t null_value;      /* depth of an invalid pixel (depthNullValue; 0 for most cameras) */
  int32_t average_passes;  /* average applied this many times (GIPCam: 2) */
  float average_threshold_mm;   /* 15 */
  float gradient_threshold_mm;  /* 10 */
  float k1, k2, p1, p2;
} of_depth_filter_params_t;
void of_depth_filter_defaults(of_depth_filter_params_t *params);
/* The chain `params->steps` from d_in to d_out (may be equal); `d_scratch`
 * (W x H uint16, distinct from both) is needed for more than one step or in
 * place. Runs on `stream` without synchronising. */
of_status_t of_depth_filter(const of_camera_t *cam, const of_depth_filter_params_t *params,
                            const uint16_t *d_in, uint16_t *d_out, uint16_t *d_scratch,
                            of_stream_t stream);
/* One filter (`kind` = one OF_DEPTH_FILTER_* bit) from d_in to d_out (distinct). */
of_status_t of_depth_filter_step(const of_camera_t *cam, int32_t kind,
                                 const of_depth_filter_params_t *params, const uint16_t *d_in,
                                 uint16_t *d_out, of_stream_t stream);

/* ---- tracker: the whole frame (RunApp::display, MainApp.cpp:786-964) ---- */

typedef struct of_tracker *of_tracker_t;

typedef struct of_tracker_desc {
  of_camera_t camera;
  of_volume_desc_t volume;
  of_filter_params_t filter;
  of_raycast_params_t raycast;
  of_icp_params_t icp;
  double initial_pose[16]; /* camera-to-world of frame 0 */
  int32_t use_graph;       /* 1 = replay each frame as a captured CUDA graph */
  int32_t pose_history;    /* frames of pose history kept on the device (0 = 1024) */
  /* Learned warm start: host FP32 weights of the warm-start CNN
   * (of_cnn_param_count floats; NULL = plain ICP from the previous pose).
   * Needs W = 80 k, H = 60 k. Each tracked frame then runs the CNN on the
   * (previous, current) depth pair and of_icp_track_warm. */
  const float *warm_start_weights;
  /* Camera-side filters applied in place to each depth frame before it is
   * used (steps = 0: none). */
  of_depth_filter_params_t depth_filter;
  /* Online tuning of the launch shapes that change no result (no reference
   * counterpart). 0: raycast.tile is used as given. k >= 1: step k times
   * every raycast block shape (of_raycast_params_t.tile) on the volume it has
   * just fused, at its tracked pose, into a scratch model (five launches each,
   * interleaved), keeps the one with the least median time (of_tracker_tuning),
   * and only then captures the step graphs; the steps
   * before it run without graphs and step k synchronises its stream. */
  int32_t tune;
} of_tracker_desc_t;

of_status_t of_tracker_create(const of_tracker_desc_t *desc, of_tracker_t *out);
of_status_t of_tracker_destroy(of_tracker_t tracker);
/* Processes one depth frame in the reference's order (RunApp::display,
 * MainApp.cpp:786-964): the previous frame is fused at its tracked pose and
 * the model raycast there, while this frame is pre-processed (graph
 * branches); then this frame is tracked against that model. Frame 0 only
 * sets the pose (its initial pose). The pose is this frame's when the call's
 * work completes; the volume and model hold the frames before it until the
 * next call or of_tracker_flush. `depth_is_host` != 0: `depth` is host memory,
 * copied on `stream`; with graphs, a pinned buffer (cudaMallocHost /
 * cudaHostRegister) is copied by the step itself at the head of the
 * pre-processing branch, beside the fusion of the previous frame, and any
 * other host buffer before the step. The buffer must stay unchanged until the
 * call's work completes. */
of_status_t of_tracker_process(of_tracker_t tracker, const uint16_t *depth, int32_t depth_is_host,
                               of_stream_t stream);
/* Fuses the last processed frame at its pose and raycasts the model there
 * now (before reading the volume or the model); the next
 * of_tracker_process then skips that fusion. No effect when already done. */
of_status_t of_tracker_flush(of_tracker_t tracker, of_stream_t stream);
/* Sets the starting pose of the next frame's ICP to `pose_delta` x previous
 * pose (host FP64 4x4, world frame); used for a warm start. NULL clears it. */
of_status_t of_tracker_set_prior(of_tracker_t tracker, const double *pose_delta);
/* Copies the current pose (FP64 4x4) to `pose` (host; asynchronous on
 * `stream` when the buffer is pinned) and, if `stats` != NULL, the last
 * frame's ICP statistics. */
of_status_t of_tracker_pose(of_tracker_t tracker, double *pose, of_icp_stats_t *stats,
                            of_stream_t stream);
/* Copies the poses of the last `count` frames (oldest first) to host memory. */
of_status_t of_tracker_pose_history(of_tracker_t tracker, double *poses, int32_t count,
                                    of_stream_t stream);
/* Checkpoint / resume: the tracker's state (volume with its brick bytes,
 * pose, pose history, frame count and the last depth frame, which the next
 * step fuses) to one file with a header, and back into a tracker created
 * with the same camera, volume and pose_history (else
 * OF_ERR_INVALID_ARGUMENT). A resumed tracker continues bit for bit as the
 * saved one would have. Synchronises `stream`; host memory for one copy of
 * the volume is allocated during the call. The reference saves only the raw
 * float volume (Source/src/MainApp.cpp:259-268) and the pose (:430-451). */
of_status_t of_tracker_save(of_tracker_t tracker, const char *path, of_stream_t stream);
of_status_t of_tracker_load(of_tracker_t tracker, const char *path, of_stream_t stream);
/* Raw device pointers of the tracker's state, for inspection and for the
 * reference-shaped C++ wrappers. */
typedef struct of_tracker_buffers {
  void *volume;
  void *frame;
  void *model;
  double *pose;
  uint16_t *depth;
  float *lambda;
  of_icp_stats_t *stats;
  int64_t frames;
  int32_t kernels_first;  /* kernel launches of frame 0's graph */
  int32_t kernels_track;  /* kernel launches of every later step's graph */
} of_tracker_buffers_t;
of_status_t of_tracker_buffers(of_tracker_t tracker, of_tracker_buffers_t *out);
/* The raycast block shape in use (of_raycast_params_t.tile) and whether the
 * online tuning has run (of_tracker_desc_t.tune). */
of_status_t of_tracker_tuning(of_tracker_t tracker, int32_t *ray_tile, int32_t *tuned);

/* ---- surface mesh and volume file (no GL) ----------------------------- */

/* Triangle mesh of the tsdf = 0 surface of the observed voxels (marching
 * tetrahedra: 6 tetrahedra per cell of 8 voxels; no cracks; triangles face
 * the free space). The reference's own extraction is commented out
 * (Source/src/MainApp.cpp:277-328). Writes up to `max_triangles` triangles as
 * 9 floats (3 vertices, world mm) to `d_triangles` and, if `d_ids` is not
 * NULL, one id each (cell * 12 + 2 * tetrahedron + k, cell = (i n + j) n + k
 * of its lowest voxel); `d_count` (device) receives the surface's triangle
 * count, which may exceed `max_triangles` (call again with room for all).
 * Triangle order is not fixed; ids identify them. */
of_status_t of_mesh_extract(const of_volume_desc_t *desc, const void *d_volume, float *d_triangles,
                            uint64_t *d_ids, uint32_t max_triangles, uint32_t *d_count,
                            of_stream_t stream);
/* Host triangles (9 floats each) as a Wavefront OBJ file (vertices and
 * 1-based faces). */
of_status_t of_mesh_write_obj(const char *path, const float *triangles, uint32_t count);
/* The volume as the reference's SavedVolume.raw: N^3 float tsdf in mm, index
 * x N^2 + y N + z, unobserved voxels +truncation (RunApp::saveVolumeToFile,
 * Source/src/MainApp.cpp:181-276). Allocates N^3 x 6 bytes of device memory
 * and N^3 x 4 bytes of host memory for the call. */
of_status_t of_volume_save_raw(const of_volume_desc_t *desc, const void *d_volume, const char *path,
                               of_stream_t stream);

/* ---- recorded sequences (the reference's on-disk format) -------------- */

/* A recording directory holds `Parameters.txt` and raw frames `recorded1`,
 * `recorded2`, ... (W x H uint16 depth in mm, row major): the format of
 * Source/data/ParametersFileFormat.txt:1-11, as CameraFromFile reads it
 * (Source/src/CameraSupport/CameraFromFile.cpp:22-98) and WriteToFile writes
 * it (WriteToFile.cpp:18-145). */
typedef struct of_recording_info {
  of_camera_t camera;   /* width, height, fx, fy, cx, cy, min/max depth (mm) */
  float z_offset_mm;    /* "Z offset in mm (for GIP, otherwise 0)" */
  int32_t frames;       /* "Number of frames" (0 if absent) */
  char name[256];
  char date[64];
  char camera_type[64];
} of_recording_info_t;
of_status_t of_recording_read_info(const char *dir, of_recording_info_t *info);
of_status_t of_recording_write_info(const char *dir, const of_recording_info_t *info);
/* Frame `number` (1-based, as the reference counts) to / from host memory;
 * the writer also takes device memory (`depth_is_device`, copied on `stream`). */
of_status_t of_recording_read_frame(const char *dir, int32_t number, int32_t width,
                                    int32_t height, uint16_t *depth);
of_status_t of_recording_write_frame(const char *dir, int32_t number, int32_t width,
                                     int32_t height, const uint16_t *depth,
                                     int32_t depth_is_device, of_stream_t stream);

/* A recording as a frame source: one background thread reads `prefetch`
 * frames ahead into pinned host buffers; of_reader_next copies the next frame
 * to device memory with one asynchronous copy on `stream` (the buffer is
 * reused only after that copy completes) and returns OF_END_OF_SEQUENCE after
 * the last frame. Replaces CameraFromFile::GetDepthFrame's synchronous read
 * and cudaMemcpy (CameraFromFile.cpp:73-98). */
typedef struct of_reader *of_reader_t;
of_status_t of_reader_open(const char *dir, int32_t prefetch, of_reader_t *out);
of_status_t of_reader_info(of_reader_t reader, int32_t *width, int32_t *height, int32_t *frames);
of_status_t of_reader_next(of_reader_t reader, uint16_t *d_depth, of_stream_t stream);
of_status_t of_reader_close(of_reader_t reader);

/* ---- many independent streams (batched) ------------------------------- */

/* One depth stream of a batch: its camera, volume and initial pose. */
typedef struct of_batch_stream {
  of_camera_t camera;
  of_volume_desc_t volume;  /* all streams of a batch use the same storage */
  double initial_pose[16];  /* camera-to-world of its frame 0 */
} of_batch_stream_t;

/* Tuning knobs of the batched stages; none changes a result. */
typedef struct of_batch_tuning {
  int32_t ray_tile;      /* raycast block (of_raycast_params_t.tile): 0 = 16x16, 1 = 32x8,
                            2 = 8x32, 3 = 32x4, 4 = 16x8, 5 = 8x16, 6 = 8x8 */
  int32_t list_div;      /* integration blocks per stream = bricks / {16,32,64,128,256}[list_div] */
  int32_t icp_clusters;  /* resident 8-CTA clusters of the batched ICP (0 = as many as fit) */
  int32_t tuned;         /* (of_batch_tuning) 1 = chosen by measurement */
} of_batch_tuning_t;

typedef struct of_batch_desc {
  int32_t count;                     /* streams */
  const of_batch_stream_t *streams;  /* count entries (copied) */
  of_filter_params_t filter;         /* shared by all streams */
  of_raycast_params_t raycast;
  of_icp_params_t icp;
  int32_t use_graph;  /* 1 = replay each step as a captured CUDA graph */
  int32_t tune;       /* 1 = choose the knobs online by timing candidates on the first steps */
  of_batch_tuning_t tuning;  /* the knobs when tune == 0 (start values otherwise) */
} of_batch_desc_t;

typedef struct of_batch *of_batch_t;

/* Many independent streams tracked and fused together, one launch per stage
 * for all of them (the tracker's step order for every stream): batched
 * filter + pyramid + maps, integration, raycast, and one persistent launch of
 * thread-block clusters for every stream's ICP. Per stream, every stage but
 * ICP writes what the single-stream stage writes; ICP sums in another order.
 * No reference counterpart (the reference runs one camera). */
of_status_t of_batch_create(const of_batch_desc_t *desc, of_batch_t *out);
of_status_t of_batch_destroy(of_batch_t batch);
/* One frame of every stream: `depth[i]` (count pointers; host memory when
 * `depth_is_host`, copied on `stream`) is stream i's next frame. */
of_status_t of_batch_process(of_batch_t batch, const uint16_t *const *depth, int32_t depth_is_host,
                             of_stream_t stream);
/* Fuses every stream's last frame now (see of_tracker_flush). */
of_status_t of_batch_flush(of_batch_t batch, of_stream_t stream);
/* Current poses (count x 16 FP64, host) and optionally each stream's last
 * ICP statistics (count entries), copied on `stream`. */
of_status_t of_batch_poses(of_batch_t batch, double *poses, of_icp_stats_t *stats,
                           of_stream_t stream);
/* The knobs in use (after tuning: the measured winners). */
of_status_t of_batch_tuning(of_batch_t batch, of_batch_tuning_t *out);
/* Device pointers of stream i's state (volume, pyramids, pose, ...). */
of_status_t of_batch_stream_buffers(of_batch_t batch, int32_t i, of_tracker_buffers_t *out);
/* Host-only planning: a stream's per-frame work in voxel-visit units, and a
 * longest-first greedy assignment of streams to `ranks` GPUs. */
of_status_t of_batch_stream_cost(const of_batch_stream_t *stream, const of_icp_params_t *icp,
                                 double *cost);
of_status_t of_batch_shard(const double *cost, int32_t count, int32_t ranks,
                           int32_t *rank_of_stream);

/* ---- reference-layout adapters (for the reference's PointInfo /
 *      CameraData: AoS float3, BAD_VERTEX = FLT_MAX, BasicTypes.h:40-49) --- */

/* Headless views (RGBA8 words, as the reference packs them for its
 * windows, rgbaFloatToIntCamera, Source/src/CameraSupport/CameraHandler.cu:55-62):
 * depth as gray depth / max depth, opaque (CameraHandler.cu:75-78); level-0
 * normals of a frame or model as (n + 1) / 2 with alpha `alpha`
 * (CameraHandler.cu:128-131: 1; the raycast's show-normals mode,
 * Raycaster.cu:214-218: 0), world space when `d_pose` (frame maps) is given.
 * The raycast's shaded view is of_raycast's `rgba` output. */
of_status_t of_depth_to_rgba(const of_camera_t *cam, const uint16_t *d_depth, uint32_t *d_rgba,
                             of_stream_t stream);
of_status_t of_normals_to_rgba(const of_camera_t *cam, const void *d_pyramid, const double *d_pose,
                               float alpha, uint32_t *d_rgba, of_stream_t stream);
/* Level 0 of a model/frame -> AoS float3 maps; invalid vertex = FLT_MAX,
 * invalid normal = 0. If `d_pose` is not NULL the points are camera-space
 * and are transformed to world space first (frame maps). */
of_status_t of_points_to_reference(const of_camera_t *cam, const void *d_pyramid,
                                   const double *d_pose, float *d_vertex3, float *d_normal3,
                                   of_stream_t stream);
/* AoS float3 world maps (reference PointInfo) -> level 0.. of a model. */
of_status_t of_points_from_reference(const of_camera_t *cam, int32_t levels,
                                     const float *d_vertex3, const float *d_normal3,
                                     void *d_model, of_stream_t stream);
/* float[16] pose <-> FP64 device pose. With `invert` != 0 the input is a
 * world-to-camera matrix (the reference's d_invCurrentTransform) and the
 * camera-to-world pose is its rigid inverse, formed in FP64. */
of_status_t of_pose_from_float(const float *d_pose_f32, double *d_pose, int32_t invert,
                               of_stream_t stream);
of_status_t of_pose_to_float(const double *d_pose, float *d_pose_f32, float *d_inv_pose_f32,
                             float *d_camera_position3, of_stream_t stream);

/* ---- learned ICP warm start (no reference counterpart: the reference
 *      starts ICP at the previous pose, Source/src/ICP.cpp:84-182) -------- */

/* A small BF16 CNN maps the pair (previous, current) of depth frames, block-
 * averaged to 80x60, to the camera motion between them: 6 outputs, the
 * rotation vector of R_prev^T R_cur times 10 (rad) and its translation
 * R_prev^T (t_cur - t_prev) divided by 100 (mm). Parameters live twice on the
 * device: FP32 master values (`d_master`, of_cnn_param_count floats; biases
 * are read from them) and their BF16 copies (`d_params`, uint16 bit patterns,
 * same count). Activations are stored in BF16, every sum runs in FP32, and
 * every reduction in a fixed order, so results are reproducible. */
of_status_t of_cnn_param_count(int64_t *count);
/* Bytes of the per-batch workspace of of_cnn_forward / of_cnn_backward. */
of_status_t of_cnn_workspace_bytes(int32_t batch, size_t *bytes);
/* He-uniform weights and zero biases from a seed. */
of_status_t of_cnn_init(float *d_master, uint16_t *d_params, uint64_t seed, of_stream_t stream);
/* Network input (BF16, batch x 2 x 60 x 80) of `batch` pairs of uint16 depth
 * frames of W x H (W = 80 k, H = 60 k), from the mean of each k x k block's
 * valid depths in metres: channel 0 the previous frame's block means minus
 * their mean over its non-empty blocks, channel 1 current minus previous
 * block mean; empty blocks give 0. Pair i is at d_prev + i * pair_stride and
 * d_cur + i * pair_stride (pixels). `d_cells`: scratch of batch x 2 x 60 x 80
 * floats. */
of_status_t of_cnn_input(const uint16_t *d_prev, const uint16_t *d_cur, int32_t width,
                         int32_t height, int32_t batch, int64_t pair_stride, float *d_cells,
                         uint16_t *d_input, of_stream_t stream);
/* Forward pass; `d_out` (may be NULL) receives batch x 6 floats. */
of_status_t of_cnn_forward(const uint16_t *d_params, const float *d_master,
                           const uint16_t *d_input, int32_t batch, void *d_workspace,
                           float *d_out, of_stream_t stream);
/* Forward and backward pass of the loss mean_b sum_k w_k (out_bk - target_bk)^2
 * (`d_loss_weights`: 6 floats): writes the gradient of every parameter into
 * `d_grad` (param-count floats) and the loss into `d_loss` (may be NULL). */
of_status_t of_cnn_backward(const uint16_t *d_params, const float *d_master,
                            const uint16_t *d_input, int32_t batch, const float *d_target,
                            const float *d_loss_weights, void *d_workspace, float *d_grad,
                            float *d_loss, of_stream_t stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8, bias-corrected; `step` counts
 * from 1) on the master values; refreshes their BF16 copies. */
of_status_t of_cnn_adam(float *d_master, uint16_t *d_params, const float *d_grad, float *d_m,
                        float *d_v, int32_t step, float lr, of_stream_t stream);
/* The prediction for one pair in one launch (one cluster of 16 CTAs, one per
 * SM, each staging its slice of the weights in shared memory and sharing the
 * activations through distributed shared memory): of_cnn_input,
 * of_cnn_forward and of_cnn_warm_pose fused, with the same arithmetic up to
 * the order of each output's sums. `d_out` (6 floats) and `d_warm_pose` (with
 * `d_prev_pose`) may each be NULL. W / 80 = H / 60 must be 1, 2, 4 or 8;
 * `d_params` and both depth frames 16-byte aligned. No scratch memory. */
of_status_t of_cnn_predict(const uint16_t *d_params, const float *d_master,
                           const uint16_t *d_prev, const uint16_t *d_cur, int32_t width,
                           int32_t height, const double *d_prev_pose, float *d_out,
                           double *d_warm_pose, of_stream_t stream);
/* BF16 copies of (loaded) master values. */
of_status_t of_cnn_load(const float *d_master, uint16_t *d_params, of_stream_t stream);
/* Warm start from a prediction: d_warm_pose = d_prev_pose x [exp(w) | t] with
 * w = out[0..2] / 10 (rad), t = 100 out[3..5] (mm); FP64 4x4 device poses. */
of_status_t of_cnn_warm_pose(const float *d_out, const double *d_prev_pose, double *d_warm_pose,
                             of_stream_t stream);

/* ---- synthetic sequences on the device (test and training data) ------- */

/* Renders `frames` uint16 depth frames (frame i at camera-to-world pose
 * d_poses[16 i .. 16 i + 15], noise counter first_frame + i) of a scene built
 * by of_synth_scene (`d_scene`: an of_synth_scene_t copied to the device), with
 * the seeded renderer of libof_synth (of_synth_render); output frame i at
 * d_depth + i * W * H. */
of_status_t of_synth_render_device(const void *d_scene, int32_t width, int32_t height, float fx,
                                   float fy, float cx, float cy, const double *d_poses,
                                   int32_t frames, uint64_t noise_seed, int32_t first_frame,
                                   float sigma_scale, float dropout, uint16_t *d_depth,
                                   of_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* OPENFUSION_B200_H_ */
