/* of_synth.h -- seeded synthetic depth sequences (host C++, OpenMP).
 *
 * The reference replays recorded uint16 depth frames (CameraFromFile.cpp:68-92);
 * no recordings ship, so benchmarks and tests render analytic scenes instead:
 * rooms of planes, spheres and boxes seen by a camera in the reference's
 * convention (camera looks along -z, X = -D (u-cx)/fx, Y = -D (v-cy)/fy),
 * with the axial noise model sigma(z) = 0.0012 + 0.0019 (z - 0.4)^2 m of
 * Nguyen, Izadi & Lovell (3DIMPVT 2012) and random dropout. Every random draw
 * is a counter-based hash of (seed, frame, pixel), so results do not depend
 * on the thread count. */
#ifndef OF_SYNTH_H_
#define OF_SYNTH_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OF_SYNTH_MAX_PRIMS 64
#define OF_PRIM_PLANE 0
#define OF_PRIM_SPHERE 1
#define OF_PRIM_BOX 2

typedef struct of_synth_prim {
  int32_t kind;
  float p[10]; /* plane: n(3), d (n.x = d); sphere: c(3), r; box: c(3), half(3), yaw */
} of_synth_prim_t;

typedef struct of_synth_scene {
  int32_t count;
  float room_half_mm;
  of_synth_prim_t prims[OF_SYNTH_MAX_PRIMS];
} of_synth_scene_t;

/* kind 0: box room of 4 planes + 6 spheres (r ~ U[100, 400] mm) in a cube of
 *         edge `cube_mm`; kind 1: room + 20 random boxes and spheres. */
int32_t of_synth_scene(int32_t kind, uint64_t seed, float cube_mm, of_synth_scene_t *out);

/* Camera-to-world poses (row-major 4x4, mm) of `frames` frames.
 * motion 0: smooth sweep around the scene, <= 10 mm and <= 0.5 deg per frame;
 * motion 1: large motion, each frame perturbed by up to 50 mm / 2.5 deg so
 *           consecutive frames differ by up to ~100 mm / 5 deg. */
int32_t of_synth_trajectory(int32_t motion, uint64_t seed, float cube_mm, int32_t frames,
                            double *poses);

/* Renders one uint16 depth frame (mm, 0 = no return). `sigma_scale` scales
 * the axial noise (0 = exact depth rounded to mm), `dropout` is the fraction
 * of pixels set to 0. `exact_mm` (may be NULL) receives the noise-free depth. */
int32_t of_synth_render(const of_synth_scene_t *scene, int32_t width, int32_t height, float fx,
                        float fy, float cx, float cy, const double *pose, uint64_t noise_seed,
                        int32_t frame, float sigma_scale, float dropout, uint16_t *depth,
                        float *exact_mm);

#ifdef __cplusplus
}
#endif

#endif
