// of_synth.cpp -- seeded analytic depth scenes, trajectories and rendering.
#include "of_synth.h"

#include <math.h>
#include <string.h>

namespace {

inline uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

inline uint64_t hash3(uint64_t a, uint64_t b, uint64_t c) {
  return mix64(a ^ mix64(b ^ mix64(c)));
}

inline double unit(uint64_t h) { return ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

struct Rng {  // sequential stream for scene / trajectory parameters
  uint64_t s;
  double next() { s = mix64(s); return unit(s); }
  double uni(double a, double b) { return a + (b - a) * next(); }
};

struct V3 { double x, y, z; };
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V3 unitv(V3 a) { double l = sqrt(dot(a, a)); return a * (1.0 / l); }

void add_plane(of_synth_scene_t *s, double nx, double ny, double nz, double d) {
  of_synth_prim_t &p = s->prims[s->count++];
  memset(&p, 0, sizeof(p));
  p.kind = OF_PRIM_PLANE;
  p.p[0] = (float)nx; p.p[1] = (float)ny; p.p[2] = (float)nz; p.p[3] = (float)d;
}

// Camera-to-world look-at in the reference convention (camera looks along -z).
void look_at(V3 eye, V3 tgt, double *P) {
  V3 f = unitv(tgt - eye);
  V3 z = f * -1.0;
  V3 up = {0.0, 1.0, 0.0};
  V3 x = unitv(cross(up, z));
  V3 y = cross(z, x);
  double M[16] = {x.x, y.x, z.x, eye.x, x.y, y.y, z.y, eye.y, x.z, y.z, z.z, eye.z, 0, 0, 0, 1};
  memcpy(P, M, sizeof(M));
}

void rot_axis_angle(V3 a, double ang, double R[9]) {
  double c = cos(ang), s = sin(ang), C = 1.0 - c;
  R[0] = c + a.x * a.x * C;       R[1] = a.x * a.y * C - a.z * s; R[2] = a.x * a.z * C + a.y * s;
  R[3] = a.y * a.x * C + a.z * s; R[4] = c + a.y * a.y * C;       R[5] = a.y * a.z * C - a.x * s;
  R[6] = a.z * a.x * C - a.y * s; R[7] = a.z * a.y * C + a.x * s; R[8] = c + a.z * a.z * C;
}

V3 random_dir(Rng &r) {
  double z = r.uni(-1.0, 1.0), ph = r.uni(0.0, 2.0 * M_PI);
  double q = sqrt(1.0 - z * z);
  return {q * cos(ph), q * sin(ph), z};
}

double hit_prim(const of_synth_prim_t &p, V3 o, V3 d) {
  const double eps = 1e-6;
  if (p.kind == OF_PRIM_PLANE) {
    V3 n = {p.p[0], p.p[1], p.p[2]};
    double den = dot(n, d);
    if (fabs(den) < 1e-12) return -1.0;
    double t = (p.p[3] - dot(n, o)) / den;
    return t > eps ? t : -1.0;
  }
  if (p.kind == OF_PRIM_SPHERE) {
    V3 c = {p.p[0], p.p[1], p.p[2]};
    double r = p.p[3];
    V3 oc = o - c;
    double a = dot(d, d), b = dot(oc, d), cc = dot(oc, oc) - r * r;
    double disc = b * b - a * cc;
    if (disc < 0.0) return -1.0;
    double sq = sqrt(disc);
    double t = (-b - sq) / a;
    if (t > eps) return t;
    t = (-b + sq) / a;
    return t > eps ? t : -1.0;
  }
  // box with yaw about +y
  V3 c = {p.p[0], p.p[1], p.p[2]};
  double h[3] = {p.p[3], p.p[4], p.p[5]};
  double cy = cos(p.p[6]), sy = sin(p.p[6]);
  V3 ol = o - c;
  double lo[3] = {cy * ol.x - sy * ol.z, ol.y, sy * ol.x + cy * ol.z};
  double ld[3] = {cy * d.x - sy * d.z, d.y, sy * d.x + cy * d.z};
  double tn = -1e300, tf = 1e300;
  for (int a = 0; a < 3; ++a) {
    if (fabs(ld[a]) < 1e-15) {
      if (lo[a] < -h[a] || lo[a] > h[a]) return -1.0;
      continue;
    }
    double t0 = (-h[a] - lo[a]) / ld[a], t1 = (h[a] - lo[a]) / ld[a];
    if (t0 > t1) { double q = t0; t0 = t1; t1 = q; }
    if (t0 > tn) tn = t0;
    if (t1 < tf) tf = t1;
  }
  if (tn > tf) return -1.0;
  if (tn > eps) return tn;
  return tf > eps ? tf : -1.0;
}

}  // namespace

extern "C" int32_t of_synth_scene(int32_t kind, uint64_t seed, float cube_mm,
                                  of_synth_scene_t *out) {
  if (!out || cube_mm <= 0.f || kind < 0 || kind > 1) return 1;
  memset(out, 0, sizeof(*out));
  const double S = cube_mm;
  out->room_half_mm = (float)(0.45 * S);
  Rng r{mix64(seed * 0x9E3779B97F4A7C15ull + 17)};
  double floor_y = -0.37 * S;
  add_plane(out, 0, 1, 0, floor_y);        // floor
  add_plane(out, 0, 0, 1, -0.45 * S);      // back wall
  add_plane(out, 1, 0, 0, -0.45 * S);      // left wall
  add_plane(out, 1, 0, 0, 0.45 * S);       // right wall
  int objects = kind == 0 ? 6 : 20;
  for (int i = 0; i < objects; ++i) {
    of_synth_prim_t &p = out->prims[out->count++];
    memset(&p, 0, sizeof(p));
    bool sphere = kind == 0 ? true : (r.next() < 0.5);
    if (sphere) {
      double rad = r.uni(100.0, 400.0);
      p.kind = OF_PRIM_SPHERE;
      p.p[0] = (float)r.uni(-0.33 * S, 0.33 * S);
      p.p[1] = (float)r.uni(floor_y + rad, 0.12 * S);
      p.p[2] = (float)r.uni(-0.42 * S + rad, 0.02 * S);
      p.p[3] = (float)rad;
    } else {
      double hx = r.uni(80.0, 300.0), hy = r.uni(80.0, 300.0), hz = r.uni(80.0, 300.0);
      p.kind = OF_PRIM_BOX;
      p.p[0] = (float)r.uni(-0.33 * S, 0.33 * S);
      p.p[1] = (float)r.uni(floor_y + hy, 0.12 * S);
      p.p[2] = (float)r.uni(-0.42 * S + hz, 0.02 * S);
      p.p[3] = (float)hx; p.p[4] = (float)hy; p.p[5] = (float)hz;
      p.p[6] = (float)r.uni(0.0, 0.5 * M_PI);
    }
  }
  return 0;
}

extern "C" int32_t of_synth_trajectory(int32_t motion, uint64_t seed, float cube_mm,
                                       int32_t frames, double *poses) {
  if (!poses || frames < 0 || cube_mm <= 0.f || motion < 0 || motion > 1) return 1;
  const double S = cube_mm;
  Rng r{mix64(seed * 0xD1B54A32D192ED03ull + 5)};
  V3 tgt = {r.uni(-0.02, 0.02) * S, -0.05 * S + r.uni(-0.02, 0.02) * S, -0.12 * S + r.uni(-0.02, 0.02) * S};
  const double rad = 0.43 * S, h0 = 0.05 * S, bob = 0.02 * S;
  const double A = 18.0 * M_PI / 180.0, P = 300.0;
  const double ph1 = r.uni(0.0, 2.0 * M_PI), ph2 = r.uni(0.0, 2.0 * M_PI);
  const double th0 = r.uni(-0.1, 0.1);
  for (int k = 0; k < frames; ++k) {
    double th = th0 + A * sin(2.0 * M_PI * k / P + ph1) - A * sin(ph1);
    double hy = h0 + bob * sin(4.0 * M_PI * k / P + ph2);
    V3 eye = {tgt.x + rad * sin(th), tgt.y + hy, tgt.z + rad * cos(th)};
    double *T = poses + 16 * (size_t)k;
    look_at(eye, tgt, T);
    if (motion == 1) {
      Rng q{hash3(seed, 0x51ed270b27ull, (uint64_t)k)};
      double R[9];
      rot_axis_angle(random_dir(q), q.uni(0.0, 2.5) * M_PI / 180.0, R);
      V3 td = random_dir(q) * q.uni(0.0, 50.0);
      double O[16];
      memcpy(O, T, sizeof(O));
      // T <- T * [R | td] (perturbation in the camera frame)
      for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j)
          T[4 * i + j] = O[4 * i] * R[j] + O[4 * i + 1] * R[3 + j] + O[4 * i + 2] * R[6 + j];
        T[4 * i + 3] = O[4 * i] * td.x + O[4 * i + 1] * td.y + O[4 * i + 2] * td.z + O[4 * i + 3];
      }
    }
  }
  return 0;
}

extern "C" int32_t of_synth_render(const of_synth_scene_t *scene, int32_t w, int32_t h, float fx,
                                   float fy, float cx, float cy, const double *P,
                                   uint64_t noise_seed, int32_t frame, float sigma_scale,
                                   float dropout, uint16_t *depth, float *exact) {
  if (!scene || !P || !depth || w <= 0 || h <= 0) return 1;
  V3 o = {P[3], P[7], P[11]};
#pragma omp parallel for schedule(static)
  for (int v = 0; v < h; ++v) {
    for (int u = 0; u < w; ++u) {
      V3 dc = {-((double)u - cx) / fx, -((double)v - cy) / fy, -1.0};
      V3 d = {P[0] * dc.x + P[1] * dc.y + P[2] * dc.z, P[4] * dc.x + P[5] * dc.y + P[6] * dc.z,
              P[8] * dc.x + P[9] * dc.y + P[10] * dc.z};
      double best = -1.0;
      for (int i = 0; i < scene->count; ++i) {
        double t = hit_prim(scene->prims[i], o, d);
        if (t > 0.0 && (best < 0.0 || t < best)) best = t;
      }
      size_t p = (size_t)v * w + u;
      if (exact) exact[p] = best > 0.0 ? (float)best : 0.f;
      uint16_t out = 0;
      if (best > 0.0 && best < 10000.0) {
        uint64_t hh = hash3(noise_seed, (uint64_t)frame, (uint64_t)p);
        double u1 = unit(mix64(hh ^ 1)), u2 = unit(mix64(hh ^ 2)), u3 = unit(mix64(hh ^ 3));
        double zm = best * 1e-3 - 0.4;
        double sigma = 1000.0 * (0.0012 + 0.0019 * zm * zm) * sigma_scale;
        double g = sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
        double dn = floor(best + sigma * g + 0.5);
        if (dn < 1.0) dn = 1.0;
        if (dn > 65535.0) dn = 65535.0;
        out = (u3 < dropout) ? 0 : (uint16_t)dn;
      }
      depth[p] = out;
    }
  }
  return 0;
}
