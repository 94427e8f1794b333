// Synthetic capacity volumes for the grid graph-cut workloads.
//
// The reference builds its grid graph on the host from an image and marker
// volume (benchmarks/graph_cut/graph_cut.cpp:33-98: t-links per voxel, one
// n-link per 6-neighbour pair with weight exp(-(Ii-Ij)^2 ...)).  No image data
// ships with the reference, so the workloads here are seeded synthetic
// volumes with the same structure: objects of one intensity on a background,
// Gaussian noise, likelihood t-links and contrast n-links.  Everything is
// computed in double and rounded once (round half away from zero), so the
// int32 capacities are bit-identical on every machine with the same libm.
//
// RNG: std::mt19937_64 (its output sequence is fixed by the C++ standard);
// uniform doubles from the top 53 bits; normals by the Box-Muller transform.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>
#include <algorithm>

#include <string>

#include "cgc_volume.h"

namespace {

thread_local std::string g_volume_error;

int fail(int code, const char* msg) {
  g_volume_error = msg;
  return code;
}

struct Rng {
  std::mt19937_64 eng;
  bool has_spare = false;
  double spare = 0.0;
  explicit Rng(uint64_t seed) : eng(seed) {}
  double uniform() { return double(eng() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
  double uniform(double a, double b) { return a + (b - a) * uniform(); }
  int32_t uniform_int(int32_t lo, int32_t hi) {  // inclusive
    int64_t span = int64_t(hi) - lo + 1;
    int64_t k = int64_t(uniform() * double(span));
    if (k >= span) k = span - 1;
    return int32_t(lo + k);
  }
  double normal() {
    if (has_spare) { has_spare = false; return spare; }
    double u1 = 1.0 - uniform();  // (0,1]
    double u2 = uniform();
    double rad = std::sqrt(-2.0 * std::log(u1));
    double ang = 2.0 * M_PI * u2;
    spare = rad * std::sin(ang);
    has_spare = true;
    return rad * std::cos(ang);
  }
};

inline int64_t lin(int64_t x, int64_t y, int64_t z, int64_t X, int64_t Y) { return x + X * (y + Y * z); }

void paint_ball(std::vector<float>& img, const cgc_volume_spec& s, double cx, double cy, double cz,
                double r, float value) {
  int64_t x0 = std::max<int64_t>(0, (int64_t)std::floor(cx - r)), x1 = std::min<int64_t>(s.X - 1, (int64_t)std::ceil(cx + r));
  int64_t y0 = std::max<int64_t>(0, (int64_t)std::floor(cy - r)), y1 = std::min<int64_t>(s.Y - 1, (int64_t)std::ceil(cy + r));
  int64_t z0 = std::max<int64_t>(0, (int64_t)std::floor(cz - r)), z1 = std::min<int64_t>(s.Z - 1, (int64_t)std::ceil(cz + r));
  double r2 = r * r;
  for (int64_t z = z0; z <= z1; ++z)
    for (int64_t y = y0; y <= y1; ++y)
      for (int64_t x = x0; x <= x1; ++x) {
        double dx = x - cx, dy = y - cy, dz = z - cz;
        if (dx * dx + dy * dy + dz * dz <= r2) img[lin(x, y, z, s.X, s.Y)] = value;
      }
}

// Ball of radius r with a Gaussian-blurred boundary: weight
// w(d) = erfc((d - r) / (sqrt(2) sigma)) / 2; overlapping objects keep the
// largest contrast.
void paint_soft_ball(std::vector<float>& img, const cgc_volume_spec& s, double cx, double cy, double cz,
                     double r, double sigma, double contrast) {
  const double R = r + 5.0 * sigma;
  int64_t x0 = std::max<int64_t>(0, (int64_t)std::floor(cx - R)), x1 = std::min<int64_t>(s.X - 1, (int64_t)std::ceil(cx + R));
  int64_t y0 = std::max<int64_t>(0, (int64_t)std::floor(cy - R)), y1 = std::min<int64_t>(s.Y - 1, (int64_t)std::ceil(cy + R));
  int64_t z0 = std::max<int64_t>(0, (int64_t)std::floor(cz - R)), z1 = std::min<int64_t>(s.Z - 1, (int64_t)std::ceil(cz + R));
  const double k = 1.0 / (std::sqrt(2.0) * sigma);
#pragma omp parallel for schedule(static) if ((z1 - z0 + 1) * (y1 - y0 + 1) * (x1 - x0 + 1) > 65536)
  for (int64_t z = z0; z <= z1; ++z)
    for (int64_t y = y0; y <= y1; ++y)
      for (int64_t x = x0; x <= x1; ++x) {
        double dx = x - cx, dy = y - cy, dz = z - cz;
        double d = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (d > R) continue;
        double v = s.background + contrast * 0.5 * std::erfc((d - r) * k);
        float& cur = img[lin(x, y, z, s.X, s.Y)];
        if (std::fabs(v - s.background) > std::fabs(double(cur) - s.background)) cur = float(v);
      }
}

double centre(Rng& rng, double r, int32_t ext) {
  double lo = r, hi = double(ext - 1) - r;
  if (hi < lo) return 0.5 * double(ext - 1);
  return rng.uniform(lo, hi);
}

void draw_spheres(std::vector<float>& img, const cgc_volume_spec& s, Rng& rng) {
  for (int32_t k = 0; k < s.count; ++k) {
    double r = (s.n_fixed_radii > 0) ? s.fixed_radii[std::min(k, s.n_fixed_radii - 1)]
                                     : rng.uniform(s.radius_min, s.radius_max);
    double cx = centre(rng, r, s.X), cy = centre(rng, r, s.Y), cz = centre(rng, r, s.Z);
    double inten = (s.intensity_max > s.intensity_min) ? rng.uniform(s.intensity_min, s.intensity_max)
                                                       : s.intensity_min;
    if (s.edge_sigma > 0) paint_soft_ball(img, s, cx, cy, cz, r, s.edge_sigma, inten - s.background);
    else paint_ball(img, s, cx, cy, cz, r, float(inten));
  }
}

// Uniform Catmull-Rom spline through the control points (end points
// duplicated), sampled at steps of at most half a voxel; every voxel within
// the radius of a sample is painted.
void draw_tubes(std::vector<float>& img, const cgc_volume_spec& s, Rng& rng) {
  for (int32_t k = 0; k < s.count; ++k) {
    int32_t n = rng.uniform_int(s.ctrl_min, s.ctrl_max);
    std::vector<double> P(3 * n);
    for (int32_t i = 0; i < n; ++i) {
      P[3 * i + 0] = rng.uniform(0.0, double(s.X - 1));
      P[3 * i + 1] = rng.uniform(0.0, double(s.Y - 1));
      P[3 * i + 2] = rng.uniform(0.0, double(s.Z - 1));
    }
    double r = rng.uniform(s.radius_min, s.radius_max);
    float inten = float((s.intensity_max > s.intensity_min) ? rng.uniform(s.intensity_min, s.intensity_max)
                                                            : s.intensity_min);
    for (int32_t i = 0; i + 1 < n; ++i) {
      const double* p0 = &P[3 * std::max(i - 1, 0)];
      const double* p1 = &P[3 * i];
      const double* p2 = &P[3 * (i + 1)];
      const double* p3 = &P[3 * std::min(i + 2, n - 1)];
      double len = std::sqrt((p2[0] - p1[0]) * (p2[0] - p1[0]) + (p2[1] - p1[1]) * (p2[1] - p1[1]) +
                             (p2[2] - p1[2]) * (p2[2] - p1[2]));
      int64_t steps = std::max<int64_t>(1, (int64_t)std::ceil(len / 0.5));
      for (int64_t st = 0; st <= steps; ++st) {
        double t = double(st) / double(steps), t2 = t * t, t3 = t2 * t;
        double c[3];
        for (int a = 0; a < 3; ++a)
          c[a] = 0.5 * (2.0 * p1[a] + (-p0[a] + p2[a]) * t + (2.0 * p0[a] - 5.0 * p1[a] + 4.0 * p2[a] - p3[a]) * t2 +
                        (-p0[a] + 3.0 * p1[a] - 3.0 * p2[a] + p3[a]) * t3);
        paint_ball(img, s, c[0], c[1], c[2], r, inten);
      }
    }
  }
}

inline int32_t round_cap(double v) {
  double r = std::round(v);
  if (r < 0) r = 0;
  if (r > 2147483647.0) r = 2147483647.0;
  return int32_t(r);
}

}  // namespace

extern "C" const char* cgc_volume_last_error(void) { return g_volume_error.c_str(); }

extern "C" int cgc_volume_preset(int which, int32_t index, cgc_volume_spec* out) {
  if (!out) return fail(CGC_ERR_ARG, "cgc_volume_preset: null output");
  cgc_volume_spec s;
  std::memset(&s, 0, sizeof(s));
  s.kind = 0;
  s.background = 0.2; s.mu_bg = 0.2; s.mu_fg = 0.8; s.class_sd = 0.1;
  s.tlink_scale = 10.0; s.nlink_scale = 50.0; s.nlink_sigma = 0.1;
  s.intensity_min = s.intensity_max = 0.8;
  s.edge_sigma = 1.5;  // "Gaussian spheres": boundary blurred over ~1.5 voxels
  switch (which) {
    case 1:  // 64^3, two spheres r = 12, 16, noise 0.05
      s.X = s.Y = s.Z = 64; s.seed = 1; s.count = 2; s.n_fixed_radii = 2;
      s.fixed_radii[0] = 12; s.fixed_radii[1] = 16; s.noise_sd = 0.05;
      break;
    case 2:  // 256^3, 40 spheres r in [8,40], intensity in [0.5,0.9], noise 0.08
      s.X = s.Y = s.Z = 256; s.seed = 2; s.count = 40; s.radius_min = 8; s.radius_max = 40;
      s.intensity_min = 0.5; s.intensity_max = 0.9; s.noise_sd = 0.08;
      break;
    case 3:  // 512x512x128, 200 tubes r in [2,6], intensity 0.7 on 0.3, noise 0.1
      s.X = 512; s.Y = 512; s.Z = 128; s.kind = 1; s.seed = 3; s.count = 200; s.edge_sigma = 0;
      s.radius_min = 2; s.radius_max = 6; s.intensity_min = s.intensity_max = 0.7;
      s.background = 0.3; s.mu_bg = 0.3; s.mu_fg = 0.7; s.noise_sd = 0.1; s.ctrl_min = 4; s.ctrl_max = 6;
      break;
    case 4: {  // batched instance: extents U[32,160], 4..20 spheres r in [4, min/4]
      if (index < 0) return fail(CGC_ERR_ARG, "cgc_volume_preset: negative index");
      s.seed = 1000 + uint64_t(index);
      Rng rng(s.seed ^ 0x9E3779B97F4A7C15ull);
      s.X = rng.uniform_int(32, 160); s.Y = rng.uniform_int(32, 160); s.Z = rng.uniform_int(32, 160);
      s.count = rng.uniform_int(4, 20);
      s.radius_min = 4; s.radius_max = double(std::min(s.X, std::min(s.Y, s.Z))) / 4.0;
      s.noise_sd = 0.05;
      break;
    }
    case 5:  // 128^3 training instance with the 64^3 generator's objects
      if (index < 0) return fail(CGC_ERR_ARG, "cgc_volume_preset: negative index");
      s.X = s.Y = s.Z = 128; s.seed = 10000 + uint64_t(index); s.count = 2; s.n_fixed_radii = 2;
      s.fixed_radii[0] = 12; s.fixed_radii[1] = 16; s.noise_sd = 0.05;
      break;
    default:
      return fail(CGC_ERR_ARG, "cgc_volume_preset: unknown workload");
  }
  *out = s;
  return CGC_OK;
}

extern "C" int cgc_volume_generate(const cgc_volume_spec* spec, int32_t* capS, int32_t* capT, int32_t* nx,
                                   int32_t* ny, int32_t* nz, float* image) {
  if (!spec || !capS || !capT || !nx || !ny || !nz) return fail(CGC_ERR_ARG, "cgc_volume_generate: null pointer");
  const cgc_volume_spec& s = *spec;
  if (s.X <= 0 || s.Y <= 0 || s.Z <= 0) return fail(CGC_ERR_ARG, "cgc_volume_generate: bad extent");
  if (s.kind == 1 && (s.ctrl_min < 2 || s.ctrl_max < s.ctrl_min)) return fail(CGC_ERR_ARG, "cgc_volume_generate: bad control point range");
  const int64_t X = s.X, Y = s.Y, Z = s.Z, N = X * Y * Z;
  std::vector<float> img;
  try { img.assign(size_t(N), float(s.background)); } catch (...) { return fail(CGC_ERR_OOM, "cgc_volume_generate: host allocation"); }
  Rng rng(s.seed);
  if (s.kind == 0) draw_spheres(img, s, rng); else draw_tubes(img, s, rng);
  // noise (one sequential stream, so the volume does not depend on the thread
  // count), then likelihood t-links and contrast n-links in parallel
  std::vector<double> I((size_t)N);
  for (int64_t v = 0; v < N; ++v) I[v] = double(img[v]) + s.noise_sd * rng.normal();
  const double inv2s2 = 1.0 / (2.0 * s.class_sd * s.class_sd);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < N; ++v) {
    const double val = I[v];
    if (image) image[v] = float(val);
    double a = ((val - s.mu_fg) * (val - s.mu_fg) - (val - s.mu_bg) * (val - s.mu_bg)) * inv2s2;
    double pfg = 1.0 / (1.0 + std::exp(a));
    pfg = std::min(std::max(pfg, 1e-6), 1.0);
    double pbg = std::min(std::max(1.0 - pfg, 1e-6), 1.0);
    capS[v] = round_cap(s.tlink_scale * -std::log(pbg));
    capT[v] = round_cap(s.tlink_scale * -std::log(pfg));
  }
  const double ninv = 1.0 / (2.0 * s.nlink_sigma * s.nlink_sigma);
#pragma omp parallel for schedule(static)
  for (int64_t z = 0; z < Z; ++z)
    for (int64_t y = 0; y < Y; ++y)
      for (int64_t x = 0; x < X; ++x) {
        int64_t v = lin(x, y, z, X, Y);
        double iv = I[v];
        nx[v] = (x + 1 < X) ? round_cap(s.nlink_scale * std::exp(-(iv - I[v + 1]) * (iv - I[v + 1]) * ninv)) : 0;
        ny[v] = (y + 1 < Y) ? round_cap(s.nlink_scale * std::exp(-(iv - I[v + X]) * (iv - I[v + X]) * ninv)) : 0;
        nz[v] = (z + 1 < Z) ? round_cap(s.nlink_scale * std::exp(-(iv - I[v + X * Y]) * (iv - I[v + X * Y]) * ninv)) : 0;
      }
  return CGC_OK;
}
