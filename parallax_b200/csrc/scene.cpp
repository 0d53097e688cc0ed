// scene.cpp -- seeded synthetic clouds and camera rigs for the benchmark
// workloads.
//
// The generator is the reference's test Rng: xorshift64 with uniform doubles
// from the top 53 bits and a Box-Muller normal
// (engine/native/cpp/include/parallax/testing/SyntheticScene.h:80-107).
// Cameras look at the origin with the reference's lookAt convention (+X right,
// +Y down, +Z forward; SyntheticScene.cpp:235-258) and phoneIntrinsics
// (SyntheticScene.cpp:129-138).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "densify.h"
#include "runtime.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

struct Rng {
  uint64_t state;
  explicit Rng(uint64_t seed) : state(seed ? seed : 1) {}
  uint64_t next() {
    state ^= state << 13;
    state ^= state >> 7;
    state ^= state << 17;
    return state;
  }
  double uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
  double uniform(double lo, double hi) { return lo + (hi - lo) * uniform(); }
  double normal() {
    const double u1 = std::max(1e-12, uniform());
    const double u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
  }
};

struct V3 {
  double x, y, z;
};
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double norm(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
V3 scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }

void look_at(V3 eye, V3 target, double R[9], double t[3]) {
  V3 forward = sub(target, eye);
  if (norm(forward) < 1e-9) forward = {0, 0, 1};
  forward = scale(forward, 1.0 / norm(forward));
  V3 up = {0, 1, 0};
  if (std::fabs(forward.y) > 0.999) up = std::fabs(forward.x) < 0.9 ? V3{1, 0, 0} : V3{0, 0, 1};
  V3 right = cross(forward, up);
  if (norm(right) < 1e-9) right = {1, 0, 0};
  right = scale(right, 1.0 / norm(right));
  const V3 down = cross(forward, right);
  const V3 rows[3] = {right, down, forward};
  for (int r = 0; r < 3; ++r) {
    R[r * 3 + 0] = rows[r].x;
    R[r * 3 + 1] = rows[r].y;
    R[r * 3 + 2] = rows[r].z;
  }
  for (int r = 0; r < 3; ++r)
    t[r] = -(R[r * 3 + 0] * eye.x + R[r * 3 + 1] * eye.y + R[r * 3 + 2] * eye.z);
}

}  // namespace

extern "C" {

int pxs_synthetic_cloud(uint64_t seed, int32_t count, int32_t rest_per_channel,
                        float log_scale_mean, float* params) {
  const int S = rest_per_channel;
  if (count < 0 || params == nullptr || (S != 0 && S != 3 && S != 8 && S != 15))
    return PXS_ERR_INVALID;
  Rng rng(seed);
  const size_t n = static_cast<size_t>(count);
  const double c0 = 0.28209479177387814;
  for (size_t g = 0; g < n; ++g) {
    for (int a = 0; a < 3; ++a) params[(PXS_C_POSITION + a) * n + g] = static_cast<float>(rng.uniform(-1.0, 1.0));
    for (int a = 0; a < 3; ++a)
      params[(PXS_C_LOG_SCALE + a) * n + g] = static_cast<float>(log_scale_mean + 0.5 * rng.normal());
    double q[4], qn = 0.0;
    for (int a = 0; a < 4; ++a) {
      q[a] = rng.normal();
      qn += q[a] * q[a];
    }
    qn = std::sqrt(qn);
    if (qn < 1e-9) {
      q[0] = 1.0;
      q[1] = q[2] = q[3] = 0.0;
      qn = 1.0;
    }
    for (int a = 0; a < 4; ++a) params[(PXS_C_ROTATION + a) * n + g] = static_cast<float>(q[a] / qn);
    params[PXS_C_OPACITY * n + g] = static_cast<float>(rng.normal());
    for (int c = 0; c < 3; ++c) {
      const double rgb = 0.5 + 0.1 * rng.normal();
      params[(PXS_C_DC + c) * n + g] = static_cast<float>((rgb - 0.5) / c0);
    }
    for (int k = 0; k < 3 * S; ++k)
      params[(PXS_C_SH_REST + k) * n + g] = static_cast<float>(0.1 * rng.normal());
  }
  return PXS_OK;
}

int pxs_synthetic_cameras(uint64_t seed, int32_t count, int32_t layout, double radius,
                          int32_t width, int32_t height, double fov_degrees, pxs_camera* out) {
  if (count < 0 || out == nullptr || width <= 0 || height <= 0 || fov_degrees <= 0.0)
    return PXS_ERR_INVALID;
  Rng rng(seed);
  const double fx = (width * 0.5) / std::tan(fov_degrees * kPi / 180.0 * 0.5);
  const double K[4] = {fx, fx, width * 0.5 - 0.5, height * 0.5 - 0.5};
  const double golden = kPi * (3.0 - std::sqrt(5.0));
  const double spin = rng.uniform(0.0, 2.0 * kPi);
  const int hemisphere = layout == 1 ? count / 2 : count;
  for (int i = 0; i < count; ++i) {
    V3 eye;
    if (i < hemisphere) {
      // Fibonacci points: the whole sphere (layout 0) or its upper half (layout 1)
      const double u = (i + 0.5) / hemisphere;
      const double y = layout == 1 ? u : 1.0 - 2.0 * u;
      const double r = std::sqrt(std::max(0.0, 1.0 - y * y));
      const double a = golden * i + spin;
      eye = {radius * r * std::cos(a), radius * y, radius * r * std::sin(a)};
    } else {
      // walk-around ring: jittered height +-0.2 and radius +-0.1
      const int j = i - hemisphere;
      const int ring = count - hemisphere;
      const double a = 2.0 * kPi * j / ring + rng.uniform(-0.05, 0.05);
      const double rr = radius + rng.uniform(-0.1, 0.1);
      const double h = rng.uniform(-0.2, 0.2);
      eye = {rr * std::cos(a), h, rr * std::sin(a)};
    }
    double R[9], t[3];
    look_at(eye, {0, 0, 0}, R, t);
    pxs_camera_from_pose(K, width, height, R, t, &out[i]);
  }
  return PXS_OK;
}

}  // extern "C"
