// wf_host.cpp -- host-side setup math of the wavefront engine, restated in
// C++ so that callers of the C ABI get the reference's exact tables:
// Q16.16 coefficients (src/layout.rs:105-216), CPML profiles
// (src/layout.rs:471-533), waveforms (src/source.rs:46-59), DFT probe
// tables and spectrum (src/probe.rs:126-167), and the scene voxelizer
// (src/scene.rs:81-230, src/main.rs:403-425).
//
// Everything here is plain f32/f64 IEEE arithmetic in the reference's
// operation order, compiled without FMA contraction (-ffp-contract=off), and
// uses the C library's expf/logf/powf/sinf/cos/sin, which is what the
// reference's f32/f64 methods call on Linux.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/wavefront_gpu.h"
#include "wf_scene.h"

namespace {

constexpr float kEps0 = 8.854188e-12f;  // src/layout.rs:29
constexpr float kMu0 = 1.2566371e-6f;   // src/layout.rs:31
constexpr float kPiF = 3.14159265358979323846f;
constexpr double kPiD = 3.14159265358979323846;

void sphere_fill(uint8_t *grid, int nx, int ny, int nz, float cx, float cy,
                 float cz, float radius, uint8_t id) {
  const float r2 = radius * radius;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        // cell-centre test x + 0.5 - cx, src/scene.rs:198-204
        const float dx = static_cast<float>(x) + 0.5f - cx;
        const float dy = static_cast<float>(y) + 0.5f - cy;
        const float dz = static_cast<float>(z) + 0.5f - cz;
        if (dx * dx + dy * dy + dz * dz <= r2)
          grid[(static_cast<size_t>(z) * ny + y) * nx + x] = id;
      }
}

// Rust `f32 as usize` saturates (NaN -> 0).
size_t sat_usize(float v) {
  if (!(v > 0.0f)) return 0;
  if (v >= 1.8e19f) return SIZE_MAX;
  return static_cast<size_t>(v);
}

bool parse_number(const std::string &tok, float *out) {
  if (tok.find_first_of("xX") != std::string::npos) return false;
  char *end = nullptr;
  const float v = std::strtof(tok.c_str(), &end);
  if (end == tok.c_str() || *end != '\0') return false;
  *out = v;
  return true;
}

struct Primitive {
  bool sphere;
  float v[9];
};

}  // namespace

extern "C" {

int32_t wf_q16_from_f32(float v) {
  const float r = std::round(v * 65536.0f);
  if (std::isnan(r)) return 0;
  if (r >= 2147483647.0f) return INT32_MAX;
  if (r <= -2147483648.0f) return INT32_MIN;
  return static_cast<int32_t>(r);
}

float wf_q16_to_f32(int32_t q) { return static_cast<float>(q) * (1.0f / 65536.0f); }

void wf_material_coeffs(float eps_r, float mu_r, float sigma, float dt, float d,
                        int32_t out[4]) {
  const float eps = eps_r * kEps0;
  const float mu = mu_r * kMu0;
  const float loss = sigma * dt / (2.0f * eps);
  out[0] = wf_q16_from_f32((1.0f - loss) / (1.0f + loss));
  out[1] = wf_q16_from_f32((dt / (eps * d)) / (1.0f + loss));
  out[2] = wf_q16_from_f32(1.0f);
  out[3] = wf_q16_from_f32(dt / (mu * d));
}

int wf_effective_pml_thickness_blocks(int nx, int ny, int nz, int requested) {
  if (requested == 0) return 0;
  int req_blocks = (requested + 7) / 8;
  if (req_blocks < 1) req_blocks = 1;
  int max_blocks = std::min(nx / 8, std::min(ny / 8, nz / 8)) / 2;
  if (max_blocks < 1) max_blocks = 1;
  return std::min(req_blocks, max_blocks);
}

void wf_pml_profile(int n, float grading_order, float kappa_max, float alpha_max,
                    float target_reflection, float dt, float dx, int thickness,
                    float *b, float *a, float *inv_kappa) {
  for (int i = 0; i < n; ++i) {  // PmlCoeffs::IDENTITY everywhere first
    b[i] = 1.0f;
    a[i] = 0.0f;
    inv_kappa[i] = 1.0f;
  }
  if (thickness == 0) return;
  const float depth = static_cast<float>(thickness) * dx;
  const float eta0 = std::sqrt(kMu0 / kEps0);
  const float sigma_max =
      -(grading_order + 1.0f) * std::log(target_reflection) / (2.0f * eta0 * depth);
  for (int g = 0; g < thickness; ++g) {
    const float rho = static_cast<float>(thickness - g) / static_cast<float>(thickness);
    const float sigma = sigma_max * std::pow(rho, grading_order);
    const float kappa = 1.0f + (kappa_max - 1.0f) * std::pow(rho, grading_order);
    const float alpha = alpha_max * (1.0f - rho);
    const float bb = std::exp(-(sigma / kappa + alpha) * dt / kEps0);
    const float denom = kappa * (sigma + kappa * alpha);
    const float aa = std::fabs(denom) > 1.0e-30f ? sigma * (bb - 1.0f) / denom : 0.0f;
    const float ik = 1.0f / kappa;
    // low face first, then the mirrored high face (a later write wins when
    // the two faces overlap on a one-block axis)
    b[g] = bb; a[g] = aa; inv_kappa[g] = ik;
    b[n - 1 - g] = bb; a[n - 1 - g] = aa; inv_kappa[n - 1 - g] = ik;
  }
}

float wf_waveform_eval(int kind, float p0, float p1, float t) {
  switch (kind) {
    case 0: {
      const float arg = (t - p0) / p1;
      return std::exp(-0.5f * arg * arg);
    }
    case 1:
      return std::sin(2.0f * kPiF * p0 * t);
    case 2: {
      const float arg = kPiF * p0 * (t - p1);
      const float arg_sq = arg * arg;
      return (1.0f - 2.0f * arg_sq) * std::exp(-arg_sq);
    }
    default:
      return 0.0f;
  }
}

void wf_source_values(int kind, float p0, float p1, float amplitude, float dt,
                      int first_step, int nsteps, float *values) {
  for (int i = 0; i < nsteps; ++i) {
    // t = (step as f32 + 1.0) * dt, src/engine.rs:769
    const float t = (static_cast<float>(first_step + i) + 1.0f) * dt;
    values[i] = amplitude * wf_waveform_eval(kind, p0, p1, t);
  }
}

int wf_probe_first_step(float start, float dt) {
  // smallest s with !((s+1)*dt < start); t is non-decreasing in s
  int s = 0;
  if (start > 0.0f) {
    double guess = static_cast<double>(start) / static_cast<double>(dt) - 2.0;
    if (guess > 0.0 && guess < 2.0e9) s = static_cast<int>(guess);
    while (s > 0 && !((static_cast<float>(s - 1) + 1.0f) * dt < start)) --s;
    while ((static_cast<float>(s) + 1.0f) * dt < start) ++s;
  }
  return s;
}

void wf_probe_tables(const float *freqs, int nfreq, float dt, int first_step,
                     int nsteps, double *cos_tab, double *sin_tab) {
  for (int i = 0; i < nsteps; ++i) {
    const float t = (static_cast<float>(first_step + i) + 1.0f) * dt;
    for (int f = 0; f < nfreq; ++f) {
      const double omega = 2.0 * kPiD * static_cast<double>(freqs[f]);
      const double phase = omega * static_cast<double>(t);
      cos_tab[static_cast<size_t>(i) * nfreq + f] = std::cos(phase);
      sin_tab[static_cast<size_t>(i) * nfreq + f] = std::sin(phase);
    }
  }
}

void wf_spectrum(const double *sum_cos, const double *sum_sin, uint64_t n,
                 int nfreq, double *amplitude, double *phase_rad) {
  const double nn = static_cast<double>(n > 0 ? n : 1);
  for (int f = 0; f < nfreq; ++f) {
    const double a = 2.0 * sum_cos[f] / nn;
    const double b = 2.0 * sum_sin[f] / nn;
    amplitude[f] = std::sqrt(a * a + b * b);
    phase_rad[f] = std::atan2(a, b);
  }
}

wf_status wf_scene_voxelize(const char *text, int nx, int ny, int nz, float dt,
                            float dx, uint8_t *grid, int32_t (*table)[4],
                            int *n_materials, char *err, int errlen) {
  std::vector<wf::RasterOp> ops;
  std::string msg;
  if (!grid || !wf::scene_parse(text, nx, ny, nz, dt, dx, &ops, table, n_materials, &msg)) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", grid ? msg.c_str() : "null argument");
    return WF_ERR_ARG;
  }
  for (const wf::RasterOp &op : ops) {
    if (op.sphere) {
      for (long long z = op.z0; z < op.z1; ++z)
        for (long long y = op.y0; y < op.y1; ++y)
          for (long long x = op.x0; x < op.x1; ++x) {
            // cell-centre test x + 0.5 - cx, src/scene.rs:198-204
            const float ddx = static_cast<float>(x) + 0.5f - op.cx;
            const float ddy = static_cast<float>(y) + 0.5f - op.cy;
            const float ddz = static_cast<float>(z) + 0.5f - op.cz;
            if (ddx * ddx + ddy * ddy + ddz * ddz <= op.r2)
              grid[(static_cast<size_t>(z) * ny + y) * nx + x] = op.id;
          }
    } else {
      for (long long z = op.z0; z < op.z1; ++z)
        for (long long y = op.y0; y < op.y1; ++y)
          for (long long x = op.x0; x < op.x1; ++x)
            grid[(static_cast<size_t>(z) * ny + y) * nx + x] = op.id;
    }
  }
  return WF_OK;
}

void wf_demo_sphere(int nx, int ny, int nz, uint8_t *grid) {
  const float r = static_cast<float>(std::min(nx, std::min(ny, nz))) / 4.0f;
  sphere_fill(grid, nx, ny, nz, static_cast<float>(nx) / 2.0f, static_cast<float>(ny) / 2.0f,
              static_cast<float>(nz) / 2.0f, r, 1);
}

}  // extern "C"

namespace wf {

namespace {

// Integer cell range [lo, hi) that contains every cell centre within r of c
// on one axis (a margin of 2 cells covers the f32 rounding of the test);
// the whole axis when c or r is not finite.
void sphere_range(float c, float r, int n, long long *lo, long long *hi) {
  if (!std::isfinite(c) || !std::isfinite(r)) {
    *lo = 0;
    *hi = n;
    return;
  }
  const double a = std::floor(static_cast<double>(c) - std::fabs(static_cast<double>(r))) - 2.0;
  const double b = std::ceil(static_cast<double>(c) + std::fabs(static_cast<double>(r))) + 2.0;
  *lo = static_cast<long long>(std::max(0.0, std::min(a, static_cast<double>(n))));
  *hi = static_cast<long long>(std::max(0.0, std::min(b, static_cast<double>(n))));
}

}  // namespace

bool scene_parse(const char *text, int nx, int ny, int nz, float dt, float dx,
                 std::vector<RasterOp> *ops, int32_t (*table)[4], int *n_materials,
                 std::string *err) {
  auto fail = [&](const std::string &msg) {
    *err = msg;
    return false;
  };
  if (!text || !table) return fail("null argument");
  // Scene::parse, src/scene.rs:81-143: every line first, then voxelize.
  std::vector<Primitive> prims;
  const std::string all(text);
  size_t pos = 0;
  int line_no = 0;
  while (pos <= all.size()) {
    size_t nl = all.find('\n', pos);
    std::string line = all.substr(pos, nl == std::string::npos ? std::string::npos : nl - pos);
    ++line_no;
    const char *ws = " \t\r\n\v\f";
    const size_t b = line.find_first_not_of(ws);
    if (b != std::string::npos) {
      line = line.substr(b, line.find_last_not_of(ws) - b + 1);
      if (line[0] != '#') {
        std::vector<std::string> toks;
        size_t p = 0;
        while (p < line.size()) {
          const size_t s0 = line.find_first_not_of(ws, p);
          if (s0 == std::string::npos) break;
          const size_t e = line.find_first_of(ws, s0);
          toks.push_back(line.substr(s0, e == std::string::npos ? std::string::npos : e - s0));
          p = e == std::string::npos ? line.size() : e;
        }
        const bool sphere = toks[0] == "sphere", box = toks[0] == "box";
        if (!sphere && !box)
          return fail("scene line " + std::to_string(line_no) + ": unknown primitive '" + toks[0] + "'");
        std::vector<float> v;
        for (size_t i = 1; i < toks.size(); ++i) {
          float f;
          if (!parse_number(toks[i], &f))
            return fail("scene line " + std::to_string(line_no) + ": invalid number '" + toks[i] + "'");
          v.push_back(f);
        }
        if (sphere && v.size() != 7)
          return fail("scene line " + std::to_string(line_no) +
                      ": expected 'sphere eps_r mu_r sigma cx cy cz radius', got " +
                      std::to_string(v.size()) + " values");
        if (box && v.size() != 9)
          return fail("scene line " + std::to_string(line_no) +
                      ": expected 'box eps_r mu_r sigma x0 y0 z0 x1 y1 z1', got " +
                      std::to_string(v.size()) + " values");
        Primitive pr{};
        pr.sphere = sphere;
        for (size_t i = 0; i < v.size(); ++i) pr.v[i] = v[i];
        prims.push_back(pr);
      }
    }
    if (nl == std::string::npos) break;
    pos = nl + 1;
  }
  // Scene::voxelize, src/scene.rs:149-188: ids de-duplicated by bit pattern.
  std::vector<std::array<uint32_t, 3>> keys;
  ops->clear();
  for (const Primitive &pr : prims) {
    std::array<uint32_t, 3> key;
    std::memcpy(key.data(), pr.v, 12);
    int id = -1;
    for (size_t i = 0; i < keys.size(); ++i)
      if (keys[i] == key) id = static_cast<int>(i) + 1;
    if (id < 0) {
      if (keys.size() + 1 > 255) return fail("scene uses more than 255 distinct materials");
      keys.push_back(key);
      id = static_cast<int>(keys.size());
      wf_material_coeffs(pr.v[0], pr.v[1], pr.v[2], dt, dx, table[id]);
    }
    RasterOp op{};
    op.id = static_cast<uint8_t>(id);
    if (pr.sphere) {
      op.sphere = 1;
      op.cx = pr.v[3];
      op.cy = pr.v[4];
      op.cz = pr.v[5];
      op.r2 = pr.v[6] * pr.v[6];
      sphere_range(op.cx, pr.v[6], nx, &op.x0, &op.x1);
      sphere_range(op.cy, pr.v[6], ny, &op.y0, &op.y1);
      sphere_range(op.cz, pr.v[6], nz, &op.z0, &op.z1);
    } else {
      // src/scene.rs:212-226: floor/ceil clamps
      auto lo = [](float v) { return sat_usize(std::floor(std::fmax(v, 0.0f))); };
      auto hi = [](float v, int n) {
        return std::min(sat_usize(std::fmax(std::ceil(v), 0.0f)), static_cast<size_t>(n));
      };
      auto clamp = [](size_t v, int n) { return static_cast<long long>(std::min(v, static_cast<size_t>(n))); };
      op.x0 = clamp(lo(std::fmin(pr.v[3], pr.v[6])), nx);
      op.x1 = static_cast<long long>(hi(std::fmax(pr.v[3], pr.v[6]), nx));
      op.y0 = clamp(lo(std::fmin(pr.v[4], pr.v[7])), ny);
      op.y1 = static_cast<long long>(hi(std::fmax(pr.v[4], pr.v[7]), ny));
      op.z0 = clamp(lo(std::fmin(pr.v[5], pr.v[8])), nz);
      op.z1 = static_cast<long long>(hi(std::fmax(pr.v[5], pr.v[8]), nz));
    }
    ops->push_back(op);
  }
  if (n_materials) *n_materials = static_cast<int>(keys.size());
  return true;
}

}  // namespace wf
