/*
 * wf_oracle.c -- CPU oracle for the wavefront FDTD hot path.
 * TEST INFRASTRUCTURE ONLY (see wf_oracle.h).  Build: oracle/Makefile
 * (-O3 -ffp-contract=off, never -ffast-math: the reference's Rust code never
 * contracts a*b+c into an FMA and keeps IEEE semantics, denormals included).
 *
 * Transcendentals use glibc expf/logf/powf/sinf/cosf/asinf/log10f and the
 * double cos/sin/atan2, which is what Rust's f32/f64 methods lower to on
 * Linux.
 */
#include "wf_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* src/layout.rs:29-31 */
static const float EPS0 = 8.854188e-12f;
static const float MU0 = 1.2566371e-6f;
static const float PI_F = 3.14159265358979323846f;
static const double PI_D = 3.14159265358979323846;
static const float C0 = 299792458.0f; /* SPEED_OF_LIGHT_M_PER_S of the examples */

/* ------------------------------------------------------------------------ */
/* setup math                                                                */
/* ------------------------------------------------------------------------ */

int32_t or_q16_from_f32(float v) {
  /* (v * FIXED_ONE as f32).round() as i32: round half away from zero, and
   * Rust's saturating float->int cast (NaN -> 0). */
  float r = roundf(v * 65536.0f);
  if (r != r) return 0;
  if (r >= 2147483647.0f) return 2147483647;
  if (r <= -2147483648.0f) return (int32_t)0x80000000u;
  return (int32_t)r;
}

float or_q16_to_f32(int32_t q) { return (float)q * (1.0f / 65536.0f); }

void or_material_coeffs(float eps_r, float mu_r, float sigma, float dt, float d,
                        int32_t out[4]) {
  float eps = eps_r * EPS0;
  float mu = mu_r * MU0;
  float loss = sigma * dt / (2.0f * eps);
  float ca = (1.0f - loss) / (1.0f + loss);
  float cb = (dt / (eps * d)) / (1.0f + loss);
  float da = 1.0f;
  float db = dt / (mu * d);
  out[0] = or_q16_from_f32(ca);
  out[1] = or_q16_from_f32(cb);
  out[2] = or_q16_from_f32(da);
  out[3] = or_q16_from_f32(db);
}

int or_effective_pml_thickness_blocks(int nx, int ny, int nz, int req) {
  if (req == 0) return 0;
  int bx = nx / 8, by = ny / 8, bz = nz / 8;
  int rb = (req + 7) / 8;
  if (rb < 1) rb = 1;
  int mn = bx < by ? bx : by;
  mn = mn < bz ? mn : bz;
  int mb = mn / 2;
  if (mb < 1) mb = 1;
  return rb < mb ? rb : mb;
}

void or_pml_profile(int n, float m, float kmax, float amax, float r0, float dt,
                    float dx, int T, float *b, float *a, float *ik) {
  for (int i = 0; i < n; i++) { b[i] = 1.0f; a[i] = 0.0f; ik[i] = 1.0f; }
  if (T == 0) return;
  float depth = (float)T * dx;
  float eta0 = sqrtf(MU0 / EPS0);
  float sigma_max = -(m + 1.0f) * logf(r0) / (2.0f * eta0 * depth);
  for (int g = 0; g < T; g++) {
    float rho = (float)(T - g) / (float)T;
    float sigma = sigma_max * powf(rho, m);
    float kappa = 1.0f + (kmax - 1.0f) * powf(rho, m);
    float alpha = amax * (1.0f - rho);
    /* PmlProfile1D::coeffs_from_physical, src/layout.rs:500-513 */
    float bb = expf(-(sigma / kappa + alpha) * dt / EPS0);
    float denom = kappa * (sigma + kappa * alpha);
    float aa = fabsf(denom) > 1.0e-30f ? sigma * (bb - 1.0f) / denom : 0.0f;
    float kk = 1.0f / kappa;
    b[g] = bb; a[g] = aa; ik[g] = kk;
    b[n - 1 - g] = bb; a[n - 1 - g] = aa; ik[n - 1 - g] = kk;
  }
}

float or_waveform_eval(int kind, float p0, float p1, float t) {
  switch (kind) {
    case 0: { /* GaussianPulse{t0=p0, spread=p1} */
      float arg = (t - p0) / p1;
      return expf(-0.5f * arg * arg);
    }
    case 1: /* Sinusoid{freq=p0} */
      return sinf(2.0f * PI_F * p0 * t);
    case 2: { /* RickerWavelet{peak=p0, t0=p1} */
      float arg = PI_F * p0 * (t - p1);
      float arg_sq = arg * arg;
      return (1.0f - 2.0f * arg_sq) * expf(-arg_sq);
    }
  }
  return 0.0f;
}

void or_source_values(int kind, float p0, float p1, float amplitude, float dt,
                      int nsteps, float *values) {
  for (int s = 0; s < nsteps; s++) {
    float t = ((float)s + 1.0f) * dt;
    values[s] = amplitude * or_waveform_eval(kind, p0, p1, t);
  }
}

void or_probe_tables(const float *freqs, int nfreq, float dt, int nsteps,
                     double *cos_tab, double *sin_tab) {
  for (int s = 0; s < nsteps; s++) {
    float t = ((float)s + 1.0f) * dt;
    for (int f = 0; f < nfreq; f++) {
      double omega = 2.0 * PI_D * (double)freqs[f];
      double ph = omega * (double)t;
      cos_tab[(size_t)s * nfreq + f] = cos(ph);
      sin_tab[(size_t)s * nfreq + f] = sin(ph);
    }
  }
}

int or_probe_first_step(float start, float dt) {
  int s = 0;
  while (((float)s + 1.0f) * dt < start) s++;
  return s;
}

/* ------------------------------------------------------------------------ */
/* scene format + voxelizer, src/scene.rs:81-230                             */
/* ------------------------------------------------------------------------ */

static int parse_f32(const char *tok, float *out) {
  /* Rust's str::parse::<f32>: decimal with optional sign/exponent, or
   * inf/infinity/nan.  Hex floats are not accepted. */
  if (strchr(tok, 'x') || strchr(tok, 'X')) return 0;
  char *end = NULL;
  float v = strtof(tok, &end);
  if (end == tok || *end != '\0') return 0;
  *out = v;
  return 1;
}

static void rasterize_sphere(uint8_t *g, int nx, int ny, int nz, float cx,
                             float cy, float cz, float r, uint8_t id) {
  float r2 = r * r;
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        float dx = (float)x + 0.5f - cx;
        float dy = (float)y + 0.5f - cy;
        float dz = (float)z + 0.5f - cz;
        if (dx * dx + dy * dy + dz * dz <= r2) g[((size_t)z * ny + y) * nx + x] = id;
      }
}

static size_t clamp_lo(float v) {
  float m = v > 0.0f ? v : 0.0f; /* f32::max(v, 0.0), NaN -> 0 */
  if (v != v) m = 0.0f;
  float f = floorf(m);
  return f >= 1.8e19f ? (size_t)-1 : (size_t)f;
}
static size_t clamp_hi(float v, size_t n) {
  float c = ceilf(v);
  float m = c > 0.0f ? c : 0.0f;
  if (c != c) m = 0.0f;
  size_t u = m >= 1.8e19f ? (size_t)-1 : (size_t)m;
  return u < n ? u : n;
}

int or_scene_voxelize(const char *text, int nx, int ny, int nz, float dt,
                      float dx, uint8_t *grid, int32_t (*table)[4], char *err,
                      int errlen) {
  uint32_t keys[256][3];
  int nkeys = 0;
  int lineno = 0;
  const char *p = text;
  while (*p || p == text) {
    const char *nl = strchr(p, '\n');
    size_t len = nl ? (size_t)(nl - p) : strlen(p);
    lineno++;
    char *line = (char *)malloc(len + 1);
    memcpy(line, p, len);
    line[len] = 0;
    /* trim */
    char *s = line;
    while (*s == ' ' || *s == '\t' || *s == '\r' || *s == '\v' || *s == '\f') s++;
    char *e = s + strlen(s);
    while (e > s && (e[-1] == ' ' || e[-1] == '\t' || e[-1] == '\r' || e[-1] == '\v' || e[-1] == '\f')) *--e = 0;
    if (*s && *s != '#') {
      char *toks[64] = {0};
      int nt = 0;
      char *save = NULL;
      for (char *t = strtok_r(s, " \t\r\v\f", &save); t && nt < 64; t = strtok_r(NULL, " \t\r\v\f", &save)) toks[nt++] = t;
      int is_sphere = strcmp(toks[0], "sphere") == 0;
      int is_box = strcmp(toks[0], "box") == 0;
      if (!is_sphere && !is_box) {
        snprintf(err, errlen, "scene line %d: unknown primitive '%s'", lineno, toks[0]);
        free(line);
        return -1;
      }
      float v[64];
      for (int i = 1; i < nt; i++) {
        if (!parse_f32(toks[i], &v[i - 1])) {
          snprintf(err, errlen, "scene line %d: invalid number '%s'", lineno, toks[i]);
          free(line);
          return -1;
        }
      }
      int nv = nt - 1;
      if (is_sphere && nv != 7) {
        snprintf(err, errlen, "scene line %d: expected 'sphere eps_r mu_r sigma cx cy cz radius', got %d values", lineno, nv);
        free(line);
        return -1;
      }
      if (is_box && nv != 9) {
        snprintf(err, errlen, "scene line %d: expected 'box eps_r mu_r sigma x0 y0 z0 x1 y1 z1', got %d values", lineno, nv);
        free(line);
        return -1;
      }
      /* material de-duplication by bit pattern, src/scene.rs:161-180 */
      uint32_t k[3];
      memcpy(&k[0], &v[0], 4); memcpy(&k[1], &v[1], 4); memcpy(&k[2], &v[2], 4);
      int id = -1;
      for (int i = 0; i < nkeys; i++)
        if (keys[i][0] == k[0] && keys[i][1] == k[1] && keys[i][2] == k[2]) id = i + 1;
      if (id < 0) {
        if (nkeys + 1 > 255) {
          snprintf(err, errlen, "scene uses more than 255 distinct materials");
          free(line);
          return -1;
        }
        keys[nkeys][0] = k[0]; keys[nkeys][1] = k[1]; keys[nkeys][2] = k[2];
        id = ++nkeys;
        or_material_coeffs(v[0], v[1], v[2], dt, dx, table[id]);
      }
      if (is_sphere) {
        rasterize_sphere(grid, nx, ny, nz, v[3], v[4], v[5], v[6], (uint8_t)id);
      } else {
        float x0 = v[3], y0 = v[4], z0 = v[5], x1 = v[6], y1 = v[7], z1 = v[8];
        size_t xlo = clamp_lo(fminf(x0, x1)), xhi = clamp_hi(fmaxf(x0, x1), nx);
        size_t ylo = clamp_lo(fminf(y0, y1)), yhi = clamp_hi(fmaxf(y0, y1), ny);
        size_t zlo = clamp_lo(fminf(z0, z1)), zhi = clamp_hi(fmaxf(z0, z1), nz);
        for (size_t z = zlo; z < zhi; z++)
          for (size_t y = ylo; y < yhi; y++)
            for (size_t x = xlo; x < xhi; x++) grid[(z * ny + y) * nx + x] = (uint8_t)id;
      }
    }
    free(line);
    if (!nl) break;
    p = nl + 1;
  }
  return nkeys;
}

void or_demo_sphere(int nx, int ny, int nz, uint8_t *grid) {
  float cx = (float)nx / 2.0f, cy = (float)ny / 2.0f, cz = (float)nz / 2.0f;
  int mn = nx < ny ? nx : ny;
  mn = mn < nz ? mn : nz;
  float r = (float)mn / 4.0f;
  rasterize_sphere(grid, nx, ny, nz, cx, cy, cz, r, 1);
}

/* ------------------------------------------------------------------------ */
/* the engine, instantiated for f32 and f64                                  */
/* ------------------------------------------------------------------------ */

typedef void (*or_range_fn)(void *ctx, int b0, int b1);
typedef struct { or_range_fn fn; void *ctx; int b0, b1; } or_job;
static void *or_job_main(void *p) {
  or_job *j = (or_job *)p;
  j->fn(j->ctx, j->b0, j->b1);
  return NULL;
}
/* Runs fn over [0, nb) split into nthreads contiguous ranges.  A phase is a
 * pure function of the other field, so the split never changes results. */
static void or_parallel_blocks(int nb, int nthreads, or_range_fn fn, void *ctx) {
  if (nthreads <= 1 || nb < 2) { fn(ctx, 0, nb); return; }
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  or_job jobs[256];
  int per = (nb + nthreads - 1) / nthreads;
  int nj = 0;
  for (int b0 = 0; b0 < nb; b0 += per) {
    jobs[nj].fn = fn; jobs[nj].ctx = ctx; jobs[nj].b0 = b0;
    jobs[nj].b1 = b0 + per < nb ? b0 + per : nb;
    nj++;
  }
  for (int i = 1; i < nj; i++) pthread_create(&th[i], NULL, or_job_main, &jobs[i]);
  or_job_main(&jobs[0]);
  for (int i = 1; i < nj; i++) pthread_join(th[i], NULL);
}

/* ------------------------------------------------------------------------ */
/* 16-bit field storage (no reference counterpart): the mixed-precision      */
/* form's storage rounding, emulated exactly so the CUDA kernels that store   */
/* f16/bf16 can be checked bit for bit.                                       */
/* ------------------------------------------------------------------------ */

static inline uint32_t or_f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float or_u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

/* |v| as its bit pattern: non-negative floats order like their bits. */
static inline uint32_t or_abs_bits(float v) { return or_f2u(v) & 0x7fffffffu; }

/* Power-of-two shift that maps a bound b into [2^13, 2^14): the biased
 * exponent field of b minus 140, clamped to [-60, 15] (zero or subnormal
 * bounds take -60). */
int or_store_shift(float bound) {
  int e8 = (int)((or_f2u(bound) >> 23) & 0xffu);
  int sh = e8 == 0 ? -60 : e8 - 127 - 13;
  return sh < -60 ? -60 : (sh > 15 ? 15 : sh);
}

/* bf16 from f32, round to nearest even on the dropped 16 bits (NaN and
 * infinities pass unchanged). */
static inline float or_round_bf16(float v) {
  uint32_t u = or_f2u(v);
  if ((u & 0x7f800000u) == 0x7f800000u) return v;
  u += 0x7fffu + ((u >> 16) & 1u);
  return or_u2f(u & 0xffff0000u);
}

/* Rounds u to the 16-bit format: kind 1 = IEEE binary16, round to nearest
 * even, finite values saturating at +-65504; kind 2 = bf16, round to nearest
 * even.  The result is exactly what a device kernel reads back after storing
 * u in that format. */
float or_round16(float u, int kind) {
  if (kind == 1 || kind == 3) {
    if (u > 65504.0f) u = 65504.0f;
    if (u < -65504.0f) u = -65504.0f;
    const float h = (float)(_Float16)u;
    if (kind == 1) return h;
    /* kind 3 (emulation only, no device form): binary16 plus a residual
     * byte, the rounding error u - h (exact in f32) rounded to a signed
     * multiple of 1/256 of h's last place; h + residual is exact in f32
     * (at most 19 significant bits). */
    const float ulp = fabsf(h) >= 6.103515625e-05f ? ldexpf(1.0f, ilogbf(h) - 10)
                                                   : ldexpf(1.0f, -24);
    float q = rintf((u - h) / ulp * 256.0f);
    q = q > 127.0f ? 127.0f : (q < -128.0f ? -128.0f : q);
    return h + q * (ulp / 256.0f);
  }
  return or_round_bf16(u);
}

/* Stores v as a 16-bit value of v * 2^-shift and returns the decoded f32
 * value (scaling by a power of two is exact).  overflow is unused: the
 * simulation counts slabs whose maximum reached +-65504, see next_shifts. */
float or_store16(float v, int kind, int shift, long long *overflow) {
  (void)overflow;
  return or_round16(v * ldexpf(1.0f, -shift), kind) * ldexpf(1.0f, shift);
}

#define REAL float
#define SIM or_sim_f32
#define FN(n) or_sim_f32_##n
#include "wf_oracle_sim.inc"
#undef REAL
#undef SIM
#undef FN

#define REAL double
#define SIM or_sim_f64
#define FN(n) or_sim_f64_##n
#include "wf_oracle_sim.inc"
#undef REAL
#undef SIM
#undef FN

/* ------------------------------------------------------------------------ */
/* validation studies                                                        */
/* ------------------------------------------------------------------------ */

static size_t nx8(size_t v) { return (v + 7) / 8 * 8; }

/* run_plane_wave of examples/convergence_study.rs:81-179 and
 * examples/pml_reflection_study.rs:88-202: vacuum nx*8*8, periodic y/z,
 * hard Ez sheet at x_source with sin(omega t), probe trace at x_probe. */
static double *plane_wave_trace(int nx, float dx, float dt, float freq,
                                int x_source, int x_probe, int steps,
                                int pml_voxels) {
  uint8_t *mat = (uint8_t *)calloc((size_t)nx * 64, 1);
  int32_t table[256][4];
  int32_t vac[4];
  or_material_coeffs(1.0f, 1.0f, 0.0f, dt, dx, vac);
  for (int i = 0; i < 256; i++) memcpy(table[i], vac, sizeof(vac));
  int periodic[3] = {0, 1, 1};
  or_sim_f32 *s = or_sim_f32_create(nx, 8, 8, mat, (const int32_t(*)[4])table, periodic);
  free(mat);
  if (pml_voxels > 0) {
    int bx_n = nx / 8;
    int tb = (pml_voxels + 7) / 8;
    if (tb > bx_n / 2) tb = bx_n / 2;
    int teff = tb * 8;
    float *b = (float *)malloc(4 * nx), *a = (float *)malloc(4 * nx), *k = (float *)malloc(4 * nx);
    or_pml_profile(nx, 3.0f, 7.0f, 0.05f, 1.0e-6f, dt, dx, teff, b, a, k);
    const float *bb[3] = {b, NULL, NULL}, *aa[3] = {a, NULL, NULL}, *kk[3] = {k, NULL, NULL};
    int shell[3] = {tb, 0, 0};
    if (tb > 0) or_sim_f32_set_pml(s, bb, aa, kk, shell);
    free(b); free(a); free(k);
  }
  float omega = 2.0f * PI_F * freq;
  float *vals = (float *)malloc(sizeof(float) * steps);
  for (int st = 0; st < steps; st++) {
    float t = ((float)st + 1.0f) * dt;
    vals[st] = sinf(omega * t);
  }
  or_sim_f32_add_source(s, x_source, 0, 0, 2, OR_SRC_HARD_SHEET_X, vals, steps);
  free(vals);
  or_sim_f32_add_probe(s, x_probe, 0, 0, 2, 0, NULL, NULL, steps, 0, 1);
  or_sim_f32_step(s, steps, 1);
  double *tr = (double *)malloc(sizeof(double) * steps);
  or_sim_f32_probe_trace(s, 0, tr);
  or_sim_f32_destroy(s);
  return tr;
}

static float yee_theory_v(float dx, float dt, float f) {
  float omega = 2.0f * PI_F * f;
  float rhs = (dx / (C0 * dt)) * sinf(omega * dt / 2.0f);
  float k = (2.0f / dx) * asinf(rhs);
  return omega / k;
}

static float log_log_slope(const float *xs, const float *ys, int n) {
  float lx[8], ly[8];
  for (int i = 0; i < n; i++) { lx[i] = log10f(xs[i]); ly[i] = log10f(ys[i]); }
  float sx = -0.0f, sy = -0.0f;
  for (int i = 0; i < n; i++) sx += lx[i];
  for (int i = 0; i < n; i++) sy += ly[i];
  float mx = sx / (float)n, my = sy / (float)n;
  float cov = -0.0f, var = -0.0f;
  for (int i = 0; i < n; i++) cov += (lx[i] - mx) * (ly[i] - my);
  for (int i = 0; i < n; i++) { float d = lx[i] - mx; var += d * d; }
  return cov / var;
}

void or_convergence_study(float rows[4][6], float *mslope, float *tslope, float *maxd) {
  const float freq = 3.0e10f;
  const float wl = C0 / freq;
  const float courant = 0.4f;
  const float periods = 8.0f;
  const float ppws[4] = {10.0f, 15.0f, 20.0f, 30.0f};
  for (int r = 0; r < 4; r++) {
    float ppw = ppws[r];
    float dx = wl / ppw;
    float dt = courant * dx / C0;
    float period_s = 1.0f / freq;
    float period_steps = ppw / courant;
    size_t n_vox = (size_t)roundf(periods * ppw);
    size_t x_source = 3 * n_vox;
    size_t x_probe = x_source + n_vox;
    size_t nx = nx8(7 * n_vox);
    size_t steps = (size_t)ceilf((periods + 12.0f) * period_steps);
    float expected_delay = ((float)n_vox * dx) / C0;
    double omega = 2.0 * PI_D * (double)freq;
    double *tr = plane_wave_trace((int)nx, dx, dt, freq, (int)x_source, (int)x_probe, (int)steps, 0);
    float skip = expected_delay + 5.0f * period_s;
    double sc = 0.0, ss = 0.0;
    uint32_t count = 0;
    for (size_t i = 0; i < steps; i++) {
      float t = ((float)i + 1.0f) * dt;
      if (t > skip) {
        double ph = omega * (double)t;
        sc += tr[i] * cos(ph);
        ss += tr[i] * sin(ph);
        count++;
      }
    }
    free(tr);
    double a = 2.0 * sc / (double)count;
    double b = 2.0 * ss / (double)count;
    double raw_delay = atan2(-a, b) / omega;
    double k = round(((double)expected_delay - raw_delay) / (double)period_s);
    float measured_delay = (float)(raw_delay + k * (double)period_s);
    float mv = ((float)n_vox * dx) / measured_delay;
    float tv = yee_theory_v(dx, dt, freq);
    rows[r][0] = dx;
    rows[r][1] = ppw;
    rows[r][2] = mv;
    rows[r][3] = tv;
    rows[r][4] = fabsf(mv - C0) / C0;
    rows[r][5] = fabsf(tv - C0) / C0;
  }
  float dxs[4], me[4], te[4];
  for (int r = 0; r < 4; r++) { dxs[r] = rows[r][0]; me[r] = rows[r][4]; te[r] = rows[r][5]; }
  *mslope = log_log_slope(dxs, me, 4);
  *tslope = log_log_slope(dxs, te, 4);
  float md = 0.0f;
  for (int r = 0; r < 4; r++) {
    float d = fabsf(rows[r][4] - rows[r][5]);
    md = fmaxf(md, d);
  }
  *maxd = md;
}

static double quad_amp(const double *tr, size_t n, float dt, double omega, float skip) {
  double sc = 0.0, ss = 0.0;
  uint32_t count = 0;
  for (size_t i = 0; i < n; i++) {
    float t = ((float)i + 1.0f) * dt;
    if (t > skip) {
      double ph = omega * (double)t;
      sc += tr[i] * cos(ph);
      ss += tr[i] * sin(ph);
      count++;
    }
  }
  double a = 2.0 * sc / (double)count;
  double b = 2.0 * ss / (double)count;
  return sqrt(a * a + b * b);
}

void or_pml_reflection_study(double refl[4]) {
  const float freq = 3.0e10f;
  const float wl = C0 / freq;
  const float courant = 0.4f;
  const float ppw = 20.0f;
  const float dx = wl / ppw;
  const float dt = courant * dx / C0;
  const float period_s = 1.0f / freq;
  size_t probe_off = (size_t)roundf(3.0f * ppw);
  size_t right_gap = (size_t)roundf(2.0f * ppw);
  const int tbs[4] = {1, 2, 4, 8};
  for (int r = 0; r < 4; r++) {
    size_t T = (size_t)tbs[r] * 8;
    size_t xs_test = T + (size_t)roundf(2.0f * ppw);
    size_t xp_test = xs_test + probe_off;
    size_t face = xp_test + right_gap;
    size_t nx_test = nx8(face + T);
    float incident_delay = (float)probe_off * dx / C0;
    size_t rt_vox = 2 * (face - xp_test);
    float rt_s = (float)rt_vox * dx / C0;
    float settle = 6.0f;
    float skip = incident_delay + rt_s + settle * period_s;
    float meas = 10.0f;
    size_t steps = (size_t)ceilf((skip + meas * period_s) / dt) + 4;
    double *tt = plane_wave_trace((int)nx_test, dx, dt, freq, (int)xs_test, (int)xp_test, (int)steps, (int)T);
    size_t req = (size_t)ceilf(((float)steps * dt + 2.0f * period_s) * C0 / dx) + 8;
    size_t xp_ref = req + probe_off;
    size_t xs_ref = xp_ref - probe_off;
    size_t nx_ref = nx8(xp_ref + req);
    double *rt = plane_wave_trace((int)nx_ref, dx, dt, freq, (int)xs_ref, (int)xp_ref, (int)steps, 0);
    double omega = 2.0 * PI_D * (double)freq;
    double inc = quad_amp(rt, steps, dt, omega, skip);
    double *diff = (double *)malloc(sizeof(double) * steps);
    for (size_t i = 0; i < steps; i++) diff[i] = (double)((float)tt[i] - (float)rt[i]);
    double refl_amp = quad_amp(diff, steps, dt, omega, skip);
    refl[r] = refl_amp / inc;
    free(tt); free(rt); free(diff);
  }
}
