/*
 * wf_oracle.h -- CPU oracle for the wavefront FDTD timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * Rust implementation (AndrejRumenovski/wavefront) used as the parity checker
 * for the CUDA library in wavefront_b200/.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it.  The product never links it.
 *
 * Parity is pinned: the restatement reproduces the reference's own golden
 * outputs validation/convergence_data.csv and validation/pml_reflection_data.csv
 * (see tests/test_oracle_golden.py).
 *
 * Layout follows the reference exactly: the field grid is block-major 8^3
 * AoSoA tiles (src/layout.rs:697-755), each tile holding ex,ey,ez,hx,hy,hz as
 * 512 floats, block index (bz*nby+by)*nbx+bx, local index (lz*8+ly)*8+lx.
 * All arithmetic is evaluated in the reference's operation order with no FMA
 * contraction (build with -ffp-contract=off).
 */
#ifndef WF_ORACLE_H
#define WF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- setup math (src/layout.rs, src/source.rs) ------------------------- */
int32_t or_q16_from_f32(float v);                    /* src/layout.rs:114-116 */
float   or_q16_to_f32(int32_t q);                    /* src/layout.rs:123-125 */
void    or_material_coeffs(float eps_r, float mu_r, float sigma, float dt,
                           float d, int32_t out_q16[4]); /* src/layout.rs:194-208 */
int     or_effective_pml_thickness_blocks(int nx, int ny, int nz,
                                          int requested_voxels); /* :525-533 */
void    or_pml_profile(int n, float grading_order, float kappa_max,
                       float alpha_max, float target_reflection, float dt,
                       float dx, int thickness_voxels, float *b, float *a,
                       float *inv_kappa);            /* src/layout.rs:471-513 */
/* kind: 0 Gaussian(p0=t0, p1=spread), 1 Sinusoid(p0=freq), 2 Ricker(p0=freq, p1=t0) */
float   or_waveform_eval(int kind, float p0, float p1, float t); /* src/source.rs:46-59 */

/* values[i] = amplitude * waveform(((i as f32) + 1) * dt), src/engine.rs:769 */
void    or_source_values(int kind, float p0, float p1, float amplitude, float dt,
                         int nsteps, float *values);
/* [s*nfreq+f] = cos/sin(2*pi*(double)freq_f * (double)t_s), src/probe.rs:133-136 */
void    or_probe_tables(const float *freqs, int nfreq, float dt, int nsteps,
                        double *cos_tab, double *sin_tab);
/* first step s with !(t_s < start), src/probe.rs:127 */
int     or_probe_first_step(float start, float dt);

/* ---- scene format + voxelizer (src/scene.rs:81-230) -------------------- */
/* Voxelizes scene text into `grid` (nx*ny*nz bytes, pre-filled by caller) and
 * writes Q16.16 coefficients of every registered material into table[id].
 * Returns the number of distinct materials, or -1 with a message in err. */
int or_scene_voxelize(const char *text, int nx, int ny, int nz, float dt,
                      float dx, uint8_t *grid, int32_t (*table)[4], char *err,
                      int errlen);
/* src/main.rs:403-425: material id 1 sphere at the domain centre. */
void or_demo_sphere(int nx, int ny, int nz, uint8_t *grid);

/* ---- 16-bit field storage (mixed-precision form; no reference code) ----- */
/* Shift mapping a bound into [2^13, 2^14) (biased exponent - 140, clamped
 * to [-60, 15]). */
int   or_store_shift(float bound);
/* u rounded to kind (1 f16 saturating, 2 bf16; both round to nearest even). */
float or_round16(float u, int kind);
/* Decoded value of v stored as kind of v * 2^-shift. */
float or_store16(float v, int kind, int shift, long long *overflow);

/* ---- the timestep engine (src/engine.rs, src/fdtd.rs) ------------------ */
typedef struct or_sim_f32 or_sim_f32;
typedef struct or_sim_f64 or_sim_f64;

#define OR_BOUNDARY_ZERO 0
#define OR_BOUNDARY_PERIODIC 1

#define OR_SRC_SOFT 0       /* E_c[voxel] += v           src/source.rs:79-95 */
#define OR_SRC_HARD_SHEET_X 1 /* E_c[x0, all y, all z] = v (studies' sheet) */

#define OR_DECLARE_SIM(S, R)                                                     \
  S *S##_create(int nx, int ny, int nz, const uint8_t *mat,                     \
                const int32_t (*table_q16)[4], const int periodic[3]);          \
  void S##_destroy(S *s);                                                        \
  /* per-axis graded profiles (length n of that axis) and per-axis shell        \
   * thickness in blocks; a block is in the shell if it lies within that       \
   * axis's thickness of either face on ANY axis (src/layout.rs:594-618). */   \
  int S##_set_pml(S *s, const float *const b[3], const float *const a[3],       \
                  const float *const ik[3], const int shell_blocks[3]);         \
  int S##_add_source(S *s, int x, int y, int z, int comp, int mode,             \
                     const float *values, int nvalues);                         \
  int S##_add_probe(S *s, int x, int y, int z, int comp, int nfreq,             \
                    const double *cos_tab, const double *sin_tab, int nsteps,   \
                    int first_step, int record_trace);                          \
  void S##_step(S *s, int nsteps, int nthreads);                                \
  int S##_steps_done(const S *s);                                               \
  void S##_get_fields(const S *s, R *out6); /* 6 SoA arrays, x fastest */      \
  void S##_set_fields(S *s, const R *in6);                                      \
  void S##_get_blocks(const S *s, R *out); /* raw FieldBlock order */          \
  /* psi of one of 12 reference PmlAux arrays, scattered to x-fastest grid   \
   * order (zero outside shell blocks). */                                      \
  void S##_get_psi(const S *s, int which, R *out);                              \
  void S##_probe_sums(const S *s, int p, double *cos_out, double *sin_out,      \
                      uint64_t *n);                                             \
  void S##_probe_trace(const S *s, int p, double *out);                         \
  /* 16-bit field storage (f32 sim only): 0 plain, 1 f16, 2 bf16.  Re-encodes  \
   * the current state; -1 for a bad kind or on the f64 sim. */                \
  int S##_set_storage(S *s, int kind);                                          \
  /* 1: restate the device FMA build's fused forms (f32 sim, plain storage);   \
   * -1 otherwise. */                                                           \
  int S##_set_arith(S *s, int fma);                                             \
  long long S##_storage_overflows(const S *s);                                  \
  /* write shifts (per 8-plane z slab) of the next step, E and H kinds */      \
  void S##_get_shifts(const S *s, int *shift_e, int *shift_h);

OR_DECLARE_SIM(or_sim_f32, float)
OR_DECLARE_SIM(or_sim_f64, double)

/* ---- validation studies (the reference's examples/) --------------------- */
/* examples/convergence_study.rs:204-369.  rows[4][6] receives
 * dx, ppw, measured_v, theory_v, measured_err, theory_err (f32 values). */
void or_convergence_study(float rows[4][6], float *measured_slope,
                          float *theory_slope, float *max_discrepancy);
/* examples/pml_reflection_study.rs:237-387.  refl[4] for 1,2,4,8 blocks. */
void or_pml_reflection_study(double refl[4]);

#ifdef __cplusplus
}
#endif
#endif
