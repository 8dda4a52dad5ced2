/* Test infrastructure only -- the CPU oracle for the FDTD (Yee) hot path.
 *
 * A plain-C restatement of the reference algorithm, used as the checker by tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py.  The product
 * (gdiamond_b200/, include/) never includes, links or calls it.
 *
 * Parity is pinned: the FP32 stepper and the coefficient builder are checked bit-for-bit
 * against the reference's own update_FDTD_seq / gDiamond constructor, compiled from the
 * reference sources into oracle/_ref/libgdref.so (tests/test_oracle_pin.py), and against
 * the committed golden fixtures in tests/golden/.
 *
 * Layout everywhere: x-fastest structure of arrays, idx = i + j*Nx + k*Nx*Ny.
 * Component order: Ex Ey Ez Hx Hy Hz.  Coefficient order:
 *   Cax Cay Caz Cbx Cby Cbz Dax Day Daz Dbx Dby Dbz.
 */
#ifndef GDIAMOND_ORACLE_H
#define GDIAMOND_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Source kinds: a single cell, or every interior cell of the z-plane k. */
enum { ORACLE_SRC_POINT = 0, ORACLE_SRC_PLANE_Z = 1 };

/* One current source.  component: 0..2 = Jx Jy Jz (enters the E update as -J*dx),
 * 3..5 = Mx My Mz (enters the H update as -M*dx).  Waveform sample t is used at step t. */
typedef struct oracle_source {
  int32_t component;
  int32_t kind;
  int64_t i, j, k;
} oracle_source;

/* One running-DFT monitor on the z-plane k of one field component (0..5). */
typedef struct oracle_monitor {
  int32_t component;
  int32_t nf;
  int64_t k;
  double scale;
  const double* cos_tab; /* [T_total][nf], indexed by the global step t */
  const double* sin_tab;
  double* re; /* [nf][Nx*Ny] running sums, updated in place */
  double* im;
} oracle_monitor;

/* Coefficients as built by gDiamond's constructor (gDiamond/gdiamond.hpp:20-73 calling
 * set_FDTD_matrices_3D_structure, gDiamond/utils.h:542-690), generalised to a per-cell
 * relative permittivity eps_re/eps_im (NULL = vacuum 1+0j).  t_pml cells of graded
 * pseudo-PML at every face; omega0 is the reference source omega.  Writes 12 arrays. */
void oracle_coefficients(int64_t Nx, int64_t Ny, int64_t Nz, float dx, float dt, float omega0,
                         int t_pml, const float* eps_re, const float* eps_im, float* const* c12);

/* The reference constructor's default physical constants (gDiamond/gdiamond.hpp:893-906):
 * out = {dx, dt, J_amp, M_amp, omega, t_sigma, t_peak}; t_pml = 10. */
void oracle_reference_params(float* out7, int* t_pml);

/* The reference update_FDTD_seq source waveform: M_amp*sin(omega*t*dt), FP32
 * (gDiamond/gdiamond.hpp:1189-1191). */
void oracle_reference_mz_wave(int64_t T, float* out);

/* FP64 cos/sin tables for the running DFT: ph = (2*pi*f) * ((double)t * dt), t = 0..T-1. */
void oracle_dft_tables_offset(const double* freqs, int nf, double dt, double t_offset, int64_t T,
                              double* cos_tab, double* sin_tab);
void oracle_dft_tables(const double* freqs, int nf, double dt, int64_t T, double* cos_tab,
                       double* sin_tab);

/* T Yee steps starting at global step t0, FP32 storage and arithmetic, restating the loop
 * body of update_FDTD_seq (gDiamond/gdiamond.hpp:1193-1221) in the same operation order
 * (no contraction).  F = 6 field arrays updated in place; waves = [nsrc][Tw]. */
void oracle_run_f32(int64_t Nx, int64_t Ny, int64_t Nz, float* const* F, const float* const* C,
                    float dx, const oracle_source* src, int nsrc, const float* waves, int64_t Tw,
                    int64_t t0, int64_t T, const oracle_monitor* mon, int nmon);

/* The same scheme in FP64 (fields and arithmetic), coefficients and waveforms widened
 * from their FP32 values.  The error reference for reduced-precision runs. */
void oracle_run_f64(int64_t Nx, int64_t Ny, int64_t Nz, double* const* F, const float* const* C,
                    float dx, const oracle_source* src, int nsrc, const float* waves, int64_t Tw,
                    int64_t t0, int64_t T, const oracle_monitor* mon, int nmon);

#ifdef __cplusplus
}
#endif

#endif
