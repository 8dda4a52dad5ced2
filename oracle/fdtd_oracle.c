/* Test infrastructure only -- CPU oracle for the FDTD (Yee) hot path.  See fdtd_oracle.h.
 *
 * Build flags matter: -ffp-contract=off keeps every multiply and add separately rounded, as
 * in the reference build (x86-64 g++ without FMA), so the FP32 stepper reproduces
 * update_FDTD_seq bit for bit.
 */
#include "fdtd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- constants */

/* gDiamond/utils.h:19 defines PI as this float literal. */
#define REF_PI 3.14159265359f
/* pi in double precision (the running-DFT phase is computed in FP64). */
#define PI_D 3.14159265358979323846

void oracle_reference_params(float* out7, int* t_pml) {
  /* gDiamond/gdiamond.hpp:893-906 and gDiamond/utils.h:19-22 (eps0 = mu0 = c0 = eta0 = 1). */
  const float um = 1.0f;
  const float wavelength = 1.0f * um;
  const float freq = 1.0f / wavelength;           /* c0 / wavelength, c0 == 1 */
  const float omega = 2 * REF_PI * freq;          /* float arithmetic, as the reference */
  const float dx = wavelength / 10;
  const float dt = 0.05f;
  const float j_amp = 5e4f;
  const float m_amp = (float)(j_amp * pow(1.0, 3.0)); /* J_amp * eta0^3 */
  const float freq_sigma = (float)(0.05 * freq);
  const float t_sigma = (float)(1 / freq_sigma / (2 * REF_PI));
  const float t_peak = 5 * t_sigma;
  out7[0] = dx;
  out7[1] = dt;
  out7[2] = j_amp;
  out7[3] = m_amp;
  out7[4] = omega;
  out7[5] = t_sigma;
  out7[6] = t_peak;
  if (t_pml) {
    /* t_PML = ceil(h_PML / dx) with h_PML = 1 um (gDiamond/gdiamond.hpp:63-64). */
    const float h_pml = 1.0f * um;
    *t_pml = (int)ceilf(h_pml / dx);
  }
}

void oracle_reference_mz_wave(int64_t T, float* out) {
  float p[7];
  oracle_reference_params(p, NULL);
  const float dt = p[1], m_amp = p[3], omega = p[4];
  for (int64_t t = 0; t < T; ++t) {
    /* M_source_amp * std::sin(SOURCE_OMEGA * t * dt): float product, float sin. */
    const float arg = (omega * (float)t) * dt;
    out[t] = m_amp * sinf(arg);
  }
}

/* ------------------------------------------------------- coefficient builder */

typedef struct { float re, im; } cpx;

static cpx cmul(cpx a, cpx b) {
  cpx r;
  r.re = a.re * b.re - a.im * b.im;
  r.im = a.re * b.im + a.im * b.re;
  return r;
}

static cpx cdiv(cpx a, cpx b) {
  const float den = b.re * b.re + b.im * b.im;
  cpx r;
  r.re = (a.re * b.re + a.im * b.im) / den;
  r.im = (a.im * b.re - a.re * b.im) / den;
  return r;
}

/* Graded stretch factor of one axis (gDiamond/utils.h:585-619). */
static cpx stretch(int64_t i, int64_t n, int t_pml, float a_max, float sigma_max, float omega0) {
  float dist = 0;
  if (i < t_pml) dist = (float)(1.0 - (double)((float)i / (float)t_pml));
  if (i + t_pml >= n) dist = (float)(1.0 - (double)((float)(int)(n - i - 1) / (float)t_pml));
  const double d3 = pow((double)dist, 3.0);
  cpx s;
  s.re = (float)(1.0 + (double)a_max * d3);
  s.im = (float)((double)sigma_max * d3 / (double)(omega0 * 1.0f));
  return s;
}

/* One (Ca, Cb) pair from a complex material value (gDiamond/utils.h:637-686). */
static void c_pair(cpx m, float omega0, float dt, float dx, float* ca, float* cb) {
  float re = m.re;
  if (re < 1) re = 1;
  const float sigma = fabsf(omega0 * 1.0f * m.im);
  const float tmp = (float)((double)(sigma * dt) / (2.0 * (double)re * 1.0));
  *ca = (float)((1.0 - (double)tmp) / (1.0 + (double)tmp));
  *cb = (float)((double)(dt / (re * 1.0f)) / (1.0 + (double)tmp) / (double)dx);
}

void oracle_coefficients(int64_t Nx, int64_t Ny, int64_t Nz, float dx, float dt, float omega0,
                         int t_pml, const float* eps_re, const float* eps_im, float* const* c12) {
  const float a_max = 2.0f;
  const int p = 3;
  /* -(p + 1) * log(1e-5) / (2 * eta0 * t_PML * dx), eta0 = sqrt(1.0f/1.0f) as a float. */
  const float denom = 2 * 1.0f * (float)t_pml * dx;
  const float sigma_max = (float)((double)(-(p + 1)) * log(1e-5) / (double)denom);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < Nz; ++k) {
    const cpx sz = stretch(k, Nz, t_pml, a_max, sigma_max, omega0);
    for (int64_t j = 0; j < Ny; ++j) {
      const cpx sy = stretch(j, Ny, t_pml, a_max, sigma_max, omega0);
      for (int64_t i = 0; i < Nx; ++i) {
        const cpx sx = stretch(i, Nx, t_pml, a_max, sigma_max, omega0);
        const int64_t idx = i + j * Nx + k * Nx * Ny;
        cpx eps = {1.0f, 0.0f};
        if (eps_re) eps.re = eps_re[idx];
        if (eps_im) eps.im = eps_im[idx];
        const cpx mu = {1.0f, 0.0f};
        const cpx exx = cdiv(cmul(cmul(eps, sy), sz), sx);
        const cpx eyy = cdiv(cmul(cmul(eps, sx), sz), sy);
        const cpx ezz = cdiv(cmul(cmul(eps, sx), sy), sz);
        const cpx mxx = cdiv(cmul(cmul(mu, sy), sz), sx);
        const cpx myy = cdiv(cmul(cmul(mu, sx), sz), sy);
        const cpx mzz = cdiv(cmul(cmul(mu, sx), sy), sz);
        c_pair(exx, omega0, dt, dx, &c12[0][idx], &c12[3][idx]);
        c_pair(eyy, omega0, dt, dx, &c12[1][idx], &c12[4][idx]);
        c_pair(ezz, omega0, dt, dx, &c12[2][idx], &c12[5][idx]);
        c_pair(mxx, omega0, dt, dx, &c12[6][idx], &c12[9][idx]);
        c_pair(myy, omega0, dt, dx, &c12[7][idx], &c12[10][idx]);
        c_pair(mzz, omega0, dt, dx, &c12[8][idx], &c12[11][idx]);
      }
    }
  }
}

/* ----------------------------------------------------------------- DFT */

void oracle_dft_tables(const double* freqs, int nf, double dt, int64_t T, double* cos_tab,
                       double* sin_tab) {
  oracle_dft_tables_offset(freqs, nf, dt, 0.0, T, cos_tab, sin_tab);
}

/* The same with step t phased at (t + t_offset) * dt: t_offset = 1/2 for the H fields of a
 * flux monitor (H of step t is half a step later than E of step t). */
void oracle_dft_tables_offset(const double* freqs, int nf, double dt, double t_offset, int64_t T,
                              double* cos_tab, double* sin_tab) {
  for (int64_t t = 0; t < T; ++t) {
    const double tt = ((double)t + t_offset) * dt;
    for (int f = 0; f < nf; ++f) {
      const double w = 2.0 * PI_D * freqs[f];
      const double ph = w * tt;
      cos_tab[t * nf + f] = cos(ph);
      sin_tab[t * nf + f] = sin(ph);
    }
  }
}

/* ---------------------------------------------------------------- stepper */

static int covers(const oracle_source* s, int64_t i, int64_t j, int64_t k) {
  if (s->kind == ORACLE_SRC_POINT) return s->i == i && s->j == j && s->k == k;
  return s->k == k; /* plane source: every interior cell of plane k */
}

/* STEPPER(name, T): the loop body of update_FDTD_seq in storage type T.  Each curl is
 * evaluated as ((a - b) - (c - d)) and, only at cells that carry a source, minus J*dx,
 * exactly as ((a - b) - (c - d) - J*dx) evaluates when J == 0 elsewhere. */
#define STEPPER(NAME, T)                                                                         \
  void NAME(int64_t Nx, int64_t Ny, int64_t Nz, T* const* F, const float* const* C, float dx_f,  \
            const oracle_source* src, int nsrc, const float* waves, int64_t Tw, int64_t t0,      \
            int64_t nsteps, const oracle_monitor* mon, int nmon) {                               \
    T* Ex = F[0]; T* Ey = F[1]; T* Ez = F[2]; T* Hx = F[3]; T* Hy = F[4]; T* Hz = F[5];          \
    const float *Cax = C[0], *Cay = C[1], *Caz = C[2], *Cbx = C[3], *Cby = C[4], *Cbz = C[5];    \
    const float *Dax = C[6], *Day = C[7], *Daz = C[8], *Dbx = C[9], *Dby = C[10], *Dbz = C[11];  \
    const T dx = (T)dx_f;                                                                        \
    const int64_t sx = 1, sy = Nx, sz = Nx * Ny;                                                 \
    for (int64_t t = t0; t < t0 + nsteps; ++t) {                                                 \
      /* ---- E */                                                                               \
      _Pragma("omp parallel for schedule(static)")                                               \
      for (int64_t k = 1; k < Nz - 1; ++k) {                                                     \
        int plane_src = 0;                                                                       \
        for (int s = 0; s < nsrc; ++s)                                                           \
          if (src[s].component < 3 && src[s].k == k) plane_src = 1;                              \
        for (int64_t j = 1; j < Ny - 1; ++j) {                                                   \
          for (int64_t i = 1; i < Nx - 1; ++i) {                                                 \
            const int64_t idx = i + j * sy + k * sz;                                             \
            T cx = (Hz[idx] - Hz[idx - sy]) - (Hy[idx] - Hy[idx - sz]);                          \
            T cy = (Hx[idx] - Hx[idx - sz]) - (Hz[idx] - Hz[idx - sx]);                          \
            T cz = (Hy[idx] - Hy[idx - sx]) - (Hx[idx] - Hx[idx - sy]);                          \
            if (plane_src) {                                                                     \
              T J[3] = {0, 0, 0};                                                                \
              int any[3] = {0, 0, 0};                                                            \
              for (int s = 0; s < nsrc; ++s) {                                                   \
                const int c = src[s].component;                                                  \
                if (c < 3 && covers(&src[s], i, j, k)) {                                         \
                  J[c] = J[c] + (T)(t < Tw ? waves[(int64_t)s * Tw + t] : 0.0f);                 \
                  any[c] = 1;                                                                    \
                }                                                                                \
              }                                                                                  \
              if (any[0]) cx = cx - J[0] * dx;                                                   \
              if (any[1]) cy = cy - J[1] * dx;                                                   \
              if (any[2]) cz = cz - J[2] * dx;                                                   \
            }                                                                                    \
            Ex[idx] = (T)Cax[idx] * Ex[idx] + (T)Cbx[idx] * cx;                                  \
            Ey[idx] = (T)Cay[idx] * Ey[idx] + (T)Cby[idx] * cy;                                  \
            Ez[idx] = (T)Caz[idx] * Ez[idx] + (T)Cbz[idx] * cz;                                  \
          }                                                                                      \
        }                                                                                        \
      }                                                                                          \
      /* ---- H */                                                                               \
      _Pragma("omp parallel for schedule(static)")                                               \
      for (int64_t k = 1; k < Nz - 1; ++k) {                                                     \
        int plane_src = 0;                                                                       \
        for (int s = 0; s < nsrc; ++s)                                                           \
          if (src[s].component >= 3 && src[s].k == k) plane_src = 1;                             \
        for (int64_t j = 1; j < Ny - 1; ++j) {                                                   \
          for (int64_t i = 1; i < Nx - 1; ++i) {                                                 \
            const int64_t idx = i + j * sy + k * sz;                                             \
            T cx = (Ey[idx + sz] - Ey[idx]) - (Ez[idx + sy] - Ez[idx]);                          \
            T cy = (Ez[idx + sx] - Ez[idx]) - (Ex[idx + sz] - Ex[idx]);                          \
            T cz = (Ex[idx + sy] - Ex[idx]) - (Ey[idx + sx] - Ey[idx]);                          \
            if (plane_src) {                                                                     \
              T M[3] = {0, 0, 0};                                                                \
              int any[3] = {0, 0, 0};                                                            \
              for (int s = 0; s < nsrc; ++s) {                                                   \
                const int c = src[s].component - 3;                                              \
                if (c >= 0 && covers(&src[s], i, j, k)) {                                        \
                  M[c] = M[c] + (T)(t < Tw ? waves[(int64_t)s * Tw + t] : 0.0f);                 \
                  any[c] = 1;                                                                    \
                }                                                                                \
              }                                                                                  \
              if (any[0]) cx = cx - M[0] * dx;                                                   \
              if (any[1]) cy = cy - M[1] * dx;                                                   \
              if (any[2]) cz = cz - M[2] * dx;                                                   \
            }                                                                                    \
            Hx[idx] = (T)Dax[idx] * Hx[idx] + (T)Dbx[idx] * cx;                                  \
            Hy[idx] = (T)Day[idx] * Hy[idx] + (T)Dby[idx] * cy;                                  \
            Hz[idx] = (T)Daz[idx] * Hz[idx] + (T)Dbz[idx] * cz;                                  \
          }                                                                                      \
        }                                                                                        \
      }                                                                                          \
      /* ---- running DFT of the fields after step t */                                          \
      for (int m = 0; m < nmon; ++m) {                                                           \
        const oracle_monitor* mo = &mon[m];                                                      \
        const T* fld = F[mo->component] + mo->k * sz;                                            \
        const int64_t np = Nx * Ny;                                                              \
        const double* ct = mo->cos_tab + t * mo->nf;                                             \
        const double* st = mo->sin_tab + t * mo->nf;                                             \
        _Pragma("omp parallel for schedule(static)")                                             \
        for (int64_t p = 0; p < np; ++p) {                                                       \
          const double v = (double)fld[p];                                                       \
          for (int f = 0; f < mo->nf; ++f) {                                                     \
            mo->re[f * np + p] = mo->re[f * np + p] + (v * ct[f]) * mo->scale;                   \
            mo->im[f * np + p] = mo->im[f * np + p] - (v * st[f]) * mo->scale;                   \
          }                                                                                      \
        }                                                                                        \
      }                                                                                          \
    }                                                                                            \
  }

STEPPER(oracle_run_f32, float)
STEPPER(oracle_run_f64, double)
