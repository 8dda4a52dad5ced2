// gdiamond_compat.hpp -- the gdiamond::gDiamond class surface on top of the B200 C-ABI.
//
// A header-only C++ class with the reference's name, constructor and update/check methods
// (gDiamond/gdiamond.hpp:17-907), so code written against gDiamond compiles unchanged:
//
//   gdiamond::gDiamond exp(Nx, Ny, Nz);      // coefficients exactly as the reference builds them
//   exp.update_FDTD_seq(T);                  // CPU, single thread   -> results "seq"
//   exp.update_FDTD_omp(T);                  // CPU, OpenMP          -> results "omp"
//   exp.update_FDTD_gpu_2D(T);               // B200 through fdtd_capi.h -> results "gpu"
//   exp.check_correctness_gpu_2D();          // |seq - gpu| < 1e-8 on all six components
//
// Every update_FDTD_gpu* method runs CUDA kernels through the C-ABI (fdtd_step); none of them
// falls back to the CPU loops.  The CPU methods are the reference's own CPU paths (they are part
// of the class surface), restated with the same arithmetic order; build with
// -ffp-contract=off (as the reference's x86-64 build effectively is) to keep them bit-exact.
//
// Link: -Iinclude -Lgdiamond_b200 -lgdiamond_b200 (and -fopenmp for update_FDTD_omp).
#pragma once

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "fdtd_capi.h"

namespace gdiamond {

class gDiamond {
 public:
  enum Component { Ex = 0, Ey, Ez, Hx, Hy, Hz };
  enum Variant { SEQ = 0, OMP = 1, GPU = 2, GPU_BL = 3, OMP_DT = 4 };

  // gDiamond/gdiamond.hpp:20-73: Nx*Ny*Nz grid, source at the centre cell, coefficients of a
  // vacuum box with a 10-cell graded pseudo-PML on every face.
  gDiamond(size_t Nx, size_t Ny, size_t Nz) : _Nx(Nx), _Ny(Ny), _Nz(Nz) {
    init_common();
    build_coefficients(nullptr);  // vacuum
  }

  // Per-cell relative permittivity (real part), same PML grading.
  gDiamond(size_t Nx, size_t Ny, size_t Nz, const float* eps_r) : _Nx(Nx), _Ny(Ny), _Nz(Nz) {
    init_common();
    build_coefficients(eps_r);
  }

  // Arbitrary per-cell coefficients: 12 arrays of Nx*Ny*Nz in the order
  // Cax Cay Caz Cbx Cby Cbz Dax Day Daz Dbx Dby Dbz.
  gDiamond(size_t Nx, size_t Ny, size_t Nz, const float* const coef[12])
      : _Nx(Nx), _Ny(Ny), _Nz(Nz) {
    init_common();
    for (int a = 0; a < 12; ++a) _coef[a].assign(coef[a], coef[a] + cells());
  }

  ~gDiamond() {
    if (_h) fdtd_destroy(_h);
  }
  gDiamond(const gDiamond&) = delete;
  gDiamond& operator=(const gDiamond&) = delete;

  // ------------------------------------------------------------------ CPU paths
  // gDiamond/gdiamond.hpp:1164-1263: T steps from zero fields, Mz = M_amp sin(omega t dt) at the
  // source cell, E sweep then H sweep over the interior.
  void update_FDTD_seq(size_t num_timesteps) { run_cpu(num_timesteps, SEQ, false); }

  // gDiamond/gdiamond_omp.hpp:110-172: the same with `omp parallel for collapse(2)`.
  void update_FDTD_omp(size_t num_timesteps) { run_cpu(num_timesteps, OMP, true); }

  // gDiamond/gdiamond_omp.hpp:174-261: the reference's temporally tiled OpenMP path, whose
  // results equal update_FDTD_seq.  Here each block of BLT steps advances as a wavefront along z,
  // in place: at wavefront position p, level s updates E of plane p-s+1 and then H of plane p-s,
  // each plane's rows split over the OpenMP threads, so only the BLT planes in flight need to
  // stay in cache.  Every cell sees the same operations in the same order as in seq (bit-equal
  // results).  blx, bly and blz are the reference's spatial tile sizes; the plane wavefront has
  // no spatial tiles, so they are accepted and not used.  Results -> OMP_DT.
  void update_FDTD_omp_dt(size_t blx, size_t bly, size_t blz, size_t blt, size_t num_timesteps) {
    (void)blx;
    (void)bly;
    (void)blz;
    if (blt < 1) throw std::invalid_argument("BLT must be >= 1");
    run_cpu_wavefront(num_timesteps, blt, OMP_DT);
  }

  // ------------------------------------------------------------------ GPU paths (C-ABI)
  // gDiamond/gdiamond_gpu.cuh:483-648: per-step Mz source; results -> GPU.
  void update_FDTD_gpu_2D(size_t num_timesteps) {
    run_gpu(num_timesteps, mz_wave(num_timesteps), GPU, FDTD_KERNEL_AUTO);
  }

  // gDiamond/gdiamond_gpu.cuh:809-950: the reference writes Mz T times before stepping, so the
  // whole run sees the constant value M_amp sin(omega (T-1) dt); kept for drop-in parity with
  // check_correctness_gpu().  Results -> GPU_BL.
  void update_FDTD_gpu_3D_warp_underutilization_fix(size_t num_timesteps) {
    run_gpu(num_timesteps, constant_mz_wave(num_timesteps), GPU_BL, FDTD_KERNEL_NAIVE);
  }

  // gDiamond/gdiamond_gpu_naive_vectorized.cuh:28-181 (same source convention as above).
  void update_FDTD_gpu_3D_warp_underutilization_fix_vectorized(size_t num_timesteps) {
    run_gpu(num_timesteps, constant_mz_wave(num_timesteps), GPU_BL, FDTD_KERNEL_AUTO);
  }

  // gDiamond/gdiamond_gpu_mm_ver2.cuh:837-1260 and gdiamond_gpu_mm_ver3.cuh:478-740: the tiled
  // paths; Tx, Ty, Tz only fixed the grid there (Nx = 27Tx+25 ... / Nx = 13Tx ...), any grid
  // works here.  Constant-source convention as in the reference.  Results -> GPU.
  void update_FDTD_mix_mapping_gpu_ver2(size_t num_timesteps, size_t, size_t, size_t) {
    run_gpu(num_timesteps, constant_mz_wave(num_timesteps), GPU, FDTD_KERNEL_TILED);
  }
  void update_FDTD_mix_mapping_gpu_ver3(size_t num_timesteps, size_t, size_t, size_t) {
    run_gpu(num_timesteps, constant_mz_wave(num_timesteps), GPU, FDTD_KERNEL_TILED);
  }

  // gDiamond/gdiamond_gpu.cuh:24-281 without the PNG output: Gaussian-modulated Jx at the source
  // cell, running DFT of Ex on the plane z = Nz/2 at 26 frequencies 0.90..1.15 f0, scale 50/T
  // (here in FP64).  Results -> GPU; the spectra via dft_real() / dft_imag().
  void update_FDTD_gpu_figures(size_t num_timesteps) {
    std::vector<float> w(num_timesteps);
    for (size_t t = 0; t < num_timesteps; ++t) {
      const float tt = (float)t * dt;
      w[t] = J_source_amp * std::exp(-((tt - t_peak) * (tt - t_peak)) / (2 * t_sigma * t_sigma)) *
             std::sin(SOURCE_OMEGA * (float)t * dt);
    }
    _freqs.clear();
    const float f0 = SOURCE_FREQUENCY;
    const float fs = 0.9f * f0, fe = 1.15f * f0, step = 0.01f * f0;
    const int nf = (int)((fe - fs) / step) + 1;
    for (int f = 0; f < nf; ++f) _freqs.push_back((double)(fs + f * step));
    fdtd_source s = {FDTD_JX, FDTD_SRC_POINT, (int64_t)(_Nx / 2), (int64_t)(_Ny / 2),
                     (int64_t)(_Nz / 2)};
    run_gpu_sources(num_timesteps, &s, 1, w, GPU, FDTD_KERNEL_AUTO, true,
                    50.0 / (double)num_timesteps);
    _fig_wave = std::move(w);
  }

  // ------------------------------------------------------------------ checks
  // gDiamond/gdiamond.hpp:1330-1505: element-wise |a - b| < 1e-8 on all six components.
  bool check_correctness_gpu_2D() const { return same(SEQ, GPU); }
  bool check_correctness_gpu() const { return same(GPU_BL, GPU); }
  bool check_correctness_omp() const { return same(SEQ, OMP); }
  bool check_correctness_omp_dt() const { return same(SEQ, OMP_DT); }

  // ------------------------------------------------------------------ accessors
  const std::vector<float>& field(Component c, Variant v) const { return _res[v][c]; }
  const std::vector<float>& coefficient(int a) const { return _coef[a]; }
  const std::vector<double>& dft_real() const { return _dft_re; }
  const std::vector<double>& dft_imag() const { return _dft_im; }
  const std::vector<double>& dft_freqs() const { return _freqs; }
  // The Jx waveform of the last update_FDTD_gpu_figures call (sample t used at step t).
  const std::vector<float>& figures_wave() const { return _fig_wave; }
  size_t source_idx() const { return _source_idx; }
  size_t Nx() const { return _Nx; }
  size_t Ny() const { return _Ny; }
  size_t Nz() const { return _Nz; }

  void print_results() const {
    for (int v : {SEQ, GPU}) {
      if (_res[v][0].empty()) continue;
      std::cout << (v == SEQ ? "Ex_seq" : "Ex_gpu") << " = \n";
      for (size_t k = 1; k + 1 < _Nz; k++)
        for (size_t j = 1; j + 1 < _Ny; j++)
          for (size_t i = 1; i + 1 < _Nx; i++) {
            const size_t idx = i + j * _Nx + k * (_Nx * _Ny);
            if (_res[v][0][idx] != 0)
              std::cout << "(x, y, z) = " << i << ", " << j << ", " << k << ", value = "
                        << _res[v][0][idx] << "\n";
          }
    }
  }

  // Reference constants (gDiamond/gdiamond.hpp:893-906; eps0 = mu0 = c0 = eta0 = 1).
  const float um = 1.0f;
  const float SOURCE_WAVELENGTH = 1.0f * um;
  const float SOURCE_FREQUENCY = 1.0f / SOURCE_WAVELENGTH;
  const float SOURCE_OMEGA = 2 * 3.14159265359f * SOURCE_FREQUENCY;
  const float _dx = SOURCE_WAVELENGTH / 10;
  const float dt = 0.05f;
  const float J_source_amp = 5e4f;
  const float M_source_amp = 5e4f;
  const float freq_sigma = (float)(0.05 * SOURCE_FREQUENCY);
  const float t_sigma = (float)(1 / freq_sigma / (2 * 3.14159265359f));
  const float t_peak = 5 * t_sigma;

 private:
  size_t cells() const { return _Nx * _Ny * _Nz; }

  void init_common() {
    if (_Nx < 3 || _Ny < 3 || _Nz < 3) throw std::invalid_argument("grid must be >= 3 per axis");
    _source_idx = _Nx / 2 + _Ny / 2 * _Nx + _Nz / 2 * _Nx * _Ny;
    _t_pml = (int)std::ceil(1.0f * um / _dx);
  }

  struct Cpx {
    float re, im;
  };
  static Cpx cmul(Cpx a, Cpx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
  static Cpx cdiv(Cpx a, Cpx b) {
    const float den = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / den, (a.im * b.re - a.re * b.im) / den};
  }
  // gDiamond/utils.h:585-619
  Cpx stretch(long i, long n, float sigma_max) const {
    float dist = 0;
    if (i < _t_pml) dist = (float)(1.0 - (double)((float)i / (float)_t_pml));
    if (i + _t_pml >= n) dist = (float)(1.0 - (double)((float)(int)(n - i - 1) / (float)_t_pml));
    const double d3 = std::pow((double)dist, 3.0);
    return {(float)(1.0 + 2.0 * d3), (float)((double)sigma_max * d3 / (double)(SOURCE_OMEGA * 1.0f))};
  }
  // gDiamond/utils.h:637-686
  void pair(Cpx m, float* ca, float* cb) const {
    float re = m.re;
    if (re < 1) re = 1;
    const float sigma = std::fabs(SOURCE_OMEGA * 1.0f * m.im);
    const float tmp = (float)((double)(sigma * dt) / (2.0 * (double)re * 1.0));
    *ca = (float)((1.0 - (double)tmp) / (1.0 + (double)tmp));
    *cb = (float)((double)(dt / (re * 1.0f)) / (1.0 + (double)tmp) / (double)_dx);
  }
  // gDiamond/utils.h:542-690 (set_FDTD_matrices_3D_structure, no mask)
  void build_coefficients(const float* eps_r) {
    for (auto& c : _coef) c.assign(cells(), 0.0f);
    const float denom = 2 * 1.0f * (float)_t_pml * _dx;
    const float sigma_max = (float)((double)(-4) * std::log(1e-5) / (double)denom);
    for (size_t k = 0; k < _Nz; ++k) {
      const Cpx sz = stretch((long)k, (long)_Nz, sigma_max);
      for (size_t j = 0; j < _Ny; ++j) {
        const Cpx sy = stretch((long)j, (long)_Ny, sigma_max);
        for (size_t i = 0; i < _Nx; ++i) {
          const Cpx sx = stretch((long)i, (long)_Nx, sigma_max);
          const size_t idx = i + j * _Nx + k * _Nx * _Ny;
          const Cpx eps = {eps_r ? eps_r[idx] : 1.0f, 0.0f};
          const Cpx mu = {1.0f, 0.0f};
          pair(cdiv(cmul(cmul(eps, sy), sz), sx), &_coef[0][idx], &_coef[3][idx]);
          pair(cdiv(cmul(cmul(eps, sx), sz), sy), &_coef[1][idx], &_coef[4][idx]);
          pair(cdiv(cmul(cmul(eps, sx), sy), sz), &_coef[2][idx], &_coef[5][idx]);
          pair(cdiv(cmul(cmul(mu, sy), sz), sx), &_coef[6][idx], &_coef[9][idx]);
          pair(cdiv(cmul(cmul(mu, sx), sz), sy), &_coef[7][idx], &_coef[10][idx]);
          pair(cdiv(cmul(cmul(mu, sx), sy), sz), &_coef[8][idx], &_coef[11][idx]);
        }
      }
    }
  }

  std::vector<float> mz_wave(size_t T) const {
    std::vector<float> w(T);
    for (size_t t = 0; t < T; ++t) w[t] = M_source_amp * std::sin(SOURCE_OMEGA * (float)t * dt);
    return w;
  }
  std::vector<float> constant_mz_wave(size_t T) const {
    const float v = T ? M_source_amp * std::sin(SOURCE_OMEGA * (float)(T - 1) * dt) : 0.0f;
    return std::vector<float>(T, v);
  }

  void run_cpu(size_t T, Variant v, bool parallel) {
    const size_t n = cells(), sx = 1, sy = _Nx, sz = _Nx * _Ny;
    std::vector<float> F[6];
    for (auto& f : F) f.assign(n, 0.0f);
    float *Ex_ = F[0].data(), *Ey_ = F[1].data(), *Ez_ = F[2].data();
    float *Hx_ = F[3].data(), *Hy_ = F[4].data(), *Hz_ = F[5].data();
    const float* C[12];
    for (int a = 0; a < 12; ++a) C[a] = _coef[a].data();
    const long Nx = (long)_Nx, Ny = (long)_Ny, Nz = (long)_Nz;
    for (size_t t = 0; t < T; ++t) {
      const float mz = M_source_amp * std::sin(SOURCE_OMEGA * (float)t * dt);
#pragma omp parallel for collapse(2) if (parallel)
      for (long k = 1; k < Nz - 1; k++)
        for (long j = 1; j < Ny - 1; j++)
          for (long i = 1; i < Nx - 1; i++) {
            const size_t idx = i + j * sy + k * sz;
            Ex_[idx] = C[0][idx] * Ex_[idx] + C[3][idx] * ((Hz_[idx] - Hz_[idx - sy]) - (Hy_[idx] - Hy_[idx - sz]));
            Ey_[idx] = C[1][idx] * Ey_[idx] + C[4][idx] * ((Hx_[idx] - Hx_[idx - sz]) - (Hz_[idx] - Hz_[idx - sx]));
            Ez_[idx] = C[2][idx] * Ez_[idx] + C[5][idx] * ((Hy_[idx] - Hy_[idx - sx]) - (Hx_[idx] - Hx_[idx - sy]));
          }
#pragma omp parallel for collapse(2) if (parallel)
      for (long k = 1; k < Nz - 1; k++)
        for (long j = 1; j < Ny - 1; j++)
          for (long i = 1; i < Nx - 1; i++) {
            const size_t idx = i + j * sy + k * sz;
            float cz = (Ex_[idx + sy] - Ex_[idx]) - (Ey_[idx + sx] - Ey_[idx]);
            if (idx == _source_idx) cz = cz - mz * _dx;
            Hx_[idx] = C[6][idx] * Hx_[idx] + C[9][idx] * ((Ey_[idx + sz] - Ey_[idx]) - (Ez_[idx + sy] - Ez_[idx]));
            Hy_[idx] = C[7][idx] * Hy_[idx] + C[10][idx] * ((Ez_[idx + sx] - Ez_[idx]) - (Ex_[idx + sz] - Ex_[idx]));
            Hz_[idx] = C[8][idx] * Hz_[idx] + C[11][idx] * cz;
          }
    }
    for (int c = 0; c < 6; ++c) _res[v][c] = std::move(F[c]);
  }

  // One plane of the E sweep / H sweep of run_cpu (rows split over OpenMP threads).
  void e_plane(std::vector<float>* F, long k) const {
    const long Nx = (long)_Nx, Ny = (long)_Ny;
    const size_t sx = 1, sy = _Nx, sz = _Nx * _Ny;
    float *Ex_ = F[0].data(), *Ey_ = F[1].data(), *Ez_ = F[2].data();
    const float *Hx_ = F[3].data(), *Hy_ = F[4].data(), *Hz_ = F[5].data();
    const float* const* C = _cptr;
#pragma omp parallel for
    for (long j = 1; j < Ny - 1; j++)
      for (long i = 1; i < Nx - 1; i++) {
        const size_t idx = i + j * sy + k * sz;
        Ex_[idx] = C[0][idx] * Ex_[idx] + C[3][idx] * ((Hz_[idx] - Hz_[idx - sy]) - (Hy_[idx] - Hy_[idx - sz]));
        Ey_[idx] = C[1][idx] * Ey_[idx] + C[4][idx] * ((Hx_[idx] - Hx_[idx - sz]) - (Hz_[idx] - Hz_[idx - sx]));
        Ez_[idx] = C[2][idx] * Ez_[idx] + C[5][idx] * ((Hy_[idx] - Hy_[idx - sx]) - (Hx_[idx] - Hx_[idx - sy]));
      }
  }
  void h_plane(std::vector<float>* F, long k, float mz) const {
    const long Nx = (long)_Nx, Ny = (long)_Ny;
    const size_t sx = 1, sy = _Nx, sz = _Nx * _Ny;
    const float *Ex_ = F[0].data(), *Ey_ = F[1].data(), *Ez_ = F[2].data();
    float *Hx_ = F[3].data(), *Hy_ = F[4].data(), *Hz_ = F[5].data();
    const float* const* C = _cptr;
#pragma omp parallel for
    for (long j = 1; j < Ny - 1; j++)
      for (long i = 1; i < Nx - 1; i++) {
        const size_t idx = i + j * sy + k * sz;
        float cz = (Ex_[idx + sy] - Ex_[idx]) - (Ey_[idx + sx] - Ey_[idx]);
        if (idx == _source_idx) cz = cz - mz * _dx;
        Hx_[idx] = C[6][idx] * Hx_[idx] + C[9][idx] * ((Ey_[idx + sz] - Ey_[idx]) - (Ez_[idx + sy] - Ez_[idx]));
        Hy_[idx] = C[7][idx] * Hy_[idx] + C[10][idx] * ((Ez_[idx + sx] - Ez_[idx]) - (Ex_[idx + sz] - Ex_[idx]));
        Hz_[idx] = C[8][idx] * Hz_[idx] + C[11][idx] * cz;
      }
  }

  // Blocks of blt steps as an in-place z-wavefront (see update_FDTD_omp_dt).  E(e) at level s
  // reads H(e) at level s-1 (updated earlier in this position by level s-1) and H(e-1) at level
  // s-1 (advanced to level s only after E(e), in the same position); H(e-1) at level s reads
  // E(e) and E(e-1) at level s (E(e-1) reaches level s+1 only after it).
  void run_cpu_wavefront(size_t T, size_t blt, Variant v) {
    const size_t n = cells();
    std::vector<float> F[6];
    for (auto& f : F) f.assign(n, 0.0f);
    for (int a = 0; a < 12; ++a) _cptr[a] = _coef[a].data();
    const long Nz = (long)_Nz;
    for (size_t t0 = 0; t0 < T; t0 += blt) {
      const long b = (long)std::min(blt, T - t0);
      for (long p = 1; p <= Nz - 2 + b; ++p)
        for (long s = 1; s <= b; ++s) {
          const long e = p - s + 1, h = p - s;
          if (e >= 1 && e <= Nz - 2) e_plane(F, e);
          if (h >= 1 && h <= Nz - 2) {
            const size_t t = t0 + (size_t)(s - 1);
            h_plane(F, h, M_source_amp * std::sin(SOURCE_OMEGA * (float)t * dt));
          }
        }
    }
    for (int c = 0; c < 6; ++c) _res[v][c] = std::move(F[c]);
  }

  void ensure_handle(int kernel) {
    if (_h && _h_kernel == kernel) return;
    if (_h) fdtd_destroy(_h);
    _h = nullptr;
    fdtd_desc d = {};
    d.nx = (int64_t)_Nx;
    d.ny = (int64_t)_Ny;
    d.nz = (int64_t)_Nz;
    d.dx = _dx;
    d.kernel = kernel;
    if (fdtd_create(&d, &_h) != FDTD_OK) throw std::runtime_error(fdtd_last_error(nullptr));
    _h_kernel = kernel;
    const float* c[12];
    for (int a = 0; a < 12; ++a) c[a] = _coef[a].data();
    check(fdtd_set_coefficients(_h, c));
  }

  void check(fdtd_status s) const {
    if (s != FDTD_OK) throw std::runtime_error(std::string("fdtd: ") + fdtd_last_error(_h));
  }

  void run_gpu(size_t T, const std::vector<float>& wave, Variant v, int kernel) {
    fdtd_source s = {FDTD_MZ, FDTD_SRC_POINT, (int64_t)(_Nx / 2), (int64_t)(_Ny / 2),
                     (int64_t)(_Nz / 2)};
    run_gpu_sources(T, &s, 1, wave, v, kernel, false, 0.0);
  }

  void run_gpu_sources(size_t T, const fdtd_source* s, int ns, const std::vector<float>& wave,
                       Variant v, int kernel, bool monitor, double scale) {
    ensure_handle(kernel);
    check(fdtd_reset(_h));
    check(fdtd_set_sources(_h, s, ns, wave.data(), (int64_t)std::max<size_t>(T, 1)));
    int32_t mid = -1;
    if (monitor) {
      if (_mon_id < 0)
        check(fdtd_add_dft_monitor(_h, FDTD_EX, (int64_t)(_Nz / 2), _freqs.data(),
                                   (int32_t)_freqs.size(), scale, (double)dt, &_mon_id));
      mid = _mon_id;
    }
    check(fdtd_step(_h, (int64_t)T, nullptr));
    check(fdtd_sync(_h));
    for (int c = 0; c < 6; ++c) {
      _res[v][c].resize(cells());
      check(fdtd_get_field(_h, c, _res[v][c].data()));
    }
    if (mid >= 0) {
      _dft_re.resize(_freqs.size() * _Nx * _Ny);
      _dft_im.resize(_freqs.size() * _Nx * _Ny);
      check(fdtd_get_dft(_h, mid, _dft_re.data(), _dft_im.data()));
    }
  }

  bool same(Variant a, Variant b) const {
    for (int c = 0; c < 6; ++c) {
      const auto& x = _res[a][c];
      const auto& y = _res[b][c];
      if (x.size() != cells() || y.size() != cells()) return false;
      for (size_t i = 0; i < cells(); ++i)
        if (std::fabs(x[i] - y[i]) >= 1e-8) return false;
    }
    return true;
  }

  size_t _Nx, _Ny, _Nz;
  size_t _source_idx = 0;
  int _t_pml = 10;
  std::vector<float> _coef[12];
  std::vector<float> _res[5][6];
  mutable const float* _cptr[12] = {};
  std::vector<double> _freqs, _dft_re, _dft_im;
  std::vector<float> _fig_wave;
  fdtd_handle* _h = nullptr;
  int _h_kernel = -1;
  int32_t _mon_id = -1;
};

}  // namespace gdiamond
