// Test infrastructure only: a C-callable wrapper around the REFERENCE's own CPU solvers.
//
// This file compiles gDiamond's headers where they lie (the include path is given by
// oracle/Makefile); nothing of the reference is copied here.  The product never links it:
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm load the
// resulting oracle/_ref/libgdref.so.
//
// Wrapped reference entry points:
//   gdiamond::gDiamond::gDiamond(Nx,Ny,Nz)        gDiamond/gdiamond.hpp:20-73
//   gdiamond::gDiamond::update_FDTD_seq(T)        gDiamond/gdiamond.hpp:1164-1263
//   gdiamond::gDiamond::update_FDTD_omp(T)        gDiamond/gdiamond_omp.hpp:110-172
//   gdiamond::gDiamond::update_FDTD_omp_dt(...)   gDiamond/gdiamond_omp.hpp:174-261
//   save_field_png(u, filename, Nx, Ny, vmax)     gDiamond/utils.h:210-255
//
// Two harness workarounds (both needed to run the reference as shipped):
//   1. the standard headers are included before `#define private public`, which otherwise
//      breaks libstdc++;
//   2. the `_E*_omp` / `_E*_omp_dt` result vectors are resized before omp / omp_dt run; the
//      reference leaves them zero-sized (their initialisers are commented out at
//      gDiamond/gdiamond.hpp:37-40), so its own omp checkers write out of bounds.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <map>
#include <random>
#include <set>
#include <sstream>
#include <string>
#include <utility>
#include <vector>
#include <omp.h>

#define private public
#include "gdiamond_omp.hpp"
#undef private

namespace {

using gdiamond::gDiamond;

std::vector<float>* field_vec(gDiamond* g, int variant, int comp) {
  // variant: 0 = seq, 1 = omp, 2 = omp_dt ; comp: Ex Ey Ez Hx Hy Hz
  std::vector<float>* tab[3][6] = {
      {&g->_Ex_seq, &g->_Ey_seq, &g->_Ez_seq, &g->_Hx_seq, &g->_Hy_seq, &g->_Hz_seq},
      {&g->_Ex_omp, &g->_Ey_omp, &g->_Ez_omp, &g->_Hx_omp, &g->_Hy_omp, &g->_Hz_omp},
      {&g->_Ex_omp_dt, &g->_Ey_omp_dt, &g->_Ez_omp_dt, &g->_Hx_omp_dt, &g->_Hy_omp_dt,
       &g->_Hz_omp_dt}};
  return tab[variant][comp];
}

void resize_variant(gDiamond* g, int variant) {
  const size_t n = g->_Nx * g->_Ny * g->_Nz;
  for (int c = 0; c < 6; ++c) field_vec(g, variant, c)->assign(n, 0.0f);
}

double seconds_since(std::chrono::high_resolution_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
}

// The time the reference prints for its own loop ("... runtime: <s>s") during the last run.
double g_printed = -1.0;

// Runs f with std::cout captured, keeps the printed runtime, and echoes the text.
template <typename F>
void capture_printed(F f) {
  std::ostringstream cap;
  std::streambuf* old = std::cout.rdbuf(cap.rdbuf());
  f();
  std::cout.rdbuf(old);
  const std::string text = cap.str();
  g_printed = -1.0;
  const size_t at = text.find("runtime: ");
  if (at != std::string::npos) g_printed = std::strtod(text.c_str() + at + 9, nullptr);
  std::cout << text << std::flush;
}

}  // namespace

extern "C" {

void* gdref_create(size_t nx, size_t ny, size_t nz) { return new gDiamond(nx, ny, nz); }

void gdref_destroy(void* h) { delete static_cast<gDiamond*>(h); }

// Copies the 12 coefficient arrays in the order Cax Cay Caz Cbx Cby Cbz Dax Day Daz Dbx Dby Dbz.
void gdref_get_coefficients(void* h, float* const* out12) {
  gDiamond* g = static_cast<gDiamond*>(h);
  const std::vector<float>* src[12] = {&g->_Cax, &g->_Cay, &g->_Caz, &g->_Cbx, &g->_Cby, &g->_Cbz,
                                       &g->_Dax, &g->_Day, &g->_Daz, &g->_Dbx, &g->_Dby, &g->_Dbz};
  for (int a = 0; a < 12; ++a) std::memcpy(out12[a], src[a]->data(), src[a]->size() * sizeof(float));
}

size_t gdref_source_idx(void* h) { return static_cast<gDiamond*>(h)->_source_idx; }

// dx, dt, J amplitude, M amplitude, source omega, t_sigma, t_peak (all as the reference stores them).
void gdref_params(void* h, float* out7) {
  gDiamond* g = static_cast<gDiamond*>(h);
  out7[0] = g->_dx;
  out7[1] = g->dt;
  out7[2] = g->J_source_amp;
  out7[3] = g->M_source_amp;
  out7[4] = g->SOURCE_OMEGA;
  out7[5] = g->t_sigma;
  out7[6] = g->t_peak;
}

// Each runner returns the wall time of the whole reference call (allocation of its temporaries,
// the time loop and the copy-out included).
double gdref_run_seq(void* h, size_t T) {
  auto t0 = std::chrono::high_resolution_clock::now();
  capture_printed([&] { static_cast<gDiamond*>(h)->update_FDTD_seq(T); });
  return seconds_since(t0);
}

double gdref_run_omp(void* h, size_t T) {
  gDiamond* g = static_cast<gDiamond*>(h);
  resize_variant(g, 1);
  auto t0 = std::chrono::high_resolution_clock::now();
  capture_printed([&] { g->update_FDTD_omp(T); });
  return seconds_since(t0);
}

double gdref_run_omp_dt(void* h, size_t blx, size_t bly, size_t blz, size_t blt, size_t T) {
  gDiamond* g = static_cast<gDiamond*>(h);
  resize_variant(g, 2);
  auto t0 = std::chrono::high_resolution_clock::now();
  capture_printed([&] { g->update_FDTD_omp_dt(blx, bly, blz, blt, T); });
  return seconds_since(t0);
}

// variant: 0 = seq, 1 = omp, 2 = omp_dt.  out6 = Ex Ey Ez Hx Hy Hz, Nx*Ny*Nz floats each.
int gdref_get_fields(void* h, int variant, float* const* out6) {
  gDiamond* g = static_cast<gDiamond*>(h);
  if (variant < 0 || variant > 2) return -1;
  const size_t n = g->_Nx * g->_Ny * g->_Nz;
  for (int c = 0; c < 6; ++c) {
    std::vector<float>* v = field_vec(g, variant, c);
    if (v->size() != n) return -2;
    std::memcpy(out6[c], v->data(), n * sizeof(float));
  }
  return 0;
}

int gdref_max_threads(void) { return omp_get_max_threads(); }

// The runtime the reference printed for its own time loop in the last gdref_run_* call (its
// chrono clock around the loop only), or -1 when it printed none.
double gdref_last_printed_seconds(void) { return g_printed; }

// The reference's field-slice PNG writer (blue-white-red map clipped to +-vmax).
void gdref_save_field_png(const float* u, const char* filename, int nx, int ny, float vmax) {
  save_field_png(const_cast<float*>(u), filename, nx, ny, vmax);
}

}  // extern "C"
