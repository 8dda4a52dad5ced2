// The reference's unit tests (unittests/checker_gpu.cu, checker_omp.cpp, checker_omp_dt.cpp)
// and example checks
// (examples/gpu_mm_ver3.cu) written against include/gdiamond_compat.hpp.
//
//   compat_checker cpu Nx Ny Nz T [dump_prefix]   seq vs omp and vs omp_dt (BLT 5 and 3);
//                                                 optional raw dump of seq fields
//   compat_checker gpu Nx Ny Nz T [dump_prefix]   seq vs gpu_2D, 3D-fix vs mix-mapping ver3,
//                                                 ver3 vs the vectorized 3D-fix alias,
//                                                 the figures path (Jx + Ex DFT); with
//                                                 dump_prefix, its waveform, frequencies,
//                                                 DFT sums and coefficients as raw files
// Prints one JSON object; exit code 0 when every check holds.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>

#include "gdiamond_compat.hpp"

template <class T>
static void dump(const std::string& path, const std::vector<T>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), v.size() * sizeof(T));
}

static double l2(const std::vector<float>& v) {
  double s = 0;
  for (float x : v) s += (double)x * x;
  return std::sqrt(s);
}

int main(int argc, char** argv) {
  if (argc < 6) {
    std::fprintf(stderr, "usage: compat_checker cpu|gpu Nx Ny Nz T [dump_prefix]\n");
    return 2;
  }
  const std::string mode = argv[1];
  const size_t Nx = std::atoi(argv[2]), Ny = std::atoi(argv[3]), Nz = std::atoi(argv[4]);
  const size_t T = std::atoi(argv[5]);
  gdiamond::gDiamond exp(Nx, Ny, Nz);
  exp.update_FDTD_seq(T);
  bool ok = true;
  std::printf("{\"mode\": \"%s\"", mode.c_str());
  std::printf(", \"seq_l2\": [");
  for (int c = 0; c < 6; ++c)
    std::printf("%s%.17g", c ? ", " : "", l2(exp.field((gdiamond::gDiamond::Component)c, gdiamond::gDiamond::SEQ)));
  std::printf("]");
  if (argc > 6) {
    for (int c = 0; c < 6; ++c) {
      std::ofstream f(std::string(argv[6]) + std::to_string(c) + ".bin", std::ios::binary);
      const auto& v = exp.field((gdiamond::gDiamond::Component)c, gdiamond::gDiamond::SEQ);
      f.write(reinterpret_cast<const char*>(v.data()), v.size() * sizeof(float));
    }
  }
  if (mode == "cpu") {
    exp.update_FDTD_omp(T);
    const bool omp_ok = exp.check_correctness_omp();
    exp.update_FDTD_omp_dt(16, 16, 16, 5, T);
    const bool dt_ok = exp.check_correctness_omp_dt();
    exp.update_FDTD_omp_dt(16, 16, 16, 3, T);
    const bool dt3_ok = exp.check_correctness_omp_dt();
    ok = ok && omp_ok && dt_ok && dt3_ok;
    std::printf(", \"omp_matches_seq\": %s, \"omp_dt_matches_seq\": %s",
                omp_ok ? "true" : "false", dt_ok && dt3_ok ? "true" : "false");
  } else {
    exp.update_FDTD_gpu_2D(T);
    const bool g2 = exp.check_correctness_gpu_2D();
    exp.update_FDTD_gpu_3D_warp_underutilization_fix(T);
    exp.update_FDTD_mix_mapping_gpu_ver3(T, 0, 0, 0);
    const bool g3 = exp.check_correctness_gpu();
    // the float4 naive path's drop-in (gDiamond/gdiamond_gpu_naive_vectorized.cuh:28-181)
    // writes the 3D-fix results, so ver3 vs it is the same check again
    exp.update_FDTD_gpu_3D_warp_underutilization_fix_vectorized(T);
    const bool gv = exp.check_correctness_gpu();
    exp.update_FDTD_gpu_figures(T);
    double dmax = 0;
    for (double v : exp.dft_real()) dmax = std::max(dmax, std::fabs(v));
    const bool figs = exp.dft_freqs().size() == 26 && dmax > 0 && std::isfinite(dmax);
    if (argc > 6) {
      const std::string pre = argv[6];
      dump(pre + "fig_wave.bin", exp.figures_wave());
      dump(pre + "fig_freqs.bin", exp.dft_freqs());
      dump(pre + "fig_re.bin", exp.dft_real());
      dump(pre + "fig_im.bin", exp.dft_imag());
      for (int a = 0; a < 12; ++a) dump(pre + "coef" + std::to_string(a) + ".bin", exp.coefficient(a));
    }
    ok = ok && g2 && g3 && gv && figs;
    std::printf(", \"gpu_2D_matches_seq\": %s, \"ver3_matches_3D_fix\": %s, "
                "\"vectorized_matches_ver3\": %s, \"figures_nf\": %zu, \"figures_dft_max\": %.17g",
                g2 ? "true" : "false", g3 ? "true" : "false", gv ? "true" : "false",
                exp.dft_freqs().size(), dmax);
  }
  std::printf(", \"ok\": %s}\n", ok ? "true" : "false");
  return ok ? 0 : 1;
}
