// dft_fold.cu -- the deferred half of the running DFT monitors.
//
// The tiled kernels do not touch a monitor's FP64 sums: every step they write the monitor
// plane's FP32 values into slot t % kDftSlots of the monitor's staging ring (dft_record).  A fold
// adds a window of n <= kDftSlots consecutive steps to the sums:
//   re[f][p] += (v_t[p] * cos_t[f]) * scale,  im[f][p] -= (v_t[p] * sin_t[f]) * scale
// for t ascending, with separately rounded FP64 operations -- the same operations in the same
// order per (f, p) as accumulating once per step (the FP64 form of the reference's
// update_field_FFT_xy, kernels.cuh:87-113), so the sums are bit-identical to it.  What changes
// is the memory traffic: a step costs 4 bytes per monitor cell written and read back instead of
// a read-modify-write of 2 * nf doubles (1 KB at 32 frequencies), and the sums are read and
// written once per window.
//
// A thread owns one plane cell and kFoldF frequencies: their sums stay in registers for the
// whole window, the staged values of consecutive cells are coalesced, and the (cos, sin) table
// row of each step is a broadcast.
#include "fdtd_kernels.cuh"

namespace fdtd {

namespace {

constexpr int kFoldThreads = 128;
constexpr int kFoldF = 8;  // frequencies per thread

__device__ __forceinline__ void fold_monitor(const MonitorDev& m, const Grid& g, long long t0,
                                             int n) {
  const long long np = (long long)g.nx * g.ny;
  const long long p = (long long)blockIdx.x * kFoldThreads + threadIdx.x;
  const int f0 = (int)blockIdx.y * kFoldF;
  if (m.stage == nullptr || p >= np || f0 >= m.nf) return;
  const int nfc = min(kFoldF, m.nf - f0);
  double re[kFoldF], im[kFoldF];
#pragma unroll
  for (int q = 0; q < kFoldF; ++q) {
    re[q] = q < nfc ? m.re[(long long)(f0 + q) * np + p] : 0.0;
    im[q] = q < nfc ? m.im[(long long)(f0 + q) * np + p] : 0.0;
  }
  const float* st = m.stage + p;
  for (int s = 0; s < n; ++s) {
    const long long t = t0 + s;
    const double v = (double)st[(t & (kDftSlots - 1)) * np];
    const double2* tab = m.tab + t * m.nf + f0;
#pragma unroll
    for (int q = 0; q < kFoldF; ++q) {
      if (q < nfc) {
        const double2 cs = __ldg(&tab[q]);
        re[q] = dadd(re[q], dmul(dmul(v, cs.x), m.scale));
        im[q] = dsub(im[q], dmul(dmul(v, cs.y), m.scale));
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kFoldF; ++q) {
    if (q < nfc) {
      m.re[(long long)(f0 + q) * np + p] = re[q];
      m.im[(long long)(f0 + q) * np + p] = im[q];
    }
  }
}

// One grid: blockIdx.z is the monitor.
__global__ void __launch_bounds__(kFoldThreads) dft_fold(const __grid_constant__ Monitors M,
                                                         const Grid g, long long t0, int n) {
  if ((int)blockIdx.z < M.n) fold_monitor(M.m[blockIdx.z], g, t0, n);
}

// A batch: blockIdx.z is the grid; its arguments (monitors, step counter t0 at the start of the
// batch step) are the ones the batched kernel reads (TiledArgs, or CpmlSim for CPML batches).
// The window starts t_offset steps later.
template <class Args>
__global__ void __launch_bounds__(kFoldThreads) dft_fold_batch(const Args* grids,
                                                               long long t_offset, int n) {
  const Args& a = grids[blockIdx.z];
  for (int k = 0; k < a.M.n; ++k) fold_monitor(a.M.m[k], a.g, a.t0 + t_offset, n);
}

dim3 fold_grid(long long max_np, int max_nf, int nz) {
  return dim3((unsigned)((max_np + kFoldThreads - 1) / kFoldThreads),
              (unsigned)((max_nf + kFoldF - 1) / kFoldF), (unsigned)nz);
}

}  // namespace

cudaError_t launch_dft_fold(const Monitors& M, const Grid& g, long long t0, int n,
                            cudaStream_t st) {
  if (M.n <= 0 || n <= 0) return cudaSuccess;
  if (n > kDftSlots || t0 < 0) return cudaErrorInvalidValue;
  int max_nf = 0;
  for (int k = 0; k < M.n; ++k) max_nf = max_nf > M.m[k].nf ? max_nf : M.m[k].nf;
  dft_fold<<<fold_grid((long long)g.nx * g.ny, max_nf, M.n), kFoldThreads, 0, st>>>(M, g, t0, n);
  return cudaGetLastError();
}

cudaError_t launch_dft_fold_batch(const TiledArgs* grids, int ngrids, long long max_np,
                                  int max_nf, long long t_offset, int n, cudaStream_t st) {
  if (ngrids <= 0 || max_nf <= 0 || n <= 0) return cudaSuccess;
  if (n > kDftSlots || t_offset < 0 || ngrids > 65535) return cudaErrorInvalidValue;
  dft_fold_batch<TiledArgs>
      <<<fold_grid(max_np, max_nf, ngrids), kFoldThreads, 0, st>>>(grids, t_offset, n);
  return cudaGetLastError();
}

cudaError_t launch_dft_fold_cpml_batch(const CpmlSim* sims, int nsims, long long max_np,
                                       int max_nf, long long t_offset, int n, cudaStream_t st) {
  if (nsims <= 0 || max_nf <= 0 || n <= 0) return cudaSuccess;
  if (n > kDftSlots || t_offset < 0 || nsims > 65535) return cudaErrorInvalidValue;
  dft_fold_batch<CpmlSim>
      <<<fold_grid(max_np, max_nf, nsims), kFoldThreads, 0, st>>>(sims, t_offset, n);
  return cudaGetLastError();
}

}  // namespace fdtd
