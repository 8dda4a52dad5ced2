// flux.cu -- Poynting flux through a z-plane from running DFTs of the tangential fields.
//
// The reference has only a per-cell running DFT of one component (update_field_FFT_xy,
// gDiamond/kernels.cuh:87-113).  A flux monitor on the E plane z = k keeps six such DFTs:
// Ex and Ey on plane k, and Hx and Hy on planes k-1 and k (their z positions k - 1/2 and
// k + 1/2 average to k), the H ones phased at (t + 1/2) dt because H of step t is half a step
// later than E of step t in the Yee scheme.  In the plane, Ex and Hy share the point
// (i + 1/2, j) and Ey and Hx the point (i, j + 1/2), so no in-plane interpolation is needed:
//
//   flux(f) = dx^2 * sum over cells of Re[ Ex conj(Hy) - Ey conj(Hx) ],  H = (H(k-1) + H(k)) / 2
//
// with X(f) = sum_t x(t) exp(-i w t') as accumulated by the monitors.  One CTA per frequency
// reduces the plane in FP64 in a fixed order (per-thread strided sums, then a tree), so the
// result is the same on every run.
#include "fdtd_kernels.cuh"

namespace fdtd {

namespace {

constexpr int kFluxThreads = 256;

__global__ void __launch_bounds__(kFluxThreads)
    flux_reduce(FluxPlanes p, long long np, double area, double* out) {
  __shared__ double part[kFluxThreads];
  const int f = blockIdx.x;
  const long long o = (long long)f * np;
  double acc = 0.0;
  for (long long q = threadIdx.x; q < np; q += kFluxThreads) {
    const long long i = o + q;
    const double hyr = 0.5 * (p.hy0_re[i] + p.hy1_re[i]), hyi = 0.5 * (p.hy0_im[i] + p.hy1_im[i]);
    const double hxr = 0.5 * (p.hx0_re[i] + p.hx1_re[i]), hxi = 0.5 * (p.hx0_im[i] + p.hx1_im[i]);
    const double sxy = p.ex_re[i] * hyr + p.ex_im[i] * hyi;  // Re(Ex conj(Hy))
    const double syx = p.ey_re[i] * hxr + p.ey_im[i] * hxi;  // Re(Ey conj(Hx))
    acc += sxy - syx;
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int s = kFluxThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[f] = part[0] * area;
}

}  // namespace

cudaError_t launch_flux_reduce(const FluxPlanes& p, long long np, int nf, double area,
                               double* out_dev, cudaStream_t st) {
  if (nf < 1) return cudaErrorInvalidValue;
  flux_reduce<<<nf, kFluxThreads, 0, st>>>(p, np, area, out_dev);
  return cudaGetLastError();
}

}  // namespace fdtd
