// coefs.cu -- gDiamond's coefficient formula evaluated on the GPU.
//
// gDiamond's constructor fills 12 per-cell arrays on the host with set_FDTD_matrices_3D_structure
// (gDiamond/utils.h:542-690): complex stretch factors s = 1 + a d^3 + j sigma d^3 / omega0 in a
// graded shell of t_pml cells, eps_xx = Re((eps * sy * sz) / sx) (clamped to >= 1), and
// Ca = (1 - tmp) / (1 + tmp), Cb = (dt / eps) / (1 + tmp) / dx with tmp = sigma dt / (2 eps).
// Here the per-axis stretch factors (3 short vectors, computed on the host with the C library's
// pow as the reference does) are uploaded and every cell's 12 coefficients are computed by one
// thread, with the reference's operation order and its float/double promotions, each operation
// separately rounded -- so the arrays are bit-identical to the reference's.
#include "fdtd_kernels.cuh"

namespace fdtd {
namespace {

struct Cpx {
  float re, im;
};

__device__ __forceinline__ Cpx cmul(Cpx a, Cpx b) {
  return {__fsub_rn(__fmul_rn(a.re, b.re), __fmul_rn(a.im, b.im)),
          __fadd_rn(__fmul_rn(a.re, b.im), __fmul_rn(a.im, b.re))};
}

__device__ __forceinline__ Cpx cdiv(Cpx a, Cpx b) {
  const float den = __fadd_rn(__fmul_rn(b.re, b.re), __fmul_rn(b.im, b.im));
  return {__fdiv_rn(__fadd_rn(__fmul_rn(a.re, b.re), __fmul_rn(a.im, b.im)), den),
          __fdiv_rn(__fsub_rn(__fmul_rn(a.im, b.re), __fmul_rn(a.re, b.im)), den)};
}

// (Ca, Cb) of one axis from its complex material value (gDiamond/utils.h:637-686).
__device__ __forceinline__ void c_pair(Cpx m, float omega0, float dt, float dx, float* ca,
                                       float* cb) {
  float re = m.re;
  if (re < 1.0f) re = 1.0f;
  const float sigma = fabsf(__fmul_rn(__fmul_rn(omega0, 1.0f), m.im));
  const float tmp =
      __double2float_rn(__ddiv_rn((double)__fmul_rn(sigma, dt), __dmul_rn(__dmul_rn(2.0, (double)re), 1.0)));
  const double t = (double)tmp;
  *ca = __double2float_rn(__ddiv_rn(__dsub_rn(1.0, t), __dadd_rn(1.0, t)));
  *cb = __double2float_rn(
      __ddiv_rn(__ddiv_rn((double)__fdiv_rn(dt, __fmul_rn(re, 1.0f)), __dadd_rn(1.0, t)),
                (double)dx));
}

// One thread per cell of row (j, k); out12 are pitched per-cell arrays.
__global__ void coefficients_kernel(Grid g, const float* eps, const float2* sx, const float2* sy,
                                    const float2* sz, float omega0, float dt, float dx,
                                    Coef12Out out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const long long lin = i + (long long)j * g.nx + (long long)k * g.nx * g.ny;
  const long long idx = i + (long long)j * g.pitch + (long long)k * g.plane;
  const Cpx X = {sx[i].x, sx[i].y}, Y = {sy[j].x, sy[j].y}, Z = {sz[k].x, sz[k].y};
  const Cpx e = {eps ? eps[lin] : 1.0f, 0.0f};
  const Cpx mu = {1.0f, 0.0f};
  c_pair(cdiv(cmul(cmul(e, Y), Z), X), omega0, dt, dx, &out.c[0][idx], &out.c[3][idx]);
  c_pair(cdiv(cmul(cmul(e, X), Z), Y), omega0, dt, dx, &out.c[1][idx], &out.c[4][idx]);
  c_pair(cdiv(cmul(cmul(e, X), Y), Z), omega0, dt, dx, &out.c[2][idx], &out.c[5][idx]);
  c_pair(cdiv(cmul(cmul(mu, Y), Z), X), omega0, dt, dx, &out.c[6][idx], &out.c[9][idx]);
  c_pair(cdiv(cmul(cmul(mu, X), Z), Y), omega0, dt, dx, &out.c[7][idx], &out.c[10][idx]);
  c_pair(cdiv(cmul(cmul(mu, X), Y), Z), omega0, dt, dx, &out.c[8][idx], &out.c[11][idx]);
}

}  // namespace

cudaError_t build_coefficients(const Grid& g, const float* eps_dev, const float2* sx,
                               const float2* sy, const float2* sz, float omega0, float dt,
                               float dx, const Coef12Out& out, cudaStream_t st) {
  const dim3 blk(128), grd((g.nx + 127) / 128, g.ny, g.nz);
  coefficients_kernel<<<grd, blk, 0, st>>>(g, eps_dev, sx, sy, sz, omega0, dt, dx, out);
  return cudaGetLastError();
}

}  // namespace fdtd
