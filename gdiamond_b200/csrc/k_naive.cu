// k_naive.cu -- one thread per cell, separate E and H launches per step, in place.
//
// The B200 counterpart of the reference's naive GPU kernels updateE_3Dmap_fix /
// updateH_3Dmap_fix (gDiamond/kernels.cuh:337-394) and of the per-step DFT kernel
// update_field_FFT_xy (gDiamond/kernels.cuh:87-113).  Differences by design: the pitched
// layout, per-step source values read from a device waveform table (no per-step memcpy), FP64
// monitor sums, and the coefficients read either from 12 per-cell arrays or from a material
// map + table.  Every multiply/add is separately rounded, so results are bit-identical to the
// reference's CPU update.
#include "fdtd_kernels.cuh"

namespace fdtd {

struct CoefArrays {
  const float* c[12];  // pitched per-cell arrays, Cax Cay Caz Cbx Cby Cbz Dax Day Daz Dbx Dby Dbz
};

template <bool kMat>
__device__ __forceinline__ void load_e_coefs(const CoefArrays& A, const uint16_t* mat,
                                             const Material* tab, long long idx, float* ca,
                                             float* cb) {
  if (kMat) {
    const Material m = tab[mat[idx]];
    ca[0] = m.a.x; cb[0] = m.a.y; ca[1] = m.a.z; cb[1] = m.a.w; ca[2] = m.b.x; cb[2] = m.b.y;
  } else {
    for (int c = 0; c < 3; ++c) {
      ca[c] = A.c[c][idx];
      cb[c] = A.c[3 + c][idx];
    }
  }
}

template <bool kMat>
__device__ __forceinline__ void load_h_coefs(const CoefArrays& A, const uint16_t* mat,
                                             const Material* tab, long long idx, float* da,
                                             float* db) {
  if (kMat) {
    const Material m = tab[mat[idx]];
    da[0] = m.b.z; db[0] = m.b.w; da[1] = m.c.x; db[1] = m.c.y; da[2] = m.c.z; db[2] = m.c.w;
  } else {
    for (int c = 0; c < 3; ++c) {
      da[c] = A.c[6 + c][idx];
      db[c] = A.c[9 + c][idx];
    }
  }
}

// Arithmetic of one field type, every operation separately rounded.
template <typename T>
struct Arith;
template <>
struct Arith<float> {
  __device__ static float sub(float a, float b) { return __fsub_rn(a, b); }
  __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
  __device__ static float add(float a, float b) { return __fadd_rn(a, b); }
};
template <>
struct Arith<double> {
  __device__ static double sub(double a, double b) { return __dsub_rn(a, b); }
  __device__ static double mul(double a, double b) { return __dmul_rn(a, b); }
  __device__ static double add(double a, double b) { return __dadd_rn(a, b); }
};

// Source term in type T: the FP32 waveform samples of all covering sources summed in T.
template <typename T>
__device__ __forceinline__ bool source_value_t(const Sources& S, int comp, int i, int j, int k,
                                               long long t, T* v) {
  T acc = 0;
  bool any = false;
  for (int n = 0; n < S.n; ++n) {
    const SourceDev& s = S.s[n];
    if (s.comp != comp) continue;
    const bool hit = (s.kind == 0) ? (s.i == i && s.j == j && s.k == k) : (s.k == k);
    if (hit) {
      acc = Arith<T>::add(acc, (T)(t < S.tw ? S.wave[n * S.tw + t] : 0.0f));
      any = true;
    }
  }
  *v = acc;
  return any;
}

// grid (ceil(nx/32), ceil(ny/4), nz), block (32, 4).  T = float or double (FP64 storage: the
// error reference of reduced-precision runs; coefficients and waveforms are widened).
template <typename T, bool kMat>
__global__ void __launch_bounds__(128) naive_e(Grid g, FieldPtrs Fp, CoefArrays A,
                                               const uint16_t* mat, const Material* tab,
                                               Sources S, long long t, float dx_f) {
  using R = Arith<T>;
  T* const* F = reinterpret_cast<T* const*>(Fp.f);
  const int i = blockIdx.x * 32 + threadIdx.x;
  const int j = blockIdx.y * 4 + threadIdx.y;
  const int k = blockIdx.z;
  if (i < 1 || i > g.nx - 2 || j < 1 || j > g.ny - 2 || k < 1 || k > g.nz - 2) return;
  const long long sy = g.pitch, sz = g.plane;
  const long long idx = i + j * sy + k * sz;
  const T dx = (T)dx_f;
  const T hx = F[3][idx], hy = F[4][idx], hz = F[5][idx];
  T cx = R::sub(R::sub(hz, F[5][idx - sy]), R::sub(hy, F[4][idx - sz]));
  T cy = R::sub(R::sub(hx, F[3][idx - sz]), R::sub(hz, F[5][idx - 1]));
  T cz = R::sub(R::sub(hy, F[4][idx - 1]), R::sub(hx, F[3][idx - sy]));
  if (S.n) {
    T v;
    if (source_value_t<T>(S, 0, i, j, k, t, &v)) cx = R::sub(cx, R::mul(v, dx));
    if (source_value_t<T>(S, 1, i, j, k, t, &v)) cy = R::sub(cy, R::mul(v, dx));
    if (source_value_t<T>(S, 2, i, j, k, t, &v)) cz = R::sub(cz, R::mul(v, dx));
  }
  float ca[3], cb[3];
  load_e_coefs<kMat>(A, mat, tab, idx, ca, cb);
  F[0][idx] = R::add(R::mul((T)ca[0], F[0][idx]), R::mul((T)cb[0], cx));
  F[1][idx] = R::add(R::mul((T)ca[1], F[1][idx]), R::mul((T)cb[1], cy));
  F[2][idx] = R::add(R::mul((T)ca[2], F[2][idx]), R::mul((T)cb[2], cz));
}

template <typename T, bool kMat>
__global__ void __launch_bounds__(128) naive_h(Grid g, FieldPtrs Fp, CoefArrays A,
                                               const uint16_t* mat, const Material* tab,
                                               Sources S, long long t, float dx_f) {
  using R = Arith<T>;
  T* const* F = reinterpret_cast<T* const*>(Fp.f);
  const int i = blockIdx.x * 32 + threadIdx.x;
  const int j = blockIdx.y * 4 + threadIdx.y;
  const int k = blockIdx.z;
  if (i < 1 || i > g.nx - 2 || j < 1 || j > g.ny - 2 || k < 1 || k > g.nz - 2) return;
  const long long sy = g.pitch, sz = g.plane;
  const long long idx = i + j * sy + k * sz;
  const T dx = (T)dx_f;
  const T ex = F[0][idx], ey = F[1][idx], ez = F[2][idx];
  T cx = R::sub(R::sub(F[1][idx + sz], ey), R::sub(F[2][idx + sy], ez));
  T cy = R::sub(R::sub(F[2][idx + 1], ez), R::sub(F[0][idx + sz], ex));
  T cz = R::sub(R::sub(F[0][idx + sy], ex), R::sub(F[1][idx + 1], ey));
  if (S.n) {
    T v;
    if (source_value_t<T>(S, 3, i, j, k, t, &v)) cx = R::sub(cx, R::mul(v, dx));
    if (source_value_t<T>(S, 4, i, j, k, t, &v)) cy = R::sub(cy, R::mul(v, dx));
    if (source_value_t<T>(S, 5, i, j, k, t, &v)) cz = R::sub(cz, R::mul(v, dx));
  }
  float da[3], db[3];
  load_h_coefs<kMat>(A, mat, tab, idx, da, db);
  F[3][idx] = R::add(R::mul((T)da[0], F[3][idx]), R::mul((T)db[0], cx));
  F[4][idx] = R::add(R::mul((T)da[1], F[4][idx]), R::mul((T)db[1], cy));
  F[5][idx] = R::add(R::mul((T)da[2], F[5][idx]), R::mul((T)db[2], cz));
}

// One thread per plane cell of every monitor: grid (ceil(nx/32), ceil(ny/8), nmon), block (32, 8)
template <typename T>
__global__ void __launch_bounds__(256) naive_dft(Grid g, FieldPtrs Fp, Monitors M, long long t) {
  T* const* F = reinterpret_cast<T* const*>(Fp.f);
  const int i = blockIdx.x * 32 + threadIdx.x;
  const int j = blockIdx.y * 8 + threadIdx.y;
  if (i >= g.nx || j >= g.ny || (int)blockIdx.z >= M.n) return;
  const MonitorDev& m = M.m[blockIdx.z];
  const double v = (double)F[m.comp][i + (long long)j * g.pitch + (long long)m.k * g.plane];
  const double2* tab = m.tab + t * m.nf;
  const long long np = (long long)g.nx * g.ny;
  const long long p = i + (long long)j * g.nx;
  for (int f = 0; f < m.nf; ++f) {
    const double2 cs = tab[f];
    double* re = m.re + f * np + p;
    double* im = m.im + f * np + p;
    *re = dadd(*re, dmul(dmul(v, cs.x), m.scale));
    *im = dsub(*im, dmul(dmul(v, cs.y), m.scale));
  }
}

template <typename T>
void naive_step_t(const Grid& g, const FieldPtrs& F, const CoefArrays& A, const uint16_t* mat,
                  const Material* tab, const Sources& S, const Monitors& M, long long t, float dx,
                  cudaStream_t st, int* launches) {
  const dim3 blk(32, 4), grd((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz);
  if (mat) {
    naive_e<T, true><<<grd, blk, 0, st>>>(g, F, A, mat, tab, S, t, dx);
    naive_h<T, true><<<grd, blk, 0, st>>>(g, F, A, mat, tab, S, t, dx);
  } else {
    naive_e<T, false><<<grd, blk, 0, st>>>(g, F, A, mat, tab, S, t, dx);
    naive_h<T, false><<<grd, blk, 0, st>>>(g, F, A, mat, tab, S, t, dx);
  }
  *launches += 2;
  if (M.n) {
    const dim3 b2(32, 8), g2((g.nx + 31) / 32, (g.ny + 7) / 8, M.n);
    naive_dft<T><<<g2, b2, 0, st>>>(g, F, M, t);
    *launches += 1;
  }
}

cudaError_t launch_naive_dft(const Grid& g, const FieldPtrs& F, const Monitors& M, long long t,
                             cudaStream_t st, int* launches) {
  if (M.n == 0) return cudaSuccess;
  const dim3 b2(32, 8), g2((g.nx + 31) / 32, (g.ny + 7) / 8, M.n);
  naive_dft<float><<<g2, b2, 0, st>>>(g, F, M, t);
  *launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_naive_step(const Grid& g, const FieldPtrs& F, const float* const* coef,
                              const uint16_t* mat, const Material* tab, const Sources& S,
                              const Monitors& M, long long t, float dx, cudaStream_t st,
                              int* launches, bool fp64) {
  CoefArrays A;
  for (int c = 0; c < 12; ++c) A.c[c] = coef ? coef[c] : nullptr;
  if (fp64)
    naive_step_t<double>(g, F, A, mat, tab, S, M, t, dx, st, launches);
  else
    naive_step_t<float>(g, F, A, mat, tab, S, M, t, dx, st, launches);
  return cudaGetLastError();
}

}  // namespace fdtd
