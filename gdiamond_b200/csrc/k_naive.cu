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

// grid (ceil(nx/32), ceil(ny/4), nz), block (32, 4)
template <bool kMat>
__global__ void __launch_bounds__(128) naive_e(Grid g, FieldPtrs F, CoefArrays A,
                                               const uint16_t* mat, const Material* tab,
                                               Sources S, long long t, float dx) {
  const int i = blockIdx.x * 32 + threadIdx.x;
  const int j = blockIdx.y * 4 + threadIdx.y;
  const int k = blockIdx.z;
  if (i < 1 || i > g.nx - 2 || j < 1 || j > g.ny - 2 || k < 1 || k > g.nz - 2) return;
  const long long sy = g.pitch, sz = g.plane;
  const long long idx = i + j * sy + k * sz;
  const float hx = F.f[3][idx], hy = F.f[4][idx], hz = F.f[5][idx];
  float cx = sub(sub(hz, F.f[5][idx - sy]), sub(hy, F.f[4][idx - sz]));
  float cy = sub(sub(hx, F.f[3][idx - sz]), sub(hz, F.f[5][idx - 1]));
  float cz = sub(sub(hy, F.f[4][idx - 1]), sub(hx, F.f[3][idx - sy]));
  if (S.n) {
    float v;
    if (source_value(S, 0, i, j, k, t, &v)) cx = sub(cx, mul(v, dx));
    if (source_value(S, 1, i, j, k, t, &v)) cy = sub(cy, mul(v, dx));
    if (source_value(S, 2, i, j, k, t, &v)) cz = sub(cz, mul(v, dx));
  }
  float ca[3], cb[3];
  load_e_coefs<kMat>(A, mat, tab, idx, ca, cb);
  F.f[0][idx] = yee(ca[0], F.f[0][idx], cb[0], cx);
  F.f[1][idx] = yee(ca[1], F.f[1][idx], cb[1], cy);
  F.f[2][idx] = yee(ca[2], F.f[2][idx], cb[2], cz);
}

template <bool kMat>
__global__ void __launch_bounds__(128) naive_h(Grid g, FieldPtrs F, CoefArrays A,
                                               const uint16_t* mat, const Material* tab,
                                               Sources S, long long t, float dx) {
  const int i = blockIdx.x * 32 + threadIdx.x;
  const int j = blockIdx.y * 4 + threadIdx.y;
  const int k = blockIdx.z;
  if (i < 1 || i > g.nx - 2 || j < 1 || j > g.ny - 2 || k < 1 || k > g.nz - 2) return;
  const long long sy = g.pitch, sz = g.plane;
  const long long idx = i + j * sy + k * sz;
  const float ex = F.f[0][idx], ey = F.f[1][idx], ez = F.f[2][idx];
  float cx = sub(sub(F.f[1][idx + sz], ey), sub(F.f[2][idx + sy], ez));
  float cy = sub(sub(F.f[2][idx + 1], ez), sub(F.f[0][idx + sz], ex));
  float cz = sub(sub(F.f[0][idx + sy], ex), sub(F.f[1][idx + 1], ey));
  if (S.n) {
    float v;
    if (source_value(S, 3, i, j, k, t, &v)) cx = sub(cx, mul(v, dx));
    if (source_value(S, 4, i, j, k, t, &v)) cy = sub(cy, mul(v, dx));
    if (source_value(S, 5, i, j, k, t, &v)) cz = sub(cz, mul(v, dx));
  }
  float da[3], db[3];
  load_h_coefs<kMat>(A, mat, tab, idx, da, db);
  F.f[3][idx] = yee(da[0], F.f[3][idx], db[0], cx);
  F.f[4][idx] = yee(da[1], F.f[4][idx], db[1], cy);
  F.f[5][idx] = yee(da[2], F.f[5][idx], db[2], cz);
}

// One thread per plane cell of every monitor: grid (ceil(nx/32), ceil(ny/8), nmon), block (32, 8)
__global__ void __launch_bounds__(256) naive_dft(Grid g, FieldPtrs F, Monitors M, long long t) {
  const int i = blockIdx.x * 32 + threadIdx.x;
  const int j = blockIdx.y * 8 + threadIdx.y;
  if (i >= g.nx || j >= g.ny || (int)blockIdx.z >= M.n) return;
  const MonitorDev& m = M.m[blockIdx.z];
  const float v = F.f[m.comp][i + (long long)j * g.pitch + (long long)m.k * g.plane];
  dft_accumulate(m, t, i, j, g, v);
}

cudaError_t launch_naive_step(const Grid& g, const FieldPtrs& F, const float* const* coef,
                              const uint16_t* mat, const Material* tab, const Sources& S,
                              const Monitors& M, long long t, float dx, cudaStream_t st,
                              int* launches) {
  CoefArrays A;
  for (int c = 0; c < 12; ++c) A.c[c] = coef ? coef[c] : nullptr;
  const dim3 blk(32, 4), grd((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz);
  if (mat) {
    naive_e<true><<<grd, blk, 0, st>>>(g, F, A, mat, tab, S, t, dx);
    naive_h<true><<<grd, blk, 0, st>>>(g, F, A, mat, tab, S, t, dx);
  } else {
    naive_e<false><<<grd, blk, 0, st>>>(g, F, A, mat, tab, S, t, dx);
    naive_h<false><<<grd, blk, 0, st>>>(g, F, A, mat, tab, S, t, dx);
  }
  *launches += 2;
  if (M.n) {
    const dim3 b2(32, 8), g2((g.nx + 31) / 32, (g.ny + 7) / 8, M.n);
    naive_dft<<<g2, b2, 0, st>>>(g, F, M, t);
    *launches += 1;
  }
  return cudaGetLastError();
}

}  // namespace fdtd
