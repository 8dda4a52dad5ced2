// cpml.cu -- convolutional PML (CPML) absorbing layers: per-step E and H kernels with the
// auxiliary psi fields of the layers.
//
// The reference absorbs with a graded pseudo-PML folded into Ca/Cb/Da/Db (a real-valued
// stretch, gDiamond/utils.h:585-660) in front of PEC faces that are never updated
// (gDiamond/gdiamond.hpp:1193-1221); outgoing waves are partly reflected.  A CPML layer instead
// replaces each spatial difference d in the curl by d / kappa + psi, with the recursive
// convolution psi <- b psi + a d (complex-frequency-shifted stretch s = kappa + sigma /
// (alpha + i w), in the normalised units of the reference: eps0 = mu0 = c = 1):
//
//   Ex <- Ca Ex + Cb [ (dyHz/ky + psi_exy) - (dzHy/kz + psi_exz) - Jx dx ],   dyHz = Hz(j) - Hz(j-1)
//
// and likewise for the other five components.  Profiles along each axis are tabulated at the E
// positions (integer n) and the H positions (n + 1/2).  Outside every layer a component's update
// is the reference's formula, operation for operation, so the interior stays bit-identical to
// the non-PML solver; psi is stored only in the slabs of its axis (2L + 1 positions).
//
// One grid: cpml_e / cpml_h per step, monitors accumulated per step.  A batch of grids:
// cpml_e_batch / cpml_h_batch cover every grid in one launch each (blockIdx.z = grid * max_nz
// + k, arguments from a device array) and stage the monitor values for the deferred DFT.
#include "fdtd_kernels.cuh"

namespace fdtd {

namespace {

struct CoefRefs {
  const float* c[12];  // pitched per-cell arrays (or null with a material map)
};

__device__ __forceinline__ void e_coefs(const float* const* A, const uint16_t* mat,
                                        const Material* tab, long long idx, float* ca, float* cb) {
  if (mat) {
    const Material m = tab[mat[idx]];
    ca[0] = m.a.x; cb[0] = m.a.y; ca[1] = m.a.z; cb[1] = m.a.w; ca[2] = m.b.x; cb[2] = m.b.y;
  } else {
    for (int c = 0; c < 3; ++c) {
      ca[c] = A[c][idx];
      cb[c] = A[3 + c][idx];
    }
  }
}

__device__ __forceinline__ void h_coefs(const float* const* A, const uint16_t* mat,
                                        const Material* tab, long long idx, float* da, float* db) {
  if (mat) {
    const Material m = tab[mat[idx]];
    da[0] = m.b.z; db[0] = m.b.w; da[1] = m.c.x; db[1] = m.c.y; da[2] = m.c.z; db[2] = m.c.w;
  } else {
    for (int c = 0; c < 3; ++c) {
      da[c] = A[6 + c][idx];
      db[c] = A[9 + c][idx];
    }
  }
}

// psi slab element of axis a at slot s for cell (i, j, k)
__device__ __forceinline__ long long psi_at(const Grid& g, int a, int S, int s, int i, int j, int k) {
  if (a == 0) return s + (long long)S * (j + (long long)g.ny * k);
  if (a == 1) return i + (long long)g.nx * (s + (long long)S * k);
  return i + (long long)g.nx * (j + (long long)g.ny * s);
}

// The CPML form of one difference d along axis a at table position n: updates psi in place and
// returns d / kappa + psi; outside the layer (slot < 0) returns d itself.
__device__ __forceinline__ float stretched(float d, const CpmlAxis& ax, bool h, int n,
                                           float* psi, long long pidx) {
  const int s = h ? ax.slot_h[n] : ax.slot_e[n];
  if (s < 0) return d;
  const float b = h ? ax.bh[n] : ax.be[n], a = h ? ax.ah[n] : ax.ae[n];
  const float ik = h ? ax.ikh[n] : ax.ike[n];
  const float p = add(mul(b, psi[pidx]), mul(a, d));
  psi[pidx] = p;
  return add(mul(d, ik), p);
}

__device__ __forceinline__ bool src_sum(const Sources& S, int comp, int i, int j, int k,
                                        long long t, float* v) {
  return source_value(S, comp, i, j, k, t, v);
}

__device__ __forceinline__ bool interior(const Grid& g, int i, int j, int k) {
  return i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2 && k >= 1 && k <= g.nz - 2;
}

// E update of interior cell (i, j, k) at step t: E and H of step t from Fi, the new E into Fo
// (Fi == Fo: in place).
__device__ __forceinline__ void e_cell(const Grid& g, const FieldPtrs& Fi, const FieldPtrs& Fo,
                                       const float* const* A, const uint16_t* mat,
                                       const Material* tab, const Sources& S, long long t,
                                       float dx, const CpmlDev& P, int i, int j, int k) {
  const long long sy = g.pitch, sz = g.plane, idx = i + j * sy + k * sz;
  float* const* f = Fi.f;
  const float hx = f[3][idx], hy = f[4][idx], hz = f[5][idx];
  const float dyHz = sub(hz, f[5][idx - sy]), dzHy = sub(hy, f[4][idx - sz]);
  const float dzHx = sub(hx, f[3][idx - sz]), dxHz = sub(hz, f[5][idx - 1]);
  const float dxHy = sub(hy, f[4][idx - 1]), dyHx = sub(hx, f[3][idx - sy]);
  const CpmlAxis& X = P.ax[0];
  const CpmlAxis& Y = P.ax[1];
  const CpmlAxis& Z = P.ax[2];
  float cx, cy, cz;
  if (X.slot_e[i] < 0 && Y.slot_e[j] < 0 && Z.slot_e[k] < 0) {  // the reference's update
    cx = sub(dyHz, dzHy);
    cy = sub(dzHx, dxHz);
    cz = sub(dxHy, dyHx);
  } else {
    const int sxs = X.slot_e[i] < 0 ? 0 : X.slot_e[i], sys = Y.slot_e[j] < 0 ? 0 : Y.slot_e[j];
    const int szs = Z.slot_e[k] < 0 ? 0 : Z.slot_e[k];
    cx = sub(stretched(dyHz, Y, false, j, P.psi_e[0], psi_at(g, 1, Y.S, sys, i, j, k)),
             stretched(dzHy, Z, false, k, P.psi_e[1], psi_at(g, 2, Z.S, szs, i, j, k)));
    cy = sub(stretched(dzHx, Z, false, k, P.psi_e[2], psi_at(g, 2, Z.S, szs, i, j, k)),
             stretched(dxHz, X, false, i, P.psi_e[3], psi_at(g, 0, X.S, sxs, i, j, k)));
    cz = sub(stretched(dxHy, X, false, i, P.psi_e[4], psi_at(g, 0, X.S, sxs, i, j, k)),
             stretched(dyHx, Y, false, j, P.psi_e[5], psi_at(g, 1, Y.S, sys, i, j, k)));
  }
  if (S.n) {
    float v;
    if (src_sum(S, 0, i, j, k, t, &v)) cx = sub(cx, mul(v, dx));
    if (src_sum(S, 1, i, j, k, t, &v)) cy = sub(cy, mul(v, dx));
    if (src_sum(S, 2, i, j, k, t, &v)) cz = sub(cz, mul(v, dx));
  }
  float ca[3], cb[3];
  e_coefs(A, mat, tab, idx, ca, cb);
  const float ex = f[0][idx], ey = f[1][idx], ez = f[2][idx];
  Fo.f[0][idx] = yee(ca[0], ex, cb[0], cx);
  Fo.f[1][idx] = yee(ca[1], ey, cb[1], cy);
  Fo.f[2][idx] = yee(ca[2], ez, cb[2], cz);
}

// H update of interior cell (i, j, k) at step t, after every E update of the step: H of step t
// from Fi, the new E from Fo, the new H into Fo (Fi == Fo: in place).
__device__ __forceinline__ void h_cell(const Grid& g, const FieldPtrs& Fi, const FieldPtrs& Fo,
                                       const float* const* A, const uint16_t* mat,
                                       const Material* tab, const Sources& S, long long t,
                                       float dx, const CpmlDev& P, int i, int j, int k) {
  const long long sy = g.pitch, sz = g.plane, idx = i + j * sy + k * sz;
  float* const* f = Fo.f;
  const float ex = f[0][idx], ey = f[1][idx], ez = f[2][idx];
  const float dzEy = sub(f[1][idx + sz], ey), dyEz = sub(f[2][idx + sy], ez);
  const float dxEz = sub(f[2][idx + 1], ez), dzEx = sub(f[0][idx + sz], ex);
  const float dyEx = sub(f[0][idx + sy], ex), dxEy = sub(f[1][idx + 1], ey);
  const CpmlAxis& X = P.ax[0];
  const CpmlAxis& Y = P.ax[1];
  const CpmlAxis& Z = P.ax[2];
  float cx, cy, cz;
  if (X.slot_h[i] < 0 && Y.slot_h[j] < 0 && Z.slot_h[k] < 0) {  // the reference's update
    cx = sub(dzEy, dyEz);
    cy = sub(dxEz, dzEx);
    cz = sub(dyEx, dxEy);
  } else {
    const int sxs = X.slot_h[i] < 0 ? 0 : X.slot_h[i], sys = Y.slot_h[j] < 0 ? 0 : Y.slot_h[j];
    const int szs = Z.slot_h[k] < 0 ? 0 : Z.slot_h[k];
    cx = sub(stretched(dzEy, Z, true, k, P.psi_h[0], psi_at(g, 2, Z.S, szs, i, j, k)),
             stretched(dyEz, Y, true, j, P.psi_h[1], psi_at(g, 1, Y.S, sys, i, j, k)));
    cy = sub(stretched(dxEz, X, true, i, P.psi_h[2], psi_at(g, 0, X.S, sxs, i, j, k)),
             stretched(dzEx, Z, true, k, P.psi_h[3], psi_at(g, 2, Z.S, szs, i, j, k)));
    cz = sub(stretched(dyEx, Y, true, j, P.psi_h[4], psi_at(g, 1, Y.S, sys, i, j, k)),
             stretched(dxEy, X, true, i, P.psi_h[5], psi_at(g, 0, X.S, sxs, i, j, k)));
  }
  if (S.n) {
    float v;
    if (src_sum(S, 3, i, j, k, t, &v)) cx = sub(cx, mul(v, dx));
    if (src_sum(S, 4, i, j, k, t, &v)) cy = sub(cy, mul(v, dx));
    if (src_sum(S, 5, i, j, k, t, &v)) cz = sub(cz, mul(v, dx));
  }
  float da[3], db[3];
  h_coefs(A, mat, tab, idx, da, db);
  const float hx = Fi.f[3][idx], hy = Fi.f[4][idx], hz = Fi.f[5][idx];
  Fo.f[3][idx] = yee(da[0], hx, db[0], cx);
  Fo.f[4][idx] = yee(da[1], hy, db[1], cy);
  Fo.f[5][idx] = yee(da[2], hz, db[2], cz);
}

// One grid: grid (ceil(nx/32), ceil(ny/4), nz), block (32, 4); interior cells only.
__global__ void __launch_bounds__(128) cpml_e(Grid g, FieldPtrs F, CoefRefs A, const uint16_t* mat,
                                              const Material* tab, Sources S, long long t,
                                              float dx, CpmlDev P) {
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 4 + threadIdx.y, k = blockIdx.z;
  if (interior(g, i, j, k)) e_cell(g, F, F, A.c, mat, tab, S, t, dx, P, i, j, k);
}

__global__ void __launch_bounds__(128) cpml_h(Grid g, FieldPtrs F, CoefRefs A, const uint16_t* mat,
                                              const Material* tab, Sources S, long long t,
                                              float dx, CpmlDev P) {
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 4 + threadIdx.y, k = blockIdx.z;
  if (interior(g, i, j, k)) h_cell(g, F, F, A.c, mat, tab, S, t, dx, P, i, j, k);
}

// Monitor values of cell (i, j) of plane k at step t into the staging rings: the E monitors
// after the E update (e_comps), the H monitors after the H update.  Face cells, which the update
// leaves unchanged, are staged too: the fold reads every cell of the plane.
__device__ __forceinline__ void stage_cell(const CpmlSim& s, long long t, int i, int j, int k,
                                           bool e_comps) {
  for (int n = 0; n < s.M.n; ++n) {
    const MonitorDev& m = s.M.m[n];
    if ((m.comp < 3) != e_comps || m.k != k) continue;
    const long long idx = i + (long long)j * s.g.pitch + (long long)k * s.g.plane;
    dft_record(m, t, i, j, s.g, s.F.f[m.comp][idx]);
  }
}

// A batch: blockIdx.z = grid * max_nz + k over the grids' argument array.
__global__ void __launch_bounds__(128) cpml_e_batch(const CpmlSim* sims, int max_nz,
                                                    long long t_offset) {
  const CpmlSim& s = sims[blockIdx.z / max_nz];
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 4 + threadIdx.y;
  const int k = (int)(blockIdx.z % max_nz);
  if (i >= s.g.nx || j >= s.g.ny || k >= s.g.nz) return;
  const long long t = s.t0 + t_offset;
  if (interior(s.g, i, j, k)) e_cell(s.g, s.F, s.F, s.coef, s.mat, s.tab, s.S, t, s.dx, s.P, i, j, k);
  if (s.M.n) stage_cell(s, t, i, j, k, true);
}

__global__ void __launch_bounds__(128) cpml_h_batch(const CpmlSim* sims, int max_nz,
                                                    long long t_offset) {
  const CpmlSim& s = sims[blockIdx.z / max_nz];
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 4 + threadIdx.y;
  const int k = (int)(blockIdx.z % max_nz);
  if (i >= s.g.nx || j >= s.g.ny || k >= s.g.nz) return;
  const long long t = s.t0 + t_offset;
  if (interior(s.g, i, j, k)) h_cell(s.g, s.F, s.F, s.coef, s.mat, s.tab, s.S, t, s.dx, s.P, i, j, k);
  if (s.M.n) stage_cell(s, t, i, j, k, false);
}

// The shell companion: blockIdx.x indexes the block list; cells inside `inner` return.
template <bool H>
__global__ void __launch_bounds__(128) cpml_region(Grid g, FieldPtrs Fi, FieldPtrs Fo,
                                                   const uint16_t* mat, const Material* tab,
                                                   Sources S, Monitors M, CpmlDev P, long long t,
                                                   float dx, const int4* blocks, CpmlBox inner) {
  const int4 b = blocks[blockIdx.x];
  const int i = b.x * 32 + threadIdx.x, j = b.y * 4 + threadIdx.y, k = b.z;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  if (i >= inner.lo[0] && i < inner.hi[0] && j >= inner.lo[1] && j < inner.hi[1] &&
      k >= inner.lo[2] && k < inner.hi[2])
    return;
  const long long idx = i + (long long)j * g.pitch + (long long)k * g.plane;
  const int c0 = H ? 3 : 0;
  if (interior(g, i, j, k)) {
    if (H)
      h_cell(g, Fi, Fo, nullptr, mat, tab, S, t, dx, P, i, j, k);
    else
      e_cell(g, Fi, Fo, nullptr, mat, tab, S, t, dx, P, i, j, k);
  } else if (Fi.f[c0] != Fo.f[c0]) {  // faces never change: carry them into the output set
    for (int c = c0; c < c0 + 3; ++c) Fo.f[c][idx] = Fi.f[c][idx];
  }
  for (int n = 0; n < M.n; ++n) {
    const MonitorDev& m = M.m[n];
    if ((m.comp >= 3) == H && m.k == k) dft_record(m, t, i, j, g, Fo.f[m.comp][idx]);
  }
}

}  // namespace

cudaError_t launch_cpml_region(bool h_half, const Grid& g, const FieldPtrs& Fi,
                               const FieldPtrs& Fo, const uint16_t* mat, const Material* tab,
                               const Sources& S, const Monitors& M, const CpmlDev& P,
                               long long t, float dx, const int4* blocks, int nblocks,
                               const CpmlBox& inner, cudaStream_t st) {
  if (nblocks <= 0) return cudaSuccess;
  if (!mat) return cudaErrorInvalidValue;
  if (h_half)
    cpml_region<true><<<nblocks, dim3(32, 4), 0, st>>>(g, Fi, Fo, mat, tab, S, M, P, t, dx,
                                                        blocks, inner);
  else
    cpml_region<false><<<nblocks, dim3(32, 4), 0, st>>>(g, Fi, Fo, mat, tab, S, M, P, t, dx,
                                                         blocks, inner);
  return cudaGetLastError();
}

cudaError_t launch_cpml_batch_step(const CpmlSim* sims, int nsims, int max_nx, int max_ny,
                                   int max_nz, long long t_offset, cudaStream_t st) {
  if (nsims <= 0) return cudaSuccess;
  if (max_nz <= 0 || max_nz > 65535) return cudaErrorInvalidValue;
  // grids per launch pair: blockIdx.z stays within its 65535 limit (grids are independent, so
  // each group's E launch before its H launch is all the order a step needs)
  const int per = 65535 / max_nz;
  const dim3 blk(32, 4);
  for (int g0 = 0; g0 < nsims; g0 += per) {
    const int n = nsims - g0 < per ? nsims - g0 : per;
    const dim3 grd((max_nx + 31) / 32, (max_ny + 3) / 4, (unsigned)(n * max_nz));
    cpml_e_batch<<<grd, blk, 0, st>>>(sims + g0, max_nz, t_offset);
    cpml_h_batch<<<grd, blk, 0, st>>>(sims + g0, max_nz, t_offset);
  }
  return cudaGetLastError();
}

cudaError_t launch_cpml_step(const Grid& g, const FieldPtrs& F, const float* const* coef,
                             const uint16_t* mat, const Material* tab, const Sources& S,
                             const Monitors& M, const CpmlDev& P, long long t, float dx,
                             cudaStream_t st, int* launches) {
  CoefRefs A;
  for (int c = 0; c < 12; ++c) A.c[c] = coef ? coef[c] : nullptr;
  const dim3 blk(32, 4), grd((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz);
  cpml_e<<<grd, blk, 0, st>>>(g, F, A, mat, tab, S, t, dx, P);
  cpml_h<<<grd, blk, 0, st>>>(g, F, A, mat, tab, S, t, dx, P);
  *launches += 2;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || M.n == 0) return e;
  return launch_naive_dft(g, F, M, t, st, launches);
}

}  // namespace fdtd
