// k_tiled.cu -- z-streaming, temporally tiled Yee kernel for sm_100a.
//
// Replaces the reference's tiled GPU paths (mix-mapping ver2 diamond tiling,
// gDiamond/kernels_mm_ver2.cuh:346-720, and ver3 overlapped tiling,
// gDiamond/kernels_mm_ver3.cuh:282-609) with a different schedule:
//
//  * A CTA owns a 32 x ROWS column of the x-y plane (one warp per row, one cell per thread) and
//    marches along z.  Each z-plane of the six fields and of the uint16 material map is staged
//    into shared memory by TMA (cp.async.bulk.tensor into this CTA's own shared memory) through a 3-stage mbarrier
//    pipeline, so HBM reads run ahead of the arithmetic.
//  * BLT time levels run as a wavefront in (z, t): when plane p arrives, level s computes
//    E^s at plane p-s+1 and H^s at plane p-s.  Neighbours along z are the thread's own values
//    from the previous iteration (registers); neighbours along x come from warp shuffles;
//    neighbours along y come from small shared-memory planes.  No z redundancy.
//  * Along x and y the tile overlaps its neighbours (trapezoid): the valid region shrinks by
//    one cell per level on each side (E needs H at -1, H needs E at +1), so a CTA writes the
//    inner (32-2*BLT) x (ROWS-2*BLT) cells of level BLT.  x tile starts are multiples of 4
//    elements (16-byte TMA rule).
//  * Coefficients come from a per-material table indexed by the uint16 map (2 bytes per cell
//    instead of 48).  Sources are a short descriptor list.  When a level passes a DFT monitor
//    plane the tile writes that step's values into the monitor's staging ring (dft_record), so
//    no extra field pass is made; dft_fold.cu adds the ring to the FP64 sums.
//  * Source set -> destination set (ping-pong), so overlapping tiles never see each other's
//    writes.  Every multiply/add is separately rounded: results are bit-identical to the
//    reference CPU update.
//  * Every mbarrier wait is bounded; on expiry the CTA sets the device error word, all its
//    threads leave the z-march together, and the host reports FDTD_ERR_DEVICE_TIMEOUT.
#include "fdtd_kernels.cuh"

namespace fdtd {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr long long kWaitLimit = 2000000000LL;  // SM clocks, about one second

template <int B, int TY>
struct Tiled {
  static constexpr int PL = 32 * TY;          // elements of one staged field plane
  static constexpr int MPL = kMatBoxX * TY;   // elements of one staged material plane
  static constexpr int NS = kTiledStages;
  static constexpr int SX = tiled_sx(B);
  static constexpr int SY = tiled_sy(B, TY);
  static constexpr int XBASE = tiled_xbase(B);
  static constexpr uint32_t STAGE_F_BYTES = 6u * PL * 4u;
  static constexpr uint32_t STAGE_M_BYTES = MPL * 2u;
  static constexpr uint32_t TX_BYTES = STAGE_F_BYTES + STAGE_M_BYTES;
  static constexpr size_t OFF_M = (size_t)NS * STAGE_F_BYTES;
  static constexpr size_t OFF_H = OFF_M + (size_t)NS * STAGE_M_BYTES;
  static constexpr size_t OFF_E = OFF_H + 2u * 2u * PL * 4u;
  static constexpr size_t OFF_BAR = OFF_E + (size_t)B * 2u * PL * 4u;
  static constexpr size_t SMEM = OFF_BAR + NS * 8u + 128u;  // + alignment slack
  static_assert(SY >= 1, "tile too short for this BLT");
  static_assert(STAGE_M_BYTES % 128 == 0, "stage alignment");
};

__device__ __forceinline__ float pick3(const float* v, int c) {
  return c == 0 ? v[0] : (c == 1 ? v[1] : v[2]);
}

template <int B, int TY>
__global__ void __launch_bounds__(32 * TY) fdtd_tiled(const __grid_constant__ TiledArgs a) {
  using K = Tiled<B, TY>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // TMA destinations must start on 128-byte boundaries: align the base by hand (the launch
  // requests 128 bytes of slack).
  unsigned char* smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  float* st_f = reinterpret_cast<float*>(smem);
  uint16_t* st_m = reinterpret_cast<uint16_t*>(smem + K::OFF_M);
  float* hbuf = reinterpret_cast<float*>(smem + K::OFF_H);  // [2][Hz,Hx][PL]
  float* ebuf = reinterpret_cast<float*>(smem + K::OFF_E);  // [B][Ex,Ez][PL]
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + K::OFF_BAR);
  __shared__ int s_abort;

  const Grid g = a.g;
  const int z0 = (int)blockIdx.z * a.zlen;
  if (z0 >= g.nz) return;  // uniform across the CTA
  const int z1 = min(g.nz, z0 + a.zlen);
  const int ps = z0 - B;                 // first plane loaded
  const int niter = (z1 - z0) + 2 * B;   // planes z0-B .. z1+B-1

  const int lx = threadIdx.x, ly = threadIdx.y;
  const int tid = ly * 32 + lx;
  const int X = (int)blockIdx.x * K::SX + K::XBASE;  // multiple of 4
  const int Y = (int)blockIdx.y * K::SY - B;
  const int X8 = X & ~7;                              // material box start, multiple of 8
  const int x = X + lx, y = Y + ly;
  const bool col_int = x >= 1 && x <= g.nx - 2 && y >= 1 && y <= g.ny - 2;
  const bool col_out = lx >= B && lx < B + K::SX && ly >= B && ly < TY - B && x >= 0 &&
                       x < g.nx && y >= 0 && y < g.ny;
  unsigned smask = 0;
  for (int n = 0; n < a.S.n; ++n) {
    const SourceDev& s = a.S.s[n];
    if ((s.kind == 0 && s.i == x && s.j == y) || (s.kind == 1 && col_int)) smask |= 1u << n;
  }
  // CTA-uniform z-iteration ranges in which some level touches a source plane inside this tile
  // or a monitor plane: E at plane p-s+1 and H at plane p-s for s = 1..B.  Outside them the
  // per-level source and monitor code is skipped by every warp.
  int src_lo = 1 << 30, src_hi = -(1 << 30), mon_lo = 1 << 30, mon_hi = -(1 << 30);
  for (int n = 0; n < a.S.n; ++n) {
    const SourceDev& s = a.S.s[n];
    if (s.kind == 0 && (s.i < X || s.i >= X + 32 || s.j < Y || s.j >= Y + TY)) continue;
    src_lo = min(src_lo, s.k);
    src_hi = max(src_hi, s.k + B);
  }
  for (int n = 0; n < a.M.n; ++n) {
    const int k = a.M.m[n].k + (a.M.m[n].comp < 3 ? 0 : 1);
    mon_lo = min(mon_lo, k);
    mon_hi = max(mon_hi, k + B - 1);
  }

  if (tid == 0) {
    s_abort = 0;
    for (int s = 0; s < K::NS; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  for (int q = tid; q < (4 + 2 * B) * K::PL; q += 32 * TY) hbuf[q] = 0.0f;  // hbuf + ebuf
  __syncthreads();

  auto issue = [&](int it_) {
    const int stage = it_ % K::NS;
    uint64_t* bar = &bars[stage];
    mbar_arrive_expect_tx(bar, K::TX_BYTES);
    float* d = st_f + stage * 6 * K::PL;
    const int pz = ps + it_;
#pragma unroll
    for (int c = 0; c < 6; ++c) tma_load_3d(d + c * K::PL, &a.tm_src[c], bar, X, Y, pz);
    tma_load_3d(st_m + stage * K::MPL, &a.tm_mat, bar, X8, Y, pz);
  };
  if (tid == 0) {
    for (int it_ = 0; it_ < K::NS && it_ < niter; ++it_) issue(it_);
  }

  // Per-level state: Ep[s] = E^s at plane (p-s+1)-1, Hp[s] = H^s at plane (p-s)-1, i.e. the
  // values this thread produced one iteration ago.  Hp[0] = H^0 of the previous plane.
  float Ep[B + 1][3], Hp[B + 1][3];
#pragma unroll
  for (int s = 0; s <= B; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) Ep[s][c] = Hp[s][c] = 0.0f;
  uint32_t mq[B + 1];  // material ids of planes p, p-1, ..., p-B
#pragma unroll
  for (int s = 0; s <= B; ++s) mq[s] = 0;

  const int o = ly * 32 + lx;
  const int oym = (ly > 0 ? ly - 1 : 0) * 32 + lx;
  const int oyp = (ly < TY - 1 ? ly + 1 : TY - 1) * 32 + lx;
  const int om = ly * kMatBoxX + lx + (X - X8);
  const float dx = a.dx;
  const long long pitch = g.pitch, plane = g.plane;

  int it = 0;
  bool abort = false;
  for (; it < niter; ++it) {
    const int p = ps + it;
    const int stage = it % K::NS;
    if (!mbar_wait_bounded(&bars[stage], (uint32_t)(it / K::NS) & 1u, kWaitLimit)) {
      s_abort = 1;
      atomicOr(a.err, kErrTimeout);
    }
    if (B == 1) __syncthreads();  // orders last iteration's ebuf writes before this read
    const bool src_iter = smask != 0 && p >= src_lo && p <= src_hi;
    const bool mon_iter = p >= mon_lo && p <= mon_hi;

    const float* S0 = st_f + stage * 6 * K::PL;
#pragma unroll
    for (int s = B; s >= 1; --s) mq[s] = mq[s - 1];
    mq[0] = st_m[stage * K::MPL + om];
    float Hc[3] = {S0[3 * K::PL + o], S0[4 * K::PL + o], S0[5 * K::PL + o]};
    float hz_ym = S0[5 * K::PL + oym], hx_ym = S0[3 * K::PL + oym];
    float Eo[3] = {S0[o], S0[K::PL + o], S0[2 * K::PL + o]};
    float EnPrev[3] = {0.0f, 0.0f, 0.0f};
    float EnB[3] = {0.0f, 0.0f, 0.0f}, HnB[3] = {0.0f, 0.0f, 0.0f};

#pragma unroll
    for (int s = 1; s <= B; ++s) {
      const int e = p - s + 1;
      const long long t = a.t0 + (s - 1);
      // ---------------- E^s(e) from E^{s-1}(e), H^{s-1}(e), H^{s-1}(e-1)
      const float hz_xm = __shfl_up_sync(kFull, Hc[2], 1);
      const float hy_xm = __shfl_up_sync(kFull, Hc[1], 1);
      float cx = sub(sub(Hc[2], hz_ym), sub(Hc[1], Hp[s - 1][1]));
      float cy = sub(sub(Hc[0], Hp[s - 1][0]), sub(Hc[2], hz_xm));
      float cz = sub(sub(Hc[1], hy_xm), sub(Hc[0], hx_ym));
      float En[3] = {Eo[0], Eo[1], Eo[2]};
      if (col_int && e >= 1 && e <= g.nz - 2) {
        if (src_iter) {
          float v;
          if (source_value(a.S, 0, x, y, e, t, &v)) cx = sub(cx, mul(v, dx));
          if (source_value(a.S, 1, x, y, e, t, &v)) cy = sub(cy, mul(v, dx));
          if (source_value(a.S, 2, x, y, e, t, &v)) cz = sub(cz, mul(v, dx));
        }
        const Material* m = a.table + mq[s - 1];
        const float4 ma = __ldg(&m->a), mb = __ldg(&m->b);
        En[0] = yee(ma.x, Eo[0], ma.y, cx);
        En[1] = yee(ma.z, Eo[1], ma.w, cy);
        En[2] = yee(mb.x, Eo[2], mb.y, cz);
      }
      // ---------------- H^s(e-1) from H^{s-1}(e-1), E^s(e-1), E^s(e)
      const float ez_xp = __shfl_down_sync(kFull, Ep[s][2], 1);
      const float ey_xp = __shfl_down_sync(kFull, Ep[s][1], 1);
      float* eb = ebuf + (s - 1) * 2 * K::PL;
      const float ex_yp = eb[oyp], ez_yp = eb[K::PL + oyp];
      cx = sub(sub(En[1], Ep[s][1]), sub(ez_yp, Ep[s][2]));
      cy = sub(sub(ez_xp, Ep[s][2]), sub(En[0], Ep[s][0]));
      cz = sub(sub(ex_yp, Ep[s][0]), sub(ey_xp, Ep[s][1]));
      float Hn[3] = {Hp[s - 1][0], Hp[s - 1][1], Hp[s - 1][2]};
      if (col_int && e - 1 >= 1 && e - 1 <= g.nz - 2) {
        if (src_iter) {
          float v;
          if (source_value(a.S, 3, x, y, e - 1, t, &v)) cx = sub(cx, mul(v, dx));
          if (source_value(a.S, 4, x, y, e - 1, t, &v)) cy = sub(cy, mul(v, dx));
          if (source_value(a.S, 5, x, y, e - 1, t, &v)) cz = sub(cz, mul(v, dx));
        }
        const Material* m = a.table + mq[s];
        const float4 mb = __ldg(&m->b), mc = __ldg(&m->c);
        Hn[0] = yee(mb.z, Hp[s - 1][0], mb.w, cx);
        Hn[1] = yee(mc.x, Hp[s - 1][1], mc.y, cy);
        Hn[2] = yee(mc.z, Hp[s - 1][2], mc.w, cz);
      }
      // ---------------- DFT monitors: stage this level's values when it passes a monitor plane
      if (mon_iter && col_out) {
        for (int n = 0; n < a.M.n; ++n) {
          const MonitorDev& m = a.M.m[n];
          const int mk = m.comp < 3 ? e : e - 1;
          if (m.k == mk && mk >= z0 && mk < z1)
            dft_record(m, t, x, y, g, m.comp < 3 ? pick3(En, m.comp) : pick3(Hn, m.comp - 3));
        }
      }
      // ---------------- exchange
      if (s < B) {
        float* hb = hbuf + (s & 1) * 2 * K::PL;
        hb[o] = Hn[2];
        hb[K::PL + o] = Hn[0];
      }
      __syncthreads();
      eb[o] = En[0];  // E^s(e) is read (as the y+1 neighbour) in the next iteration
      eb[K::PL + o] = En[2];
      if (s == 1) {
        abort = s_abort != 0;
        if (!abort && tid == 0 && it + K::NS < niter) {
          fence_proxy_async_smem();  // generic-proxy reads of this stage precede the refill
          issue(it + K::NS);
        }
      }
      // ---------------- rotate
      if (s >= 2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) Ep[s - 1][c] = EnPrev[c];
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        EnPrev[c] = En[c];
        Hp[s - 1][c] = Hc[c];
      }
      if (s < B) {
        const float* hb = hbuf + (s & 1) * 2 * K::PL;
        hz_ym = hb[oym];
        hx_ym = hb[K::PL + oym];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          Hc[c] = Hn[c];
          Eo[c] = Ep[s][c];
        }
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          EnB[c] = En[c];
          HnB[c] = Hn[c];
        }
      }
      if (abort) break;
    }
    if (abort) break;
#pragma unroll
    for (int c = 0; c < 3; ++c) Ep[B][c] = EnPrev[c];

    // ---------------- level-BLT results: E at plane p-B+1, H at plane p-B
    if (col_out) {
      const int eB = p - B + 1, hB = p - B;
      if (eB >= z0 && eB < z1) {
        const long long idx = x + (long long)y * pitch + (long long)eB * plane;
        a.dst.f[0][idx] = EnB[0];
        a.dst.f[1][idx] = EnB[1];
        a.dst.f[2][idx] = EnB[2];
      }
      if (hB >= z0 && hB < z1) {
        const long long idx = x + (long long)y * pitch + (long long)hB * plane;
        a.dst.f[3][idx] = HnB[0];
        a.dst.f[4][idx] = HnB[1];
        a.dst.f[5][idx] = HnB[2];
      }
    }
  }

  if (abort && tid == 0) {
    // Let copies that were already issued land before the CTA's shared memory is released.
    for (int q = it + 1; q < niter && q < it + K::NS; ++q)
      (void)mbar_wait_bounded(&bars[q % K::NS], (uint32_t)(q / K::NS) & 1u, kWaitLimit / 8);
  }
}

template <int B, int TY>
cudaError_t launch_one(const TiledArgs& a, dim3 grid, cudaStream_t st) {
  using K = Tiled<B, TY>;
  cudaError_t e = cudaFuncSetAttribute(fdtd_tiled<B, TY>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::SMEM);
  if (e != cudaSuccess) return e;
  fdtd_tiled<B, TY><<<grid, dim3(32, TY), K::SMEM, st>>>(a);
  return cudaGetLastError();
}

template <int TY>
cudaError_t launch_rows(int blt, const TiledArgs& a, dim3 grid, cudaStream_t st) {
  switch (blt) {
    case 1: return launch_one<1, TY>(a, grid, st);
    case 2: return launch_one<2, TY>(a, grid, st);
    case 3: return launch_one<3, TY>(a, grid, st);
    case 4: if constexpr (TY > 8) return launch_one<4, TY>(a, grid, st); break;
    case 5: if constexpr (TY > 8) return launch_one<5, TY>(a, grid, st); break;
    case 6: if constexpr (TY > 8) return launch_one<6, TY>(a, grid, st); break;
    default: break;
  }
  return cudaErrorInvalidValue;
}

template <int B, int TY>
size_t smem_of() { return Tiled<B, TY>::SMEM; }

}  // namespace

bool tiled_config_supported(const TiledConfig& c) {
  if (c.min_blocks != 1 || c.pairs32 || c.storage != 0) return false;  // FP32 fields only
  if (c.rows != 8 && c.rows != 16 && c.rows != 32) return false;
  if (c.blt < 1 || c.blt > 6) return false;
  if (c.rows == 8 && c.blt > 3) return false;
  return c.z_chunks >= 1;
}

size_t tiled_smem_bytes(const TiledConfig& c) {
  // Mirrors Tiled<B, TY>::SMEM.
  const size_t PL = 32u * c.rows, MPL = (size_t)kMatBoxX * c.rows;
  return kTiledStages * (6 * PL * 4 + MPL * 2) + 4 * PL * 4 + (size_t)c.blt * 2 * PL * 4 +
         kTiledStages * 8 + 128;
}

dim3 tiled_grid(const TiledConfig& c, const Grid& g) {
  const int sx = tiled_sx(c.blt), sy = tiled_sy(c.blt, c.rows);
  const int first = tiled_xbase(c.blt) + c.blt;  // first output x (<= 0)
  const int ntx = (g.nx - first + sx - 1) / sx;
  const int nty = (g.ny + sy - 1) / sy;
  const int zlen = (g.nz + c.z_chunks - 1) / c.z_chunks;
  const int nzc = (g.nz + zlen - 1) / zlen;
  return dim3(ntx, nty, nzc);
}

cudaError_t launch_tiled(const TiledConfig& c, const TiledArgs& a, const Grid& g,
                         cudaStream_t st) {
  if (!tiled_config_supported(c)) return cudaErrorInvalidValue;
  const dim3 grid = tiled_grid(c, g);
  switch (c.rows) {
    case 8: return launch_rows<8>(c.blt, a, grid, st);
    case 16: return launch_rows<16>(c.blt, a, grid, st);
    case 32: return launch_rows<32>(c.blt, a, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fdtd
