// k_tiled2.cuh -- the z-streaming temporally tiled Yee kernel with two cells per thread in x,
// for one grid (fdtd_tiled2) and for a batch of independent grids in one persistent launch
// (fdtd_tiled2_batch), with 64-cell rows (one per warp) or 32-cell rows (two per warp).
//
// Same schedule as k_tiled.cu (TMA plane pipeline, BLT-level (z,t) wavefront, trapezoid tiles in
// x and y, material map, monitor values staged for the deferred DFT, bounded waits), but each
// thread owns an x-pair (2l, 2l+1) of a 64-wide warp row:
//  * the pair's inner neighbours are in registers; only the pair edges cross lanes, so a level
//    needs one shuffle per field direction per pair instead of per cell;
//  * staged planes, y-exchange planes and outputs move as pairs (one shared/global instruction
//    for two cells);
//  * the x-trapezoid wastes 2*BLT of 64 columns instead of 2*BLT of 32;
//  * source and monitor planes are tested once per z-iteration against CTA-uniform ranges.
//
// Field storage S is float, __half or __nv_bfloat16 for E, and SH (default S) for H: <__half,
// float> keeps E in FP16 and H in FP32.  Arithmetic is FP32 in every case and the
// intermediate time levels never leave the SM in reduced precision: only the HBM round trip of
// each BLT-step pass is 16-bit.  A 16-bit value v is stored as v * inv_scale[c] and read back
// times scale[c]; scales are powers of two, so the scaling itself rounds nothing.  With FP32
// storage no scaling is applied and every multiply/add is separately rounded: results are
// bit-identical to the reference CPU update.
//
// x tile starts are even but otherwise free: the TMA boxes start at the tile start rounded down
// to 8 elements (16 bytes of either stored type: the TMA rule for the innermost coordinate) and
// are 8 elements wider than the row; threads index the staged planes from the remainder.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "fdtd_kernels.cuh"

namespace fdtd {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr long long kWaitLimit = 2000000000LL;  // SM clocks, about one second

template <typename S>
struct Store;

// Load / store of a field value in its storage type.  The 16-bit forms also keep, in `seen`,
// the running maximum of |stored value| (NaN-propagating) over the thread's stores, so a value
// that overflowed to +-inf (or became NaN) is reported once per thread at the end of its tile.
template <>
struct Store<float> {
  static constexpr bool kScaled = false;
  __device__ static float2 ld2(const float* p, float) {
    return *reinterpret_cast<const float2*>(p);
  }
  __device__ static void st2(float* p, float a, float b, float, uint32_t&) {
    *reinterpret_cast<float2*>(p) = make_float2(a, b);
  }
  __device__ static void st1(float* p, float a, float, uint32_t&) { *p = a; }
  __device__ static bool bad(uint32_t) { return false; }
};

template <>
struct Store<__half> {
  static constexpr bool kScaled = true;
  __device__ static float2 ld2(const __half* p, float sc) {
    const float2 v = __half22float2(*reinterpret_cast<const __half2*>(p));
    return make_float2(v.x * sc, v.y * sc);
  }
  __device__ static void track(uint32_t& seen, __half2 h) {
    __half2 m = *reinterpret_cast<const __half2*>(&seen);
    m = __hmax2_nan(m, __habs2(h));
    seen = *reinterpret_cast<const uint32_t*>(&m);
  }
  __device__ static void st2(__half* p, float a, float b, float inv, uint32_t& seen) {
    const __half2 h = __floats2half2_rn(a * inv, b * inv);
    *reinterpret_cast<__half2*>(p) = h;
    track(seen, h);
  }
  __device__ static void st1(__half* p, float a, float inv, uint32_t& seen) {
    const __half h = __float2half_rn(a * inv);
    *p = h;
    track(seen, __halves2half2(h, h));
  }
  // exponent all ones in either half: +-inf or NaN
  __device__ static bool bad(uint32_t seen) {
    return (seen & 0x7C00u) == 0x7C00u || (seen & 0x7C000000u) == 0x7C000000u;
  }
};

template <>
struct Store<__nv_bfloat16> {
  static constexpr bool kScaled = true;
  __device__ static float2 ld2(const __nv_bfloat16* p, float sc) {
    const float2 v = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
    return make_float2(v.x * sc, v.y * sc);
  }
  __device__ static void track(uint32_t& seen, uint32_t bits) {
    __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162*>(&seen);
    m = __hmax2_nan(m, __habs2(*reinterpret_cast<const __nv_bfloat162*>(&bits)));
    seen = *reinterpret_cast<const uint32_t*>(&m);
  }
  __device__ static void st2(__nv_bfloat16* p, float a, float b, float inv, uint32_t& seen) {
    const uint32_t lo = bf16_rne_bits(a * inv), hi = bf16_rne_bits(b * inv);
    *reinterpret_cast<uint32_t*>(p) = lo | (hi << 16);
    track(seen, lo | (hi << 16));
  }
  __device__ static void st1(__nv_bfloat16* p, float a, float inv, uint32_t& seen) {
    const uint32_t v = bf16_rne_bits(a * inv);
    *reinterpret_cast<uint16_t*>(p) = (uint16_t)v;
    track(seen, v | (v << 16));
  }
  __device__ static bool bad(uint32_t seen) {
    return (seen & 0x7F80u) == 0x7F80u || (seen & 0x7F800000u) == 0x7F800000u;
  }
};

// W = 64: one 64-cell row per warp (32 lanes x an x-pair).  W = 32: two 32-cell rows per warp
// (16 lanes x an x-pair each), so a CTA of the same 16 warps covers a 32 x 32 tile instead of
// 64 x 16: more of it valid under the trapezoid and a finer x granularity on small grids.
template <typename S, int B, int TY, int W = 64, typename SH = S>
struct Tiled2 {
  static constexpr int ESZ_E = (int)sizeof(S);    // stored E value
  static constexpr int ESZ_H = (int)sizeof(SH);   // stored H value
  static constexpr int ESZ = ESZ_E < ESZ_H ? ESZ_E : ESZ_H;
  static constexpr int LPR = W / 2;            // lanes per tile row
  static constexpr int THREADS = TY * LPR;
  static constexpr int WB = W + kTiled2BoxPad;  // box width of fields and material ids
  static constexpr int MBX = WB;
  static constexpr int PL = WB * TY;           // elements of one staged field plane
  static constexpr int PLX = W * TY;           // elements of one y-exchange plane
  static constexpr int MPL = MBX * TY;         // elements of one staged material plane
  static constexpr int MPL_S = (MPL * 2 + 127) / 128 * 64;  // its stage stride: 128-byte steps
  static constexpr int NS = ESZ_E + ESZ_H == 8 ? kTiled2Stages : kTiled2Stages + 1;
  static constexpr int SX = tiled2_sx_w(W, B);
  static constexpr int SY = tiled_sy(B, TY);
  static constexpr int XBASE = tiled2_xbase(B);
  static constexpr uint32_t OFF_HPLANES = 3u * PL * ESZ_E;  // H planes follow E in a stage
  static constexpr uint32_t STAGE_F_BYTES = 3u * PL * (ESZ_E + ESZ_H);
  static constexpr uint32_t STAGE_M_BYTES = MPL_S * 2u;  // TMA destinations stay 128-aligned
  static constexpr uint32_t TX_BYTES = STAGE_F_BYTES + MPL * 2u;  // bytes the copies deliver
  static constexpr size_t OFF_M = (size_t)NS * STAGE_F_BYTES;
  static constexpr size_t OFF_H = OFF_M + (size_t)NS * STAGE_M_BYTES;
  static constexpr size_t OFF_E = OFF_H + 2u * 2u * PLX * 4u;
  static constexpr size_t OFF_BAR = OFF_E + (size_t)B * 2u * PLX * 4u;
  static constexpr size_t SMEM = OFF_BAR + NS * 8u + 128u;  // + alignment slack
  static_assert(SMEM <= 227u * 1024u, "shared memory per CTA");
  static_assert(SX % 2 == 0 && XBASE % 2 == 0 && XBASE + B <= 0, "even tile starts");
  static_assert(SY >= 1, "tile too short for this BLT");
  static_assert((W == 64 || W == 32) && THREADS % 32 == 0, "warp rows of 64 or 32 cells");
  static_assert(STAGE_M_BYTES % 128 == 0 && (PL * ESZ) % 128 == 0, "stage alignment");
  static_assert(STAGE_F_BYTES % 128 == 0, "stage alignment");
};

__device__ __forceinline__ float2 ldf2(const float* p) {
  return *reinterpret_cast<const float2*>(p);
}
__device__ __forceinline__ void stf2(float* p, float2 v) {
  *reinterpret_cast<float2*>(p) = v;
}

// Shared-memory carve-up of one CTA (all tiles it processes reuse it).
struct Smem {
  unsigned char* base;
  uint64_t* bars;
  int* abort;
};

// Runs the z-march of one tile (tile column (bx, by), z-chunk bz) of the grid described by `a`.
// `gbase` counts the pipeline stages this CTA consumed before (mbarrier phases continue across
// tiles in the persistent form).  Every thread of the CTA calls it; returns false when a
// bounded wait expired (the CTA must then stop).
//
// Two forms of the per-level update, chosen per warp and z-iteration (warp-uniform, so the
// barriers and shuffles stay common):
//  * lean: every cell of the warp carries material a.lean_id in all planes this iteration
//    touches, no source is in range and the planes are off the z faces.  Then Ca = Da = 1 and
//    one Cb / Db for all axes, so E' = E + Cb*curl: paired FP32 subtractions and additions
//    (.f32x2) on the x-pair and separately rounded products; cells on an x or y face (or
//    outside the grid) are restored by a select;
//  * general: per-cell coefficients from the material table, face cells left unchanged,
//    sources applied; separately rounded scalar arithmetic.
// Both evaluate the same operations in the same order per cell, so they agree bit for bit.
//
// LO (lean only): the whole tile holds a.lean_id and no source (see tile_uniform), so every
// iteration takes the lean path; the z faces are restored by the same select, and the material
// planes are neither loaded nor tested.
template <typename S, int B, int TY, int W = 64, typename SH = S, bool LO = false>
__device__ __forceinline__ bool march(const TiledArgs& a, int bx, int by, int bz,
                                      const Smem& sm, uint32_t& gbase, long long t_offset) {
  using K = Tiled2<S, B, TY, W, SH>;
  using St = Store<S>;    // E components
  using StH = Store<SH>;  // H components
  unsigned char* st_f = sm.base;  // per stage: Ex Ey Ez as S, then Hx Hy Hz as SH
  uint16_t* st_m = reinterpret_cast<uint16_t*>(sm.base + K::OFF_M);
  float* hbuf = reinterpret_cast<float*>(sm.base + K::OFF_H);  // [2][Hz,Hx][PLX]
  float* ebuf = reinterpret_cast<float*>(sm.base + K::OFF_E);  // [B][Ex,Ez][PLX]
  uint64_t* bars = sm.bars;

  const Grid g = a.g;
  const int z0 = bz * a.zlen;
  if (z0 >= g.nz) return true;  // uniform across the CTA
  const int z1 = min(g.nz, z0 + a.zlen);
  const int ps = z0 - B;
  const int niter = (z1 - z0) + 2 * B;

  const int lx = threadIdx.x % K::LPR;                                   // pair in the row
  const int ly = threadIdx.y * (32 / K::LPR) + threadIdx.x / K::LPR;     // tile row
  const int tid = threadIdx.y * 32 + threadIdx.x;
  const int X = bx * K::SX + K::XBASE;  // even; the boxes start at X8
  const int Y = by * K::SY - B;
  const int X8 = X & ~7;
  const int cx0 = 2 * lx;               // tile column of the even cell
  const int x0 = X + cx0, x1 = x0 + 1, y = Y + ly;
  const bool row_int = y >= 1 && y <= g.ny - 2;
  const bool int0 = row_int && x0 >= 1 && x0 <= g.nx - 2;
  const bool int1 = row_int && x1 >= 1 && x1 <= g.nx - 2;
  const bool row_out = ly >= B && ly < TY - B && y >= 0 && y < g.ny;
  const bool out0 = row_out && cx0 >= B && cx0 < B + K::SX && x0 >= 0 && x0 < g.nx;
  const bool out1 = row_out && cx0 + 1 >= B && cx0 + 1 < B + K::SX && x1 >= 0 && x1 < g.nx;
  unsigned smask = 0;
  for (int n = 0; n < a.S.n; ++n) {
    const SourceDev& s = a.S.s[n];
    const bool hit = s.kind == 0 ? (s.j == y && (s.i == x0 || s.i == x1)) : (int0 || int1);
    if (hit) smask |= 1u << n;
  }
  // CTA-uniform z-iteration ranges in which some level touches a source plane inside this tile
  // or a monitor plane: E at plane p-s+1 and H at plane p-s for s = 1..B.  Outside them the
  // per-level source and monitor code is skipped by every warp.
  int src_lo = 1 << 30, src_hi = -(1 << 30), mon_lo = 1 << 30, mon_hi = -(1 << 30);
  for (int n = 0; n < a.S.n; ++n) {
    const SourceDev& s = a.S.s[n];
    if (s.kind == 0 && (s.i < X || s.i >= X + W || s.j < Y || s.j >= Y + TY)) continue;
    src_lo = min(src_lo, s.k);
    src_hi = max(src_hi, s.k + B);
  }
  for (int n = 0; n < a.M.n; ++n) {
    const int k = a.M.m[n].k + (a.M.m[n].comp < 3 ? 0 : 1);  // E at p-s+1, H at p-s
    mon_lo = min(mon_lo, k);
    mon_hi = max(mon_hi, k + B - 1);
  }
  float sc[6], inv[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    const bool scaled = c < 3 ? St::kScaled : StH::kScaled;
    sc[c] = scaled ? a.scale[c] : 1.0f;
    inv[c] = scaled ? a.inv_scale[c] : 1.0f;
  }
  // Lean-path state, warp-uniform: wface = some cell of the warp lies on an x or y face or
  // outside the grid (the lean path then keeps those cells' values with a select); uh bit q =
  // every cell of the warp in plane p-q holds lean_id.  Planes below the chunk's first loaded
  // plane count as lean: what the warm-up computes there is discarded whatever the coefficients
  // (outputs at planes >= z0 depend on loaded planes only), so the first iterations of a chunk
  // need not take the general path.
  const bool lean_on = a.lean != 0;
  const bool wface = !__all_sync(kFull, int0 && int1);
  const uint32_t lean_ids = (uint32_t)a.lean_id * 0x10001u;
  constexpr uint32_t kPlanes = (1u << (B + 1)) - 1u;
  uint32_t uh = ~0u;

  for (int q = tid; q < (4 + 2 * B) * K::PLX; q += K::THREADS) hbuf[q] = 0.0f;
  __syncthreads();  // zeroed exchange planes; the previous tile's stages are all consumed

  const long long wait_limit = a.wait_limit > 0 ? a.wait_limit : kWaitLimit;
  const bool fault_tile = a.fault_bx == bx && a.fault_by == by && a.fault_bz == bz;
  auto issue = [&](int it_) {
    if (fault_tile && it_ == a.fault_it) return;  // test hook: this copy is never issued
    const uint32_t u = gbase + (uint32_t)it_;
    const int stage = (int)(u % K::NS);
    uint64_t* bar = &bars[stage];
    mbar_arrive_expect_tx(bar, LO ? K::STAGE_F_BYTES : K::TX_BYTES);
    unsigned char* d = st_f + stage * K::STAGE_F_BYTES;
    S* de = reinterpret_cast<S*>(d);
    SH* dh = reinterpret_cast<SH*>(d + K::OFF_HPLANES);
    const int pz = ps + it_;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      tma_load_3d(de + c * K::PL, &a.tm_src[c], bar, X8, Y, pz);
      tma_load_3d(dh + c * K::PL, &a.tm_src[3 + c], bar, X8, Y, pz);
    }
    if (!LO) tma_load_3d(st_m + stage * K::MPL_S, &a.tm_mat, bar, X8, Y, pz);
  };
  if (tid == 0) {
    fence_proxy_async_smem();
    for (int it_ = 0; it_ < K::NS && it_ < niter; ++it_) issue(it_);
  }

  // Ep[s][c] / Hp[s][c]: level-s values of this thread's pair one iteration ago.
  float2 Ep[B + 1][3], Hp[B + 1][3];
#pragma unroll
  for (int s = 0; s <= B; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) Ep[s][c] = Hp[s][c] = make_float2(0.0f, 0.0f);
  uint32_t mq[B + 1];  // packed material ids (even | odd << 16) of planes p, p-1, ..., p-B
#pragma unroll
  for (int s = 0; s <= B; ++s) mq[s] = 0;

  // y-exchange planes: W per row; staged planes (fields and ids): WB per row from X8
  const int o = ly * W + cx0;
  const int oym = (ly > 0 ? ly - 1 : 0) * W + cx0;
  const int oyp = (ly < TY - 1 ? ly + 1 : TY - 1) * W + cx0;
  const int xoff = X - X8;                   // even, 0..6
  const int os = ly * K::WB + cx0 + xoff;    // even: aligned pair loads
  const int osym = (ly > 0 ? ly - 1 : 0) * K::WB + cx0 + xoff;
  const int om = ly * K::MBX + cx0 + xoff;   // even: a 4-byte aligned id pair
  const float dx = a.dx;
  const long long pitch = g.pitch, plane = g.plane;
  S* const* dst = reinterpret_cast<S* const*>(a.dst.f);        // E components
  SH* const* dsth = reinterpret_cast<SH* const*>(a.dst.f + 3);  // H components

  uint32_t seen_e = 0, seen_h = 0;  // 16-bit storage: running max |stored value| (see Store)
  int it = 0;
  bool abort = false;
  for (; it < niter; ++it) {
    const int p = ps + it;
    const uint32_t u = gbase + (uint32_t)it;
    const int stage = (int)(u % K::NS);
    if (!mbar_wait_bounded(&bars[stage], (u / K::NS) & 1u, wait_limit)) {
      *sm.abort = 1;
      atomicOr(a.err, kErrTimeout);
    }
    if (B == 1) __syncthreads();  // orders last iteration's ebuf writes before this read
    const bool mon_iter = p >= mon_lo && p <= mon_hi;
    const bool src_iter = smask != 0 && p >= src_lo && p <= src_hi;

    const S* E0 = reinterpret_cast<const S*>(st_f + stage * K::STAGE_F_BYTES);
    const SH* H0 = reinterpret_cast<const SH*>(st_f + stage * K::STAGE_F_BYTES + K::OFF_HPLANES);
    bool lean = true;
    if (!LO) {
#pragma unroll
      for (int s = B; s >= 1; --s) mq[s] = mq[s - 1];
      mq[0] = *reinterpret_cast<const uint32_t*>(st_m + stage * K::MPL_S + om);
      uh = (uh << 1) | (__all_sync(kFull, mq[0] == lean_ids) ? 1u : 0u);
      lean = lean_on && (uh & kPlanes) == kPlanes && p >= B + 1 && p <= g.nz - 2 && !src_iter;
    }
    float2 Hc[3], Eo[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Hc[c] = StH::ld2(H0 + c * K::PL + os, sc[3 + c]);
      Eo[c] = St::ld2(E0 + c * K::PL + os, sc[c]);
    }
    float2 hz_ym = StH::ld2(H0 + 2 * K::PL + osym, sc[5]);
    float2 hx_ym = StH::ld2(H0 + osym, sc[3]);
    float2 EnPrev[3] = {};
    float2 EnB[3] = {}, HnB[3] = {};

#pragma unroll
    for (int s = 1; s <= B; ++s) {
      const int e = p - s + 1;
      const long long t = a.t0 + t_offset + (s - 1);
      // Inputs of both updates.  E^s(e): x-1 neighbours = odd cell of lane-1 for the even cell,
      // own even cell for the odd cell.  H^s(e-1): x+1 neighbours = own odd cell for the even
      // cell, even cell of lane+1 for the odd cell; y+1 neighbours of level-s E at plane e-1
      // from the exchange plane written one iteration ago.
      const float hz_xm = __shfl_up_sync(kFull, Hc[2].y, 1, K::LPR);
      const float hy_xm = __shfl_up_sync(kFull, Hc[1].y, 1, K::LPR);
      const float ez_xp = __shfl_down_sync(kFull, Ep[s][2].x, 1, K::LPR);
      const float ey_xp = __shfl_down_sync(kFull, Ep[s][1].x, 1, K::LPR);
      float* eb = ebuf + (s - 1) * 2 * K::PLX;
      const float2 ex_yp = ldf2(eb + oyp), ez_yp = ldf2(eb + K::PLX + oyp);
      float2 En[3], Hn[3];
      if (lean) {
        // ---------------- E^s(e), H^s(e-1): Ca = Da = 1, one Cb and Db, paired adds
        const float2 hzxm = make_float2(hz_xm, Hc[2].x), hyxm = make_float2(hy_xm, Hc[1].x);
        const float2 ex_c = sub2(sub2(Hc[2], hz_ym), sub2(Hc[1], Hp[s - 1][1]));
        const float2 ey_c = sub2(sub2(Hc[0], Hp[s - 1][0]), sub2(Hc[2], hzxm));
        const float2 ez_c = sub2(sub2(Hc[1], hyxm), sub2(Hc[0], hx_ym));
        En[0] = add2(Eo[0], scale2(a.lean_cb, ex_c));
        En[1] = add2(Eo[1], scale2(a.lean_cb, ey_c));
        En[2] = add2(Eo[2], scale2(a.lean_cb, ez_c));
        const bool ke = !LO || (e >= 1 && e <= g.nz - 2);  // mixed tiles: lean only off z faces
        if (wface || !ke) {  // face and outside cells keep their value
          const bool u0 = int0 && ke, u1 = int1 && ke;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            En[c].x = u0 ? En[c].x : Eo[c].x;
            En[c].y = u1 ? En[c].y : Eo[c].y;
          }
        }
        const float2 ezxp = make_float2(Ep[s][2].y, ez_xp), eyxp = make_float2(Ep[s][1].y, ey_xp);
        const float2 hx_c = sub2(sub2(En[1], Ep[s][1]), sub2(ez_yp, Ep[s][2]));
        const float2 hy_c = sub2(sub2(ezxp, Ep[s][2]), sub2(En[0], Ep[s][0]));
        const float2 hz_c = sub2(sub2(ex_yp, Ep[s][0]), sub2(eyxp, Ep[s][1]));
        Hn[0] = add2(Hp[s - 1][0], scale2(a.lean_db, hx_c));
        Hn[1] = add2(Hp[s - 1][1], scale2(a.lean_db, hy_c));
        Hn[2] = add2(Hp[s - 1][2], scale2(a.lean_db, hz_c));
        const bool kh = !LO || (e - 1 >= 1 && e - 1 <= g.nz - 2);
        if (wface || !kh) {
          const bool u0 = int0 && kh, u1 = int1 && kh;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            Hn[c].x = u0 ? Hn[c].x : Hp[s - 1][c].x;
            Hn[c].y = u1 ? Hn[c].y : Hp[s - 1][c].y;
          }
        }
      } else {
        // ---------------- E^s(e): per-cell coefficients, sources, faces unchanged
        float2 cxp, cyp, czp;
        cxp.x = sub(sub(Hc[2].x, hz_ym.x), sub(Hc[1].x, Hp[s - 1][1].x));
        cxp.y = sub(sub(Hc[2].y, hz_ym.y), sub(Hc[1].y, Hp[s - 1][1].y));
        cyp.x = sub(sub(Hc[0].x, Hp[s - 1][0].x), sub(Hc[2].x, hz_xm));
        cyp.y = sub(sub(Hc[0].y, Hp[s - 1][0].y), sub(Hc[2].y, Hc[2].x));
        czp.x = sub(sub(Hc[1].x, hy_xm), sub(Hc[0].x, hx_ym.x));
        czp.y = sub(sub(Hc[1].y, Hc[1].x), sub(Hc[0].y, hx_ym.y));
        En[0] = Eo[0];
        En[1] = Eo[1];
        En[2] = Eo[2];
        if (e >= 1 && e <= g.nz - 2) {
          if (src_iter) {
            float v;
            if (source_value(a.S, 0, x0, y, e, t, &v)) cxp.x = sub(cxp.x, mul(v, dx));
            if (source_value(a.S, 1, x0, y, e, t, &v)) cyp.x = sub(cyp.x, mul(v, dx));
            if (source_value(a.S, 2, x0, y, e, t, &v)) czp.x = sub(czp.x, mul(v, dx));
            if (source_value(a.S, 0, x1, y, e, t, &v)) cxp.y = sub(cxp.y, mul(v, dx));
            if (source_value(a.S, 1, x1, y, e, t, &v)) cyp.y = sub(cyp.y, mul(v, dx));
            if (source_value(a.S, 2, x1, y, e, t, &v)) czp.y = sub(czp.y, mul(v, dx));
          }
          const Material* m0 = a.table + (mq[s - 1] & 0xFFFFu);
          const Material* m1 = a.table + (mq[s - 1] >> 16);
          // E needs {Cax, Cbx, Cay, Cby} and {Caz, Cbz}: 6 of the 12 words per cell
          const float4 a0 = __ldg(&m0->a), a1 = __ldg(&m1->a);
          const float2 b0 = __ldg(reinterpret_cast<const float2*>(&m0->b));
          const float2 b1 = __ldg(reinterpret_cast<const float2*>(&m1->b));
          if (int0) {
            En[0].x = yee(a0.x, Eo[0].x, a0.y, cxp.x);
            En[1].x = yee(a0.z, Eo[1].x, a0.w, cyp.x);
            En[2].x = yee(b0.x, Eo[2].x, b0.y, czp.x);
          }
          if (int1) {
            En[0].y = yee(a1.x, Eo[0].y, a1.y, cxp.y);
            En[1].y = yee(a1.z, Eo[1].y, a1.w, cyp.y);
            En[2].y = yee(b1.x, Eo[2].y, b1.y, czp.y);
          }
        }
        // ---------------- H^s(e-1)
        cxp.x = sub(sub(En[1].x, Ep[s][1].x), sub(ez_yp.x, Ep[s][2].x));
        cxp.y = sub(sub(En[1].y, Ep[s][1].y), sub(ez_yp.y, Ep[s][2].y));
        cyp.x = sub(sub(Ep[s][2].y, Ep[s][2].x), sub(En[0].x, Ep[s][0].x));
        cyp.y = sub(sub(ez_xp, Ep[s][2].y), sub(En[0].y, Ep[s][0].y));
        czp.x = sub(sub(ex_yp.x, Ep[s][0].x), sub(Ep[s][1].y, Ep[s][1].x));
        czp.y = sub(sub(ex_yp.y, Ep[s][0].y), sub(ey_xp, Ep[s][1].y));
        Hn[0] = Hp[s - 1][0];
        Hn[1] = Hp[s - 1][1];
        Hn[2] = Hp[s - 1][2];
        if (e - 1 >= 1 && e - 1 <= g.nz - 2) {
          if (src_iter) {
            float v;
            if (source_value(a.S, 3, x0, y, e - 1, t, &v)) cxp.x = sub(cxp.x, mul(v, dx));
            if (source_value(a.S, 4, x0, y, e - 1, t, &v)) cyp.x = sub(cyp.x, mul(v, dx));
            if (source_value(a.S, 5, x0, y, e - 1, t, &v)) czp.x = sub(czp.x, mul(v, dx));
            if (source_value(a.S, 3, x1, y, e - 1, t, &v)) cxp.y = sub(cxp.y, mul(v, dx));
            if (source_value(a.S, 4, x1, y, e - 1, t, &v)) cyp.y = sub(cyp.y, mul(v, dx));
            if (source_value(a.S, 5, x1, y, e - 1, t, &v)) czp.y = sub(czp.y, mul(v, dx));
          }
          const Material* m0 = a.table + (mq[s] & 0xFFFFu);
          const Material* m1 = a.table + (mq[s] >> 16);
          // H needs {Dax, Dbx} and {Day, Dby, Daz, Dbz}
          const float2 b0 = __ldg(reinterpret_cast<const float2*>(&m0->b) + 1);
          const float2 b1 = __ldg(reinterpret_cast<const float2*>(&m1->b) + 1);
          const float4 c0 = __ldg(&m0->c), c1 = __ldg(&m1->c);
          if (int0) {
            Hn[0].x = yee(b0.x, Hp[s - 1][0].x, b0.y, cxp.x);
            Hn[1].x = yee(c0.x, Hp[s - 1][1].x, c0.y, cyp.x);
            Hn[2].x = yee(c0.z, Hp[s - 1][2].x, c0.w, czp.x);
          }
          if (int1) {
            Hn[0].y = yee(b1.x, Hp[s - 1][0].y, b1.y, cxp.y);
            Hn[1].y = yee(c1.x, Hp[s - 1][1].y, c1.y, cyp.y);
            Hn[2].y = yee(c1.z, Hp[s - 1][2].y, c1.w, czp.y);
          }
        }
      }
      // ---------------- DFT monitors: stage the FP32 values (before any storage rounding)
      if (mon_iter && (out0 || out1)) {
        for (int n = 0; n < a.M.n; ++n) {
          const MonitorDev& m = a.M.m[n];
          const int mk = m.comp < 3 ? e : e - 1;
          if (m.k == mk && mk >= z0 && mk < z1) {
            const int c = m.comp < 3 ? m.comp : m.comp - 3;
            const float2 v = m.comp < 3 ? (c == 0 ? En[0] : (c == 1 ? En[1] : En[2]))
                                        : (c == 0 ? Hn[0] : (c == 1 ? Hn[1] : Hn[2]));
            if (out0) dft_record(m, t, x0, y, g, v.x);
            if (out1) dft_record(m, t, x1, y, g, v.y);
          }
        }
      }
      // ---------------- exchange
      if (s < B) {
        float* hb = hbuf + (s & 1) * 2 * K::PLX;
        stf2(hb + o, Hn[2]);
        stf2(hb + K::PLX + o, Hn[0]);
      }
      __syncthreads();
      stf2(eb + o, En[0]);
      stf2(eb + K::PLX + o, En[2]);
      if (s == 1) {
        abort = *sm.abort != 0;
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
        const float* hb = hbuf + (s & 1) * 2 * K::PLX;
        hz_ym = ldf2(hb + oym);
        hx_ym = ldf2(hb + K::PLX + oym);
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
    const int eB = p - B + 1, hB = p - B;
    const long long idx_e = x0 + (long long)y * pitch + (long long)eB * plane;
    const long long idx_h = idx_e - plane;
    const bool st_e = eB >= z0 && eB < z1, st_h = hB >= z0 && hB < z1;  // CTA-uniform
    if (out0 && out1) {  // the common case: both cells of the pair
      if (st_e) {
#pragma unroll
        for (int c = 0; c < 3; ++c) St::st2(dst[c] + idx_e, EnB[c].x, EnB[c].y, inv[c], seen_e);
      }
      if (st_h) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
          StH::st2(dsth[c] + idx_h, HnB[c].x, HnB[c].y, inv[3 + c], seen_h);
      }
    } else if (out0 || out1) {  // one cell: a tile edge at odd x, or the last column of odd Nx
      const int q = out0 ? 0 : 1;
      if (st_e) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
          St::st1(dst[c] + idx_e + q, q ? EnB[c].y : EnB[c].x, inv[c], seen_e);
      }
      if (st_h) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
          StH::st1(dsth[c] + idx_h + q, q ? HnB[c].y : HnB[c].x, inv[3 + c], seen_h);
      }
    }
  }

  if (St::bad(seen_e) || StH::bad(seen_h)) atomicOr(a.err, kErrNumeric);
  if (abort) {
    if (tid == 0) {
      // Let copies that were already issued land before the shared memory is released.
      for (int q = it + 1; q < niter && q < it + K::NS; ++q) {
        const uint32_t uq = gbase + (uint32_t)q;
        (void)mbar_wait_bounded(&bars[uq % K::NS], (uq / K::NS) & 1u, kWaitLimit / 8);
      }
    }
    return false;
  }
  gbase += (uint32_t)niter;
  return true;
}

// Whether tile (bx, by, bz) of the grid in `a` may run the lean-only z-march: every in-grid cell
// of its staged box over all planes it loads is in a uniform block of the lean material, and no
// source lies in that box.  Cells outside the grid never change on the lean path either (a
// select keeps them).  Every thread of the CTA calls it; the answer is CTA-uniform.
template <typename S, int B, int TY, int W, typename SH>
__device__ __forceinline__ bool tile_uniform(const TiledArgs& a, int bx, int by, int bz) {
  using K = Tiled2<S, B, TY, W, SH>;
  const Grid& g = a.g;
  const int z0 = bz * a.zlen;
  bool ok = a.ublk != nullptr && z0 < g.nz;
  if (ok) {
    const int X8 = (bx * K::SX + K::XBASE) & ~7, Y = by * K::SY - B;
    const int za = max(0, z0 - B), zb = min(g.nz, min(g.nz, z0 + a.zlen) + B);  // [za, zb)
    const int xa = max(0, X8), xb = min(g.nx, X8 + K::WB), ya = max(0, Y), yb = min(g.ny, Y + TY);
    for (int n = 0; n < a.S.n; ++n) {
      const SourceDev& s = a.S.s[n];
      const bool in_z = s.k >= za - 1 && s.k <= zb;
      if (in_z && (s.kind != 0 || (s.i >= xa && s.i < xb && s.j >= ya && s.j < yb))) ok = false;
    }
    if (ok && xa < xb && ya < yb) {
      const int bx0 = xa / kUniX, bx1 = (xb - 1) / kUniX, by0 = ya / kUniY, by1 = (yb - 1) / kUniY;
      const int bz0 = za / kUniZ, bz1 = (zb - 1) / kUniZ;
      const int nxb = bx1 - bx0 + 1, nyb = by1 - by0 + 1;
      const int nblk = nxb * nyb * (bz1 - bz0 + 1);
      const int tid = threadIdx.y * 32 + threadIdx.x;
      for (int q = tid; q < nblk; q += K::THREADS) {
        const int qx = bx0 + q % nxb, qy = by0 + (q / nxb) % nyb, qz = bz0 + q / (nxb * nyb);
        ok = ok && a.ublk[((long long)qz * a.uby + qy) * a.ubx + qx] != 0;
      }
    }
  }
  return __syncthreads_and(ok) != 0;
}

template <typename S, int B, int TY, int W = 64, typename SH = S>
__device__ __forceinline__ Smem setup_smem(unsigned char* smem_raw, int* s_abort) {
  using K = Tiled2<S, B, TY, W, SH>;
  unsigned char* base = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  Smem sm{base, reinterpret_cast<uint64_t*>(base + K::OFF_BAR), s_abort};
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    *s_abort = 0;
    for (int s = 0; s < K::NS; ++s) mbar_init(&sm.bars[s], 1);
    fence_mbar_init();
  }
  return sm;
}

// One grid: one tile per CTA.  MINB > 1 caps registers so that MINB CTAs fit on an SM (more
// warps to hide latency, at the cost of some spilled state); the autotuner decides.
template <typename S, int B, int TY, int MINB, int W = 64, typename SH = S>
__global__ void __launch_bounds__(TY * W / 2, MINB)
    fdtd_tiled2(const __grid_constant__ TiledArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ int s_abort;
  const Smem sm = setup_smem<S, B, TY, W, SH>(smem_raw, &s_abort);
  uint32_t gbase = 0;
  int bx = (int)blockIdx.x, by = (int)blockIdx.y, bz = (int)blockIdx.z;
  if (a.tile_order) {
    const int q = a.tile_order[bx + (int)gridDim.x * (by + (int)gridDim.y * bz)];
    bx = q % (int)gridDim.x;
    by = (q / (int)gridDim.x) % (int)gridDim.y;
    bz = q / ((int)gridDim.x * (int)gridDim.y);
  }
  if (tile_uniform<S, B, TY, W, SH>(a, bx, by, bz))
    (void)march<S, B, TY, W, SH, true>(a, bx, by, bz, sm, gbase, 0);
  else
    (void)march<S, B, TY, W, SH, false>(a, bx, by, bz, sm, gbase, 0);
}

// CTAs per SM the compiler must fit: two for the 24-row tiles of 32-cell rows (384 threads, the
// register budget of the 48-row instance), one otherwise.
template <int TY, int W>
constexpr int batch_min_blocks() {
  return (W == 32 && TY == 24) ? 2 : 1;
}

// A batch of independent grids: persistent CTAs pull (grid, tile) work items from a queue.
template <typename S, int B, int TY, int W = 64, typename SH = S>
__global__ void __launch_bounds__(TY * W / 2, (batch_min_blocks<TY, W>()))
    fdtd_tiled2_batch(const BatchArgs b) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ int s_abort;
  __shared__ int s_item;
  const Smem sm = setup_smem<S, B, TY, W, SH>(smem_raw, &s_abort);
  const int tid = threadIdx.y * 32 + threadIdx.x;
  uint32_t gbase = 0;
  while (true) {
    __syncthreads();  // every thread is done with the previous item (and s_item)
    if (tid == 0) s_item = (int)atomicAdd(b.counter, 1u);
    __syncthreads();
    const int item = s_item;
    if (item >= b.nitems) break;
    const int4 w = b.items[item];  // {grid, bx, by, bz}
    const TiledArgs& a = b.grids[b.flip * b.ngrids + w.x];
    const bool ok = tile_uniform<S, B, TY, W, SH>(a, w.y, w.z, w.w)
                        ? march<S, B, TY, W, SH, true>(a, w.y, w.z, w.w, sm, gbase, b.t_offset)
                        : march<S, B, TY, W, SH, false>(a, w.y, w.z, w.w, sm, gbase, b.t_offset);
    if (!ok) break;
  }
}

template <typename S, int B, int TY, int MINB, int W = 64, typename SH = S>
cudaError_t launch_one2(const TiledArgs& a, dim3 grid, cudaStream_t st) {
  using K = Tiled2<S, B, TY, W, SH>;
  cudaError_t e = cudaFuncSetAttribute(fdtd_tiled2<S, B, TY, MINB, W, SH>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::SMEM);
  if (e != cudaSuccess) return e;
  fdtd_tiled2<S, B, TY, MINB, W, SH><<<grid, dim3(32, K::THREADS / 32), K::SMEM, st>>>(a);
  return cudaGetLastError();
}

template <typename S, int B, int TY, int W = 64, typename SH = S>
cudaError_t launch_batch_one(const BatchArgs& b, int ctas, cudaStream_t st) {
  using K = Tiled2<S, B, TY, W, SH>;
  cudaError_t e = cudaFuncSetAttribute(fdtd_tiled2_batch<S, B, TY, W, SH>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::SMEM);
  if (e != cudaSuccess) return e;
  fdtd_tiled2_batch<S, B, TY, W, SH><<<ctas, dim3(32, K::THREADS / 32), K::SMEM, st>>>(b);
  return cudaGetLastError();
}

// 32-wide rows (two per warp): 24 rows (12 warps, BLT 1-2, registers capped for two CTAs per
// SM), 32 rows (16 warps, BLT 1-3) or 48 rows (24 warps, BLT 1-2).
template <typename S, typename SH = S>
cudaError_t launch_pairs32(int blt, int rows, const TiledArgs& a, dim3 grid, cudaStream_t st) {
  if (rows == 24) {
    switch (blt) {
      case 1: return launch_one2<S, 1, 24, 2, 32, SH>(a, grid, st);
      case 2: return launch_one2<S, 2, 24, 2, 32, SH>(a, grid, st);
      default: break;
    }
  } else if (rows == 32) {
    switch (blt) {
      case 1: return launch_one2<S, 1, 32, 1, 32, SH>(a, grid, st);
      case 2: return launch_one2<S, 2, 32, 1, 32, SH>(a, grid, st);
      case 3: return launch_one2<S, 3, 32, 1, 32, SH>(a, grid, st);
      default: break;
    }
  } else if (rows == 48) {
    switch (blt) {
      case 1: return launch_one2<S, 1, 48, 1, 32, SH>(a, grid, st);
      case 2: return launch_one2<S, 2, 48, 1, 32, SH>(a, grid, st);
      default: break;
    }
  }
  return cudaErrorInvalidValue;
}

template <typename S, typename SH = S>
cudaError_t launch_batch_pairs32(int blt, int rows, const BatchArgs& b, int ctas,
                                 cudaStream_t st) {
  if (rows == 24) {
    switch (blt) {
      case 1: return launch_batch_one<S, 1, 24, 32, SH>(b, ctas, st);
      case 2: return launch_batch_one<S, 2, 24, 32, SH>(b, ctas, st);
      default: break;
    }
  } else if (rows == 32) {
    switch (blt) {
      case 1: return launch_batch_one<S, 1, 32, 32, SH>(b, ctas, st);
      case 2: return launch_batch_one<S, 2, 32, 32, SH>(b, ctas, st);
      case 3: return launch_batch_one<S, 3, 32, 32, SH>(b, ctas, st);
      default: break;
    }
  } else if (rows == 48) {
    switch (blt) {
      case 1: return launch_batch_one<S, 1, 48, 32, SH>(b, ctas, st);
      case 2: return launch_batch_one<S, 2, 48, 32, SH>(b, ctas, st);
      default: break;
    }
  }
  return cudaErrorInvalidValue;
}

template <typename S, int TY, typename SH = S>
cudaError_t launch_rows2(int blt, int min_blocks, const TiledArgs& a, dim3 grid,
                         cudaStream_t st) {
  if (min_blocks > 1) {
    // register-capped FP32 variants: two CTAs of 16 rows or four of 8 rows per SM
    if constexpr (sizeof(S) == 4 && sizeof(SH) == 4 && TY == 16) {
      if (blt == 2 && min_blocks == 2) return launch_one2<S, 2, 16, 2>(a, grid, st);
    }
    if constexpr (sizeof(S) == 4 && sizeof(SH) == 4 && TY == 8) {
      if (blt == 2 && min_blocks == 4) return launch_one2<S, 2, 8, 4>(a, grid, st);
    }
    return cudaErrorInvalidValue;
  }
  switch (blt) {
    case 1: return launch_one2<S, 1, TY, 1, 64, SH>(a, grid, st);
    case 2: return launch_one2<S, 2, TY, 1, 64, SH>(a, grid, st);
    case 3: if constexpr (TY <= 20) return launch_one2<S, 3, TY, 1, 64, SH>(a, grid, st); break;
    case 4: if constexpr (TY == 16) return launch_one2<S, 4, TY, 1, 64, SH>(a, grid, st); break;
    default: break;
  }
  return cudaErrorInvalidValue;
}

template <typename S, typename SH = S>
cudaError_t launch_type2(const TiledConfig& c, const TiledArgs& a, dim3 grid, cudaStream_t st) {
  switch (c.rows) {
    case 8: return launch_rows2<S, 8, SH>(c.blt, c.min_blocks, a, grid, st);
    case 16: return launch_rows2<S, 16, SH>(c.blt, c.min_blocks, a, grid, st);
    case 20:  // FP32: 640 threads, the register file's limit at ~96 registers per thread
      if constexpr (sizeof(S) == 4 && sizeof(SH) == 4)
        return launch_rows2<S, 20>(c.blt, c.min_blocks, a, grid, st);
      break;
    case 24:
      if constexpr (sizeof(S) == 4 && sizeof(SH) == 4)
        return launch_rows2<S, 24>(c.blt, c.min_blocks, a, grid, st);
      break;
    case 32:
      if constexpr (sizeof(S) == 4 && sizeof(SH) == 4)
        return launch_rows2<S, 32>(c.blt, c.min_blocks, a, grid, st);
      break;
    default: break;
  }
  return cudaErrorInvalidValue;
}

template <typename S, typename SH = S>
cudaError_t launch_batch_type(const TiledConfig& c, const BatchArgs& b, int ctas,
                              cudaStream_t st) {
  if (c.rows == 16) {
    switch (c.blt) {
      case 1: return launch_batch_one<S, 1, 16, 64, SH>(b, ctas, st);
      case 2: return launch_batch_one<S, 2, 16, 64, SH>(b, ctas, st);
      case 3: return launch_batch_one<S, 3, 16, 64, SH>(b, ctas, st);
      case 4: return launch_batch_one<S, 4, 16, 64, SH>(b, ctas, st);
      default: break;
    }
  } else if (c.rows == 8) {
    switch (c.blt) {
      case 1: return launch_batch_one<S, 1, 8, 64, SH>(b, ctas, st);
      case 2: return launch_batch_one<S, 2, 8, 64, SH>(b, ctas, st);
      case 3: return launch_batch_one<S, 3, 8, 64, SH>(b, ctas, st);
      default: break;
    }
  } else if constexpr (sizeof(S) == 4 && sizeof(SH) == 4) {
    if (c.rows == 20) {
      switch (c.blt) {
        case 1: return launch_batch_one<S, 1, 20>(b, ctas, st);
        case 2: return launch_batch_one<S, 2, 20>(b, ctas, st);
        case 3: return launch_batch_one<S, 3, 20>(b, ctas, st);
        default: break;
      }
    } else if (c.rows == 24) {
      switch (c.blt) {
        case 1: return launch_batch_one<S, 1, 24>(b, ctas, st);
        case 2: return launch_batch_one<S, 2, 24>(b, ctas, st);
        default: break;
      }
    }
  }
  return cudaErrorInvalidValue;
}

template <typename S, int B, int TY, int W = 64, typename SH = S>
size_t smem_of() {
  return Tiled2<S, B, TY, W, SH>::SMEM;
}

template <typename S, int B, int TY, int W = 64, typename SH = S>
int occupancy_of() {
  using K = Tiled2<S, B, TY, W, SH>;
  int n = 0;
  cudaFuncSetAttribute(fdtd_tiled2_batch<S, B, TY, W, SH>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::SMEM);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fdtd_tiled2_batch<S, B, TY, W, SH>,
                                                    K::THREADS, K::SMEM) != cudaSuccess)
    return 1;
  return n > 0 ? n : 1;
}

// Shared memory (SMEM) or resident batch CTAs per SM (OCC) of the batch instance for config c.
template <typename S, typename SH, bool OCC>
size_t batch_query(const TiledConfig& c) {
#define GD_Q(B, TY, W) (OCC ? (size_t)occupancy_of<S, B, TY, W, SH>() : smem_of<S, B, TY, W, SH>())
  constexpr bool f32 = sizeof(S) == 4 && sizeof(SH) == 4;
  if (c.pairs32) {
    if (c.rows == 24) {
      switch (c.blt) {
        case 1: return GD_Q(1, 24, 32);
        case 2: return GD_Q(2, 24, 32);
      }
    } else if (c.rows == 32) {
      switch (c.blt) {
        case 1: return GD_Q(1, 32, 32);
        case 2: return GD_Q(2, 32, 32);
        case 3: return GD_Q(3, 32, 32);
      }
    } else if (c.rows == 48) {
      switch (c.blt) {
        case 1: return GD_Q(1, 48, 32);
        case 2: return GD_Q(2, 48, 32);
      }
    }
  } else if (c.rows == 16) {
    switch (c.blt) {
      case 1: return GD_Q(1, 16, 64);
      case 2: return GD_Q(2, 16, 64);
      case 3: return GD_Q(3, 16, 64);
      case 4: return GD_Q(4, 16, 64);
    }
  } else if (c.rows == 8) {
    switch (c.blt) {
      case 1: return GD_Q(1, 8, 64);
      case 2: return GD_Q(2, 8, 64);
      case 3: return GD_Q(3, 8, 64);
    }
  } else if constexpr (f32) {
    if (c.rows == 20) {
      switch (c.blt) {
        case 1: return GD_Q(1, 20, 64);
        case 2: return GD_Q(2, 20, 64);
        case 3: return GD_Q(3, 20, 64);
      }
    } else if (c.rows == 24) {
      switch (c.blt) {
        case 1: return GD_Q(1, 24, 64);
        case 2: return GD_Q(2, 24, 64);
      }
    }
  }
#undef GD_Q
  return OCC ? 1 : 0;
}

}  // namespace

// Per-storage entry points (one translation unit each: k_tiled2_<storage>.cu).
#define GD_TILED2_DECL(TAG)                                                                 \
  cudaError_t tiled2_launch_##TAG(const TiledConfig& c, const TiledArgs& a, dim3 grid,       \
                                  cudaStream_t st);                                          \
  cudaError_t tiled2_batch_launch_##TAG(const TiledConfig& c, const BatchArgs& b, int ctas,  \
                                        cudaStream_t st);                                    \
  size_t tiled2_batch_query_##TAG(const TiledConfig& c, bool occupancy);
GD_TILED2_DECL(f32)
GD_TILED2_DECL(f16)
GD_TILED2_DECL(bf16)
GD_TILED2_DECL(f16e)
#undef GD_TILED2_DECL

}  // namespace fdtd
