// k_tiled2.cu -- the z-streaming temporally tiled Yee kernel with two cells per thread in x,
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
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "fdtd_kernels.cuh"

namespace fdtd {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr long long kWaitLimit = 2000000000LL;  // SM clocks, about one second

template <typename S>
struct Store;

template <>
struct Store<float> {
  static constexpr bool kScaled = false;
  __device__ static float2 ld2(const float* p, float) {
    return *reinterpret_cast<const float2*>(p);
  }
  __device__ static void st2(float* p, float a, float b, float) {
    *reinterpret_cast<float2*>(p) = make_float2(a, b);
  }
  __device__ static void st1(float* p, float a, float) { *p = a; }
};

template <>
struct Store<__half> {
  static constexpr bool kScaled = true;
  __device__ static float2 ld2(const __half* p, float sc) {
    const float2 v = __half22float2(*reinterpret_cast<const __half2*>(p));
    return make_float2(v.x * sc, v.y * sc);
  }
  __device__ static void st2(__half* p, float a, float b, float inv) {
    *reinterpret_cast<__half2*>(p) = __floats2half2_rn(a * inv, b * inv);
  }
  __device__ static void st1(__half* p, float a, float inv) { *p = __float2half_rn(a * inv); }
};

template <>
struct Store<__nv_bfloat16> {
  static constexpr bool kScaled = true;
  __device__ static float2 ld2(const __nv_bfloat16* p, float sc) {
    const float2 v = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
    return make_float2(v.x * sc, v.y * sc);
  }
  __device__ static void st2(__nv_bfloat16* p, float a, float b, float inv) {
    const uint32_t lo = bf16_rne_bits(a * inv), hi = bf16_rne_bits(b * inv);
    *reinterpret_cast<uint32_t*>(p) = lo | (hi << 16);
  }
  __device__ static void st1(__nv_bfloat16* p, float a, float inv) {
    *reinterpret_cast<uint16_t*>(p) = bf16_rne_bits(a * inv);
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

struct Pair {
  float a, b;  // even cell, odd cell
};

__device__ __forceinline__ float2 ldf2(const float* p) {
  return *reinterpret_cast<const float2*>(p);
}
__device__ __forceinline__ void stf2(float* p, float a, float b) {
  *reinterpret_cast<float2*>(p) = make_float2(a, b);
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
template <typename S, int B, int TY, int W = 64, typename SH = S>
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

  for (int q = tid; q < (4 + 2 * B) * K::PLX; q += K::THREADS) hbuf[q] = 0.0f;
  __syncthreads();  // zeroed exchange planes; the previous tile's stages are all consumed

  auto issue = [&](int it_) {
    const uint32_t u = gbase + (uint32_t)it_;
    const int stage = (int)(u % K::NS);
    uint64_t* bar = &bars[stage];
    mbar_arrive_expect_tx(bar, K::TX_BYTES);
    unsigned char* d = st_f + stage * K::STAGE_F_BYTES;
    S* de = reinterpret_cast<S*>(d);
    SH* dh = reinterpret_cast<SH*>(d + K::OFF_HPLANES);
    const int pz = ps + it_;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      tma_load_3d(de + c * K::PL, &a.tm_src[c], bar, X8, Y, pz);
      tma_load_3d(dh + c * K::PL, &a.tm_src[3 + c], bar, X8, Y, pz);
    }
    tma_load_3d(st_m + stage * K::MPL_S, &a.tm_mat, bar, X8, Y, pz);
  };
  if (tid == 0) {
    fence_proxy_async_smem();
    for (int it_ = 0; it_ < K::NS && it_ < niter; ++it_) issue(it_);
  }

  // Ep[s][c] / Hp[s][c]: level-s values of this thread's pair one iteration ago.
  Pair Ep[B + 1][3], Hp[B + 1][3];
#pragma unroll
  for (int s = 0; s <= B; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) Ep[s][c] = Hp[s][c] = Pair{0.0f, 0.0f};
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

  int it = 0;
  bool abort = false;
  for (; it < niter; ++it) {
    const int p = ps + it;
    const uint32_t u = gbase + (uint32_t)it;
    const int stage = (int)(u % K::NS);
    if (!mbar_wait_bounded(&bars[stage], (u / K::NS) & 1u, kWaitLimit)) {
      *sm.abort = 1;
      atomicExch(a.err, kErrTimeout);
    }
    if (B == 1) __syncthreads();  // orders last iteration's ebuf writes before this read
    const bool mon_iter = p >= mon_lo && p <= mon_hi;
    const bool src_iter = smask != 0 && p >= src_lo && p <= src_hi;

    const S* E0 = reinterpret_cast<const S*>(st_f + stage * K::STAGE_F_BYTES);
    const SH* H0 = reinterpret_cast<const SH*>(st_f + stage * K::STAGE_F_BYTES + K::OFF_HPLANES);
#pragma unroll
    for (int s = B; s >= 1; --s) mq[s] = mq[s - 1];
    mq[0] = *reinterpret_cast<const uint32_t*>(st_m + stage * K::MPL_S + om);
    Pair Hc[3], Eo[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float2 hv = StH::ld2(H0 + c * K::PL + os, sc[3 + c]);
      const float2 ev = St::ld2(E0 + c * K::PL + os, sc[c]);
      Hc[c] = Pair{hv.x, hv.y};
      Eo[c] = Pair{ev.x, ev.y};
    }
    float2 hz_ym = StH::ld2(H0 + 2 * K::PL + osym, sc[5]);
    float2 hx_ym = StH::ld2(H0 + osym, sc[3]);
    Pair EnPrev[3] = {};
    Pair EnB[3] = {}, HnB[3] = {};

#pragma unroll
    for (int s = 1; s <= B; ++s) {
      const int e = p - s + 1;
      const long long t = a.t0 + t_offset + (s - 1);
      // ---------------- E^s(e)
      // x-1 neighbour: odd cell of lane-1 for the even cell, own even cell for the odd cell
      const float hz_xm = __shfl_up_sync(kFull, Hc[2].b, 1, K::LPR);
      const float hy_xm = __shfl_up_sync(kFull, Hc[1].b, 1, K::LPR);
      Pair cxp, cyp, czp;
      cxp.a = sub(sub(Hc[2].a, hz_ym.x), sub(Hc[1].a, Hp[s - 1][1].a));
      cxp.b = sub(sub(Hc[2].b, hz_ym.y), sub(Hc[1].b, Hp[s - 1][1].b));
      cyp.a = sub(sub(Hc[0].a, Hp[s - 1][0].a), sub(Hc[2].a, hz_xm));
      cyp.b = sub(sub(Hc[0].b, Hp[s - 1][0].b), sub(Hc[2].b, Hc[2].a));
      czp.a = sub(sub(Hc[1].a, hy_xm), sub(Hc[0].a, hx_ym.x));
      czp.b = sub(sub(Hc[1].b, Hc[1].a), sub(Hc[0].b, hx_ym.y));
      Pair En[3] = {Eo[0], Eo[1], Eo[2]};
      if (e >= 1 && e <= g.nz - 2) {
        if (src_iter) {
          float v;
          if (source_value(a.S, 0, x0, y, e, t, &v)) cxp.a = sub(cxp.a, mul(v, dx));
          if (source_value(a.S, 1, x0, y, e, t, &v)) cyp.a = sub(cyp.a, mul(v, dx));
          if (source_value(a.S, 2, x0, y, e, t, &v)) czp.a = sub(czp.a, mul(v, dx));
          if (source_value(a.S, 0, x1, y, e, t, &v)) cxp.b = sub(cxp.b, mul(v, dx));
          if (source_value(a.S, 1, x1, y, e, t, &v)) cyp.b = sub(cyp.b, mul(v, dx));
          if (source_value(a.S, 2, x1, y, e, t, &v)) czp.b = sub(czp.b, mul(v, dx));
        }
        const Material* m0 = a.table + (mq[s - 1] & 0xFFFFu);
        const Material* m1 = a.table + (mq[s - 1] >> 16);
        const float4 a0 = __ldg(&m0->a), b0 = __ldg(&m0->b);
        const float4 a1 = __ldg(&m1->a), b1 = __ldg(&m1->b);
        if (int0) {
          En[0].a = yee(a0.x, Eo[0].a, a0.y, cxp.a);
          En[1].a = yee(a0.z, Eo[1].a, a0.w, cyp.a);
          En[2].a = yee(b0.x, Eo[2].a, b0.y, czp.a);
        }
        if (int1) {
          En[0].b = yee(a1.x, Eo[0].b, a1.y, cxp.b);
          En[1].b = yee(a1.z, Eo[1].b, a1.w, cyp.b);
          En[2].b = yee(b1.x, Eo[2].b, b1.y, czp.b);
        }
      }
      // ---------------- H^s(e-1)
      // x+1 neighbour: own odd cell for the even cell, even cell of lane+1 for the odd cell
      const float ez_xp = __shfl_down_sync(kFull, Ep[s][2].a, 1, K::LPR);
      const float ey_xp = __shfl_down_sync(kFull, Ep[s][1].a, 1, K::LPR);
      float* eb = ebuf + (s - 1) * 2 * K::PLX;
      const float2 ex_yp = ldf2(eb + oyp), ez_yp = ldf2(eb + K::PLX + oyp);
      cxp.a = sub(sub(En[1].a, Ep[s][1].a), sub(ez_yp.x, Ep[s][2].a));
      cxp.b = sub(sub(En[1].b, Ep[s][1].b), sub(ez_yp.y, Ep[s][2].b));
      cyp.a = sub(sub(Ep[s][2].b, Ep[s][2].a), sub(En[0].a, Ep[s][0].a));
      cyp.b = sub(sub(ez_xp, Ep[s][2].b), sub(En[0].b, Ep[s][0].b));
      czp.a = sub(sub(ex_yp.x, Ep[s][0].a), sub(Ep[s][1].b, Ep[s][1].a));
      czp.b = sub(sub(ex_yp.y, Ep[s][0].b), sub(ey_xp, Ep[s][1].b));
      Pair Hn[3] = {Hp[s - 1][0], Hp[s - 1][1], Hp[s - 1][2]};
      if (e - 1 >= 1 && e - 1 <= g.nz - 2) {
        if (src_iter) {
          float v;
          if (source_value(a.S, 3, x0, y, e - 1, t, &v)) cxp.a = sub(cxp.a, mul(v, dx));
          if (source_value(a.S, 4, x0, y, e - 1, t, &v)) cyp.a = sub(cyp.a, mul(v, dx));
          if (source_value(a.S, 5, x0, y, e - 1, t, &v)) czp.a = sub(czp.a, mul(v, dx));
          if (source_value(a.S, 3, x1, y, e - 1, t, &v)) cxp.b = sub(cxp.b, mul(v, dx));
          if (source_value(a.S, 4, x1, y, e - 1, t, &v)) cyp.b = sub(cyp.b, mul(v, dx));
          if (source_value(a.S, 5, x1, y, e - 1, t, &v)) czp.b = sub(czp.b, mul(v, dx));
        }
        const Material* m0 = a.table + (mq[s] & 0xFFFFu);
        const Material* m1 = a.table + (mq[s] >> 16);
        const float4 b0 = __ldg(&m0->b), c0 = __ldg(&m0->c);
        const float4 b1 = __ldg(&m1->b), c1 = __ldg(&m1->c);
        if (int0) {
          Hn[0].a = yee(b0.z, Hp[s - 1][0].a, b0.w, cxp.a);
          Hn[1].a = yee(c0.x, Hp[s - 1][1].a, c0.y, cyp.a);
          Hn[2].a = yee(c0.z, Hp[s - 1][2].a, c0.w, czp.a);
        }
        if (int1) {
          Hn[0].b = yee(b1.z, Hp[s - 1][0].b, b1.w, cxp.b);
          Hn[1].b = yee(c1.x, Hp[s - 1][1].b, c1.y, cyp.b);
          Hn[2].b = yee(c1.z, Hp[s - 1][2].b, c1.w, czp.b);
        }
      }
      // ---------------- DFT monitors: stage the FP32 values (before any storage rounding)
      if (mon_iter && (out0 || out1)) {
        for (int n = 0; n < a.M.n; ++n) {
          const MonitorDev& m = a.M.m[n];
          const int mk = m.comp < 3 ? e : e - 1;
          if (m.k == mk && mk >= z0 && mk < z1) {
            const int c = m.comp < 3 ? m.comp : m.comp - 3;
            const Pair v = m.comp < 3 ? (c == 0 ? En[0] : (c == 1 ? En[1] : En[2]))
                                      : (c == 0 ? Hn[0] : (c == 1 ? Hn[1] : Hn[2]));
            if (out0) dft_record(m, t, x0, y, g, v.a);
            if (out1) dft_record(m, t, x1, y, g, v.b);
          }
        }
      }
      // ---------------- exchange
      if (s < B) {
        float* hb = hbuf + (s & 1) * 2 * K::PLX;
        stf2(hb + o, Hn[2].a, Hn[2].b);
        stf2(hb + K::PLX + o, Hn[0].a, Hn[0].b);
      }
      __syncthreads();
      stf2(eb + o, En[0].a, En[0].b);
      stf2(eb + K::PLX + o, En[2].a, En[2].b);
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
    if (out0 || out1) {
      const int eB = p - B + 1, hB = p - B;
      const bool both = out0 && out1;
      if (eB >= z0 && eB < z1) {
        const long long idx = x0 + (long long)y * pitch + (long long)eB * plane;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (both) St::st2(dst[c] + idx, EnB[c].a, EnB[c].b, inv[c]);
          else if (out0) St::st1(dst[c] + idx, EnB[c].a, inv[c]);
          else St::st1(dst[c] + idx + 1, EnB[c].b, inv[c]);
        }
      }
      if (hB >= z0 && hB < z1) {
        const long long idx = x0 + (long long)y * pitch + (long long)hB * plane;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (both) StH::st2(dsth[c] + idx, HnB[c].a, HnB[c].b, inv[3 + c]);
          else if (out0) StH::st1(dsth[c] + idx, HnB[c].a, inv[3 + c]);
          else StH::st1(dsth[c] + idx + 1, HnB[c].b, inv[3 + c]);
        }
      }
    }
  }

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
  (void)march<S, B, TY, W, SH>(a, (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, sm, gbase,
                               0);
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
    if (!march<S, B, TY, W, SH>(a, w.y, w.z, w.w, sm, gbase, b.t_offset)) break;
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

bool pairs32_supported(const TiledConfig& c) {
  return (c.esz == 4 || c.esz == 2) && c.width == 32 && c.min_blocks == 1 &&
         ((c.rows == 32 && c.blt >= 1 && c.blt <= 3) ||
          ((c.rows == 24 || c.rows == 48) && c.blt >= 1 && c.blt <= 2));
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

bool tiled2_config_supported(const TiledConfig& c) {
  if (c.pairs32) return pairs32_supported(c) && c.z_chunks >= 1;
  if (c.esz != 4 && c.esz != 2) return false;
  if (c.rows != 8 && c.rows != 16 && c.rows != 20 && c.rows != 24 && c.rows != 32) return false;
  if (c.rows > 16 && c.esz != 4) return false;
  if (c.blt < 1 || c.blt > 4) return false;
  if ((c.rows == 8 || c.rows == 20) && c.blt > 3) return false;
  if ((c.rows == 24 || c.rows == 32) && c.blt > 2) return false;  // the pair state spills
  if (c.min_blocks > 1 && !(c.esz == 4 && c.blt == 2 &&
                            ((c.rows == 16 && c.min_blocks == 2) ||
                             (c.rows == 8 && c.min_blocks == 4))))
    return false;
  return c.z_chunks >= 1;
}

bool tiled2_batch_supported(const TiledConfig& c) {
  if (c.pairs32) return pairs32_supported(c);
  if (c.esz != 4 && c.esz != 2) return false;
  if (c.rows == 16) return c.blt >= 1 && c.blt <= 4;
  if (c.rows == 8) return c.blt >= 1 && c.blt <= 3;
  if (c.rows == 20) return c.esz == 4 && c.blt >= 1 && c.blt <= 3;
  if (c.rows == 24) return c.esz == 4 && c.blt >= 1 && c.blt <= 2;
  return false;
}

dim3 tiled2_grid(const TiledConfig& c, const Grid& g) {
  const int sx = tiled2_sx_w(c.pairs32 ? 32 : 64, c.blt), sy = tiled_sy(c.blt, c.rows);
  const int first = tiled2_xbase(c.blt) + c.blt;
  const int ntx = (g.nx - first + sx - 1) / sx;
  const int nty = (g.ny + sy - 1) / sy;
  const int zlen = (g.nz + c.z_chunks - 1) / c.z_chunks;
  const int nzc = (g.nz + zlen - 1) / zlen;
  return dim3(ntx, nty, nzc);
}

size_t tiled2_batch_smem(const TiledConfig& c) {
  switch (c.storage) {
    case 0: return batch_query<float, float, false>(c);
    case 1: return batch_query<__half, __half, false>(c);
    case 2: return batch_query<__nv_bfloat16, __nv_bfloat16, false>(c);
    case 4: return batch_query<__half, float, false>(c);
  }
  return 0;
}

int tiled2_batch_ctas_per_sm(const TiledConfig& c) {
  switch (c.storage) {
    case 0: return (int)batch_query<float, float, true>(c);
    case 1: return (int)batch_query<__half, __half, true>(c);
    case 2: return (int)batch_query<__nv_bfloat16, __nv_bfloat16, true>(c);
    case 4: return (int)batch_query<__half, float, true>(c);
  }
  return 1;
}

// storage: 0 FP32, 1 FP16, 2 BF16, 4 FP16 E with FP32 H.
cudaError_t launch_tiled2(const TiledConfig& c, const TiledArgs& a, const Grid& g,
                          cudaStream_t st) {
  if (!tiled2_config_supported(c)) return cudaErrorInvalidValue;
  const dim3 grid = tiled2_grid(c, g);
  if (c.pairs32) {
    switch (c.storage) {
      case 0: return launch_pairs32<float>(c.blt, c.rows, a, grid, st);
      case 1: return launch_pairs32<__half>(c.blt, c.rows, a, grid, st);
      case 2: return launch_pairs32<__nv_bfloat16>(c.blt, c.rows, a, grid, st);
      case 4: return launch_pairs32<__half, float>(c.blt, c.rows, a, grid, st);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (c.storage) {
    case 0: return launch_type2<float>(c, a, grid, st);
    case 1: return launch_type2<__half>(c, a, grid, st);
    case 2: return launch_type2<__nv_bfloat16>(c, a, grid, st);
    case 4: return launch_type2<__half, float>(c, a, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_tiled2_batch(const TiledConfig& c, const BatchArgs& b, int ctas,
                                cudaStream_t st) {
  if (!tiled2_batch_supported(c)) return cudaErrorInvalidValue;
  if (c.pairs32) {
    switch (c.storage) {
      case 0: return launch_batch_pairs32<float>(c.blt, c.rows, b, ctas, st);
      case 1: return launch_batch_pairs32<__half>(c.blt, c.rows, b, ctas, st);
      case 2: return launch_batch_pairs32<__nv_bfloat16>(c.blt, c.rows, b, ctas, st);
      case 4: return launch_batch_pairs32<__half, float>(c.blt, c.rows, b, ctas, st);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (c.storage) {
    case 0: return launch_batch_type<float>(c, b, ctas, st);
    case 1: return launch_batch_type<__half>(c, b, ctas, st);
    case 2: return launch_batch_type<__nv_bfloat16>(c, b, ctas, st);
    case 4: return launch_batch_type<__half, float>(c, b, ctas, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fdtd
