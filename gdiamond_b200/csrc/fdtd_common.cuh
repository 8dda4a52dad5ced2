// fdtd_common.cuh -- shared device definitions of the B200 FDTD (Yee) solver.
//
// HBM layout (both field sets, the material map and the per-cell coefficient arrays):
//   pitched x-fastest SoA, element (i, j, k) at i + j*P + k*P*Ny with P = Nx rounded up to a
//   multiple of 8, so every row starts on a 16-byte boundary (a TMA requirement) for 4- and
//   2-byte elements.  Pad columns i >= Nx are zero and never written.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fdtd {

constexpr int kMaxSources = 8;
constexpr int kMaxMonitors = 12;  // a flux monitor takes six
constexpr int kMaxFreqs = 64;
// Steps a monitor's staging ring holds between folds (a power of two): the tiled kernels write
// each monitor-plane value there, and a fold adds a window of them to the FP64 sums.
constexpr int kDftSlots = 128;

// Device error word: bits set with atomicOr.
constexpr int kErrNone = 0;
constexpr int kErrTimeout = 1;  // a bounded mbarrier wait gave up
constexpr int kErrNumeric = 2;  // a field value stored in 16 bits was +-inf or NaN

struct Grid {
  int nx, ny, nz;   // cells per axis
  int pitch;        // row pitch in elements
  long long plane;  // pitch * ny
};

struct SourceDev {
  int comp;   // 0..2 J (E update), 3..5 M (H update)
  int kind;   // 0 point, 1 interior of z-plane k
  int i, j, k;
};

struct Sources {
  int n;
  SourceDev s[kMaxSources];
  const float* wave;  // [n][tw]
  long long tw;
};

struct MonitorDev {
  int comp;          // field component 0..5
  int k;             // z-plane
  int nf;
  double scale;
  const double2* tab;  // [t][nf] (cos, sin) of ph = (2*pi*f) * (t*dt)
  double* re;          // [nf][ny][nx]
  double* im;
  float* stage;        // [kDftSlots][ny][nx] plane values of steps not yet folded (or null)
};

struct Monitors {
  int n;
  MonitorDev m[kMaxMonitors];
};

// Per-material coefficients, 48 bytes, grouped so the E update reads the first 24 bytes and
// the H update the last 24: {Cax, Cbx, Cay, Cby}, {Caz, Cbz, Dax, Dbx}, {Day, Dby, Daz, Dbz}.
struct __align__(16) Material {
  float4 a, b, c;
};

// -------------------------------------------------------------- exact arithmetic
// Every multiply and add is rounded separately (no contraction into FMA), which is how the
// reference's CPU build evaluates the update; the GPU results are then bit-identical to it.
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// Paired FP32 arithmetic (sm_100 `.f32x2`, CUDA's __fadd2_rn): one instruction for both cells
// of an x-pair, each half rounded to nearest even with subnormals kept, i.e. __fadd_rn applied
// to .x and .y; a - b is a + (-b), which IEEE arithmetic rounds identically (negation is exact).
// The fast-path tests compare the paired lean update with the scalar general update bit for bit.
// There is deliberately no paired multiply: a paired multiply followed by a paired add was
// evaluated as one paired fused multiply-add (even when both were written with an explicit .rn),
// whose single rounding differs from the reference's separately rounded product and sum;
// scale2 multiplies each half on its own (__fmul_rn is never fused).
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
__device__ __forceinline__ float2 scale2(float c, float2 v) {
  return make_float2(__fmul_rn(c, v.x), __fmul_rn(c, v.y));
}

// FP32 -> BF16 bit pattern, round to nearest even on the FP32 bits (subnormals included, NaN
// kept quiet).  Defined here rather than taken from a conversion instruction so the rounding
// of stored fields is specified exactly, the same on the device and in the oracle.
__host__ __device__ __forceinline__ uint16_t bf16_rne_bits(float x) {
#ifdef __CUDA_ARCH__
  const uint32_t b = __float_as_uint(x);
#else
  uint32_t b;
  __builtin_memcpy(&b, &x, 4);
#endif
  if ((b & 0x7FFFFFFFu) > 0x7F800000u) return (uint16_t)((b >> 16) | 0x0040u);
  return (uint16_t)((b + 0x7FFFu + ((b >> 16) & 1u)) >> 16);
}

// new = Ca*old + Cb*curl
__device__ __forceinline__ float yee(float ca, float old, float cb, float curl) {
  return add(mul(ca, old), mul(cb, curl));
}

// Source term of one component at cell (i,j,k) and step t: the sum of the waveforms of all
// sources of component comp that cover the cell, and whether any does.
__device__ __forceinline__ bool source_value(const Sources& S, int comp, int i, int j, int k,
                                             long long t, float* v) {
  float acc = 0.0f;
  bool any = false;
  for (int n = 0; n < S.n; ++n) {
    const SourceDev& s = S.s[n];
    if (s.comp != comp) continue;
    const bool hit = (s.kind == 0) ? (s.i == i && s.j == j && s.k == k) : (s.k == k);
    if (hit) {
      acc = add(acc, t < S.tw ? S.wave[n * S.tw + t] : 0.0f);
      any = true;
    }
  }
  *v = acc;
  return any;
}

// Running-DFT update of one cell: re += (v*c)*scale, im -= (v*s)*scale, for every frequency.
__device__ __forceinline__ void dft_accumulate(const MonitorDev& m, long long t, int i, int j,
                                               const Grid& g, float value) {
  const double v = (double)value;
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

// Monitor-plane value of step t at cell (i, j): into slot t % kDftSlots of the staging ring,
// to be folded into the sums later in step order (dft_fold.cu), or straight into the sums
// when the monitor has no ring.  Both give the same FP64 sums bit for bit.
__device__ __forceinline__ void dft_record(const MonitorDev& m, long long t, int i, int j,
                                           const Grid& g, float value) {
  if (m.stage) {
    const long long np = (long long)g.nx * g.ny;
    m.stage[(t & (kDftSlots - 1)) * np + i + (long long)j * g.nx] = value;
  } else {
    dft_accumulate(m, t, i, j, g, value);
  }
}

// -------------------------------------------------------- TMA / mbarrier (sm_90+)
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase of `parity` with a bound of about `limit_cycles` SM clocks.  Returns
// false (and never blocks longer) when the bound is reached.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  long long limit_cycles) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (clock64() - t0 > limit_cycles) return false;
  }
}

// Tiled 3-D TMA load global -> this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, uint64_t* bar, int x,
                                            int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace fdtd
