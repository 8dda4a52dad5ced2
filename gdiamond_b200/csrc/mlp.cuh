// mlp.cuh -- definitions shared by the surrogate MLP's GEMM kernels (mlp.cu: mma.sync family
// and host code; mlp_tc.cu: tcgen05 / TMEM family).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace fdtd {
namespace mlp {

enum Epi { kStore = 0, kBias = 1, kBiasGelu = 2, kGeluBack = 3, kBiasGeluAct = 4 };

// op(X)(r, k) = T ? X[k*ld + r] : X[r*ld + k] (+ member * stride)
struct Operand {
  const __nv_bfloat16* p;
  int ld;
  long long stride;  // per member (elements); 0 = shared by all members
  bool vec;          // 16-byte loads allowed (ld, stride multiples of 8, base 16-byte aligned)
};

struct Epilogue {
  float* out;              // C (kStore), Z (kBias, kBiasGelu), G (kGeluBack)
  __nv_bfloat16* out_bf;   // A (kBiasGelu, kBiasGeluAct), Gbf (kGeluBack)
  const float* bias;       // kBias, kBiasGelu, kBiasGeluAct
  const float* zp;         // kGeluBack: pre-activation of the layer below, same shape as out
  int ldc;
  long long stride_out, stride_bias, stride_zp;
};

// GELU with the exact (erf) form and its derivative.
__device__ __forceinline__ float gelu(float z) {
  return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) +
         z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// The fused epilogue of one accumulator element (member e, row r, column c).
template <int EPI>
__device__ __forceinline__ void epilogue_store(const Epilogue& ep, int e, int r, int c, float v) {
  const long long o = (long long)r * ep.ldc + c;
  if (EPI == kBias || EPI == kBiasGelu || EPI == kBiasGeluAct) v += ep.bias[e * ep.stride_bias + c];
  if (EPI == kGeluBack) v *= gelu_grad(ep.zp[e * ep.stride_zp + o]);
  if (EPI != kBiasGeluAct) ep.out[e * ep.stride_out + o] = v;  // inference keeps no Z
  if (EPI == kBiasGelu || EPI == kBiasGeluAct)
    ep.out_bf[e * ep.stride_out + o] = __float2bfloat16_rn(gelu(v));
  if (EPI == kGeluBack) ep.out_bf[e * ep.stride_out + o] = __float2bfloat16_rn(v);
}

// Fused ensemble inference (mlp_tc.cu): every layer of one member for 256 rows per CTA.
constexpr int kFusedMaxLayers = 8;
struct FusedArgs {
  const float* x;                  // [n][dims[0]] FP32 inputs
  long long n;
  int L;                           // layers
  int dims[kFusedMaxLayers + 1];
  long long w_off[kFusedMaxLayers], b_off[kFusedMaxLayers];
  const __nv_bfloat16* wbf;        // [members][P] BF16 weights
  const float* params;             // [members][P] FP32 parameters (biases)
  long long P;
  float* out;                      // [members][out_stride]: [n][dims[L]] per member
  long long out_stride;
  int* err;
};
// dims[0] <= 64; every other width a multiple of 32 up to 256.
bool mlp_fused_supported(const int* dims, int L);
cudaError_t launch_mlp_fused(const FusedArgs& a, int members, cudaStream_t st);

// tcgen05 GEMM (mlp_tc.cu): C[M][N] (+epilogue) for `members` members on `st`; `err` receives
// a nonzero word if a bounded wait inside the kernel gave up.  Instantiated for the epilogues
// the MLP uses (mlp_tc.cu lists them).
template <bool TA, bool TB, int EPI>
cudaError_t launch_gemm_tc(int M, int N, int K, const Operand& A, const Operand& B,
                           const Epilogue& ep, int members, cudaStream_t st, int* err);

}  // namespace mlp
}  // namespace fdtd
