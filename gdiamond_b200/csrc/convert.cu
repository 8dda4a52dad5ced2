// convert.cu -- conversion of stored field arrays (FP16 / BF16 with a per-component scale, FP64)
// to and from FP32 / FP64 for the C-ABI's field transfers.  Pitched layout on both sides; one
// thread per element of a row, grid (ceil(nx/128), ny, nz).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <type_traits>

#include "fdtd_kernels.cuh"

namespace fdtd {
namespace {

template <typename S>
__device__ __forceinline__ double load_as(const void* p, long long i);
template <>
__device__ __forceinline__ double load_as<float>(const void* p, long long i) {
  return (double)static_cast<const float*>(p)[i];
}
template <>
__device__ __forceinline__ double load_as<__half>(const void* p, long long i) {
  return (double)__half2float(static_cast<const __half*>(p)[i]);
}
template <>
__device__ __forceinline__ double load_as<__nv_bfloat16>(const void* p, long long i) {
  return (double)__bfloat162float(static_cast<const __nv_bfloat16*>(p)[i]);
}
template <>
__device__ __forceinline__ double load_as<double>(const void* p, long long i) {
  return static_cast<const double*>(p)[i];
}

template <typename S, typename D>
__global__ void to_wide(Grid g, const void* src, float scale, D* dst) {
  const int i = blockIdx.x * 128 + threadIdx.x;
  if (i >= g.nx) return;
  const long long idx = i + (long long)blockIdx.y * g.pitch + (long long)blockIdx.z * g.plane;
  // FP32 and FP64 are stored unscaled; scaling by a power of two is exact in FP32.
  const double v = load_as<S>(src, idx);
  dst[idx] = (sizeof(S) == 2) ? (D)((float)v * scale) : (D)v;
}

template <typename S>
__global__ void from_f32(Grid g, const float* src, float inv_scale, S* dst) {
  const int i = blockIdx.x * 128 + threadIdx.x;
  if (i >= g.nx) return;
  const long long idx = i + (long long)blockIdx.y * g.pitch + (long long)blockIdx.z * g.plane;
  const float v = src[idx];
  if constexpr (sizeof(S) == 2) {
    if constexpr (std::is_same<S, __half>::value)
      dst[idx] = __float2half_rn(v * inv_scale);
    else
      *reinterpret_cast<uint16_t*>(dst + idx) = bf16_rne_bits(v * inv_scale);
  } else {
    dst[idx] = (S)v;
  }
}

dim3 conv_grid(const Grid& g) { return dim3((g.nx + 127) / 128, g.ny, g.nz); }

}  // namespace

cudaError_t convert_field_to_f32(const Grid& g, const void* src, int storage, float scale,
                                 float* dst, cudaStream_t st) {
  switch (storage) {
    case 0: to_wide<float, float><<<conv_grid(g), 128, 0, st>>>(g, src, scale, dst); break;
    case 1: to_wide<__half, float><<<conv_grid(g), 128, 0, st>>>(g, src, scale, dst); break;
    case 2: to_wide<__nv_bfloat16, float><<<conv_grid(g), 128, 0, st>>>(g, src, scale, dst); break;
    case 3: to_wide<double, float><<<conv_grid(g), 128, 0, st>>>(g, src, scale, dst); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t convert_field_to_f64(const Grid& g, const void* src, int storage, float scale,
                                 double* dst, cudaStream_t st) {
  switch (storage) {
    case 0: to_wide<float, double><<<conv_grid(g), 128, 0, st>>>(g, src, scale, dst); break;
    case 1: to_wide<__half, double><<<conv_grid(g), 128, 0, st>>>(g, src, scale, dst); break;
    case 2: to_wide<__nv_bfloat16, double><<<conv_grid(g), 128, 0, st>>>(g, src, scale, dst); break;
    case 3: to_wide<double, double><<<conv_grid(g), 128, 0, st>>>(g, src, scale, dst); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t convert_field_from_f32(const Grid& g, const float* src, int storage, float inv_scale,
                                   void* dst, cudaStream_t st) {
  switch (storage) {
    case 0: from_f32<float><<<conv_grid(g), 128, 0, st>>>(g, src, inv_scale, (float*)dst); break;
    case 1: from_f32<__half><<<conv_grid(g), 128, 0, st>>>(g, src, inv_scale, (__half*)dst); break;
    case 2:
      from_f32<__nv_bfloat16><<<conv_grid(g), 128, 0, st>>>(g, src, inv_scale,
                                                             (__nv_bfloat16*)dst);
      break;
    case 3: from_f32<double><<<conv_grid(g), 128, 0, st>>>(g, src, inv_scale, (double*)dst); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace fdtd
