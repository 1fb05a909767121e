// FP8-E4M3 per-block quantisation kernels (templates, so several translation
// units may include them).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cstdint>

namespace bbx {

// Block absmax into *amax (float bits compared as integers; values are >= 0).
template <typename T>
__global__ void k_absmax(const T* __restrict__ in, long long n, unsigned int* amax) {
  float m = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    float v;
    if constexpr (sizeof(T) == 4) v = in[i]; else v = __bfloat162float(in[i]);
    m = fmaxf(m, fabsf(v));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(amax, __float_as_uint(m));
}

// q = e4m3(x * 448 / amax); *scale_out = amax / 448 (the dequantisation factor).
// With transpose != 0 the rows x cols input is written as cols x rows, which
// turns an MN-major operand into the K-major layout the FP8 MMA reads.
template <typename T>
__global__ void k_quant_e4m3(const T* __restrict__ in, __nv_fp8_e4m3* out, int rows, int cols,
                             const unsigned int* amax, float* scale_out, int transpose) {
  const float a = __uint_as_float(*amax);
  const float s = a > 0.f ? 448.f / a : 1.f;
  if (blockIdx.x == 0 && threadIdx.x == 0) *scale_out = a > 0.f ? a / 448.f : 1.f;
  const long long n = (long long)rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    float v;
    if constexpr (sizeof(T) == 4) v = in[i]; else v = __bfloat162float(in[i]);
    long long o = i;
    if (transpose) {
      long long r = i / cols, c = i % cols;
      o = c * rows + r;
    }
    out[o] = __nv_fp8_e4m3(v * s);
  }
}

}  // namespace bbx
