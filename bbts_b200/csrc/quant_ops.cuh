// FP8-E4M3 per-block quantisation kernels (templates, so several translation
// units may include them) and the launcher both quantisation entry points use.
//
// A block is quantised in two passes: the absmax of the block, then
// q = e4m3(x * 448 / absmax). The launcher runs both passes of one block back
// to back, so for blocks that fit in L2 the second read is an L2 hit and the
// block crosses HBM once each way.
//
// Fast paths (16-byte aligned pointers, sizes that are whole vectors):
//  * k_absmax_v: 16-byte loads, four in flight per thread, one atomicMax per CTA;
//  * k_quant_e4m3_v: 16-byte loads, 8 packed e4m3 bytes stored per thread;
//  * k_quant_e4m3_t (transpose): 64 x 128 input tiles through shared memory,
//    each thread quantising a 4 x 8 sub-block and packing 4 output bytes of a
//    column into one word, then 16-byte stores along the output rows.
// k_absmax / k_quant_e4m3 remain the general element-wise forms for the rest.
// Every path computes the same values: x * s in f32, then a saturating
// round-to-nearest-even conversion to e4m3.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace bbx {

// Block absmax into *amax (float bits compared as integers; values are >= 0;
// NaN inputs are ignored by fmaxf).
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

__device__ __forceinline__ float quant_scale(const unsigned int* amax) {
  const float a = __uint_as_float(*amax);
  return a > 0.f ? 448.f / a : 1.f;
}

__device__ __forceinline__ void write_scale(const unsigned int* amax, float* scale_out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const float a = __uint_as_float(*amax);
    *scale_out = a > 0.f ? a / 448.f : 1.f;
  }
}

// q = e4m3(x * 448 / amax); *scale_out = amax / 448 (the dequantisation factor).
// With transpose != 0 the rows x cols input is written as cols x rows, which
// turns an MN-major operand into the K-major layout the FP8 MMA reads.
template <typename T>
__global__ void k_quant_e4m3(const T* __restrict__ in, __nv_fp8_e4m3* out, int rows, int cols,
                             const unsigned int* amax, float* scale_out, int transpose) {
  const float s = quant_scale(amax);
  write_scale(amax, scale_out);
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

// ------------------------------------------------------------------ vector forms
// 8 consecutive elements as f32 (p 16-byte aligned).
__device__ __forceinline__ void load8(const float* p, float v[8]) {
  const float4 a = __ldg((const float4*)p), b = __ldg((const float4*)p + 1);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
__device__ __forceinline__ void load8(const __nv_bfloat16* p, float v[8]) {
  const uint4 u = __ldg((const uint4*)p);
  const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[2 * k] = __uint_as_float(w[k] << 16);
    v[2 * k + 1] = __uint_as_float(w[k] & 0xFFFF0000u);
  }
}

// Two e4m3 bytes (lo = a) of x * s, saturating round-to-nearest-even.
__device__ __forceinline__ uint32_t q2(float a, float b, float s) {
  return (uint32_t)__nv_cvt_float2_to_fp8x2(make_float2(a * s, b * s), __NV_SATFINITE, __NV_E4M3);
}

constexpr int kQuantThreads = 256;

// A batch of blocks quantised by one launch of each pass: block y of the grid
// (blockIdx.y) works on in[y] / out[y] / scale[y] with absmax word amax[y].
constexpr int kQuantBatchMax = 64;
template <typename T>
struct QuantBatch {
  const T* in[kQuantBatchMax];
  uint8_t* out[kQuantBatchMax];
  float* scale[kQuantBatchMax];
  unsigned int* amax;
};

template <typename T>
__global__ void __launch_bounds__(kQuantThreads) k_absmax_v(const __grid_constant__ QuantBatch<T> b, long long n8) {
  const T* __restrict__ in = b.in[blockIdx.y];
  unsigned int* amax = b.amax + blockIdx.y;
  float m = 0.f;
  const long long stride = (long long)gridDim.x * blockDim.x;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (; i + 3 * stride < n8; i += 4 * stride) {
    float v[4][8];
#pragma unroll
    for (int u = 0; u < 4; ++u) load8(in + (i + u * stride) * 8, v[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int k = 0; k < 8; ++k) m = fmaxf(m, fabsf(v[u][k]));
  }
  for (; i < n8; i += stride) {
    float v[8];
    load8(in + i * 8, v);
#pragma unroll
    for (int k = 0; k < 8; ++k) m = fmaxf(m, fabsf(v[k]));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ float wm[kQuantThreads / 32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int w = 1; w < kQuantThreads / 32; ++w) m = fmaxf(m, wm[w]);
    atomicMax(amax, __float_as_uint(m));
  }
}

// Row-major output: 8 elements in, 8 packed bytes out per step.
template <typename T>
__global__ void __launch_bounds__(kQuantThreads) k_quant_e4m3_v(const __grid_constant__ QuantBatch<T> b, long long n8) {
  const T* __restrict__ in = b.in[blockIdx.y];
  uint8_t* out = b.out[blockIdx.y];
  const unsigned int* amax = b.amax + blockIdx.y;
  float* scale_out = b.scale[blockIdx.y];
  const float s = quant_scale(amax);
  write_scale(amax, scale_out);
  const long long stride = (long long)gridDim.x * blockDim.x;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (; i + stride < n8; i += 2 * stride) {
    float v[2][8];
    load8(in + i * 8, v[0]);
    load8(in + (i + stride) * 8, v[1]);
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      uint2 q;
      q.x = q2(v[u][0], v[u][1], s) | (q2(v[u][2], v[u][3], s) << 16);
      q.y = q2(v[u][4], v[u][5], s) | (q2(v[u][6], v[u][7], s) << 16);
      *(uint2*)(out + (i + u * stride) * 8) = q;
    }
  }
  if (i < n8) {
    float v[8];
    load8(in + i * 8, v);
    uint2 q;
    q.x = q2(v[0], v[1], s) | (q2(v[2], v[3], s) << 16);
    q.y = q2(v[4], v[5], s) | (q2(v[6], v[7], s) << 16);
    *(uint2*)(out + i * 8) = q;
  }
}

// Transposed output (cols x rows) through a 64 (rows) x 128 (cols) tile.
// Thread t quantises rows r0 + 4 (t % 16) .. +3, cols c0 + 8 (t / 16) .. +7
// and stores, for each of its 8 columns, the 4 bytes of its rows as one word
// of smem row c (18 words per row: 16 data + 2 pad, so the 32 lanes of a
// store hit 32 banks). The output phase writes each tile column's 64 bytes as
// four 16-byte stores. Requires rows % 16 == 0, cols % 8 == 0, 16-byte
// aligned pointers.
constexpr int kQtR = 64, kQtC = 128, kQtWords = 18;

template <typename T>
__global__ void __launch_bounds__(kQuantThreads) k_quant_e4m3_t(const __grid_constant__ QuantBatch<T> b, int rows,
                                                                int cols) {
  const T* __restrict__ in = b.in[blockIdx.y];
  uint8_t* out = b.out[blockIdx.y];
  const unsigned int* amax = b.amax + blockIdx.y;
  float* scale_out = b.scale[blockIdx.y];
  __shared__ __align__(16) uint32_t tile[kQtC * kQtWords];
  const float s = quant_scale(amax);
  write_scale(amax, scale_out);
  const int tiles_c = (cols + kQtC - 1) / kQtC;
  const long long tiles = (long long)tiles_c * ((rows + kQtR - 1) / kQtR);
  const int rg = threadIdx.x & 15, cg = threadIdx.x >> 4;
  for (long long tl = blockIdx.x; tl < tiles; tl += gridDim.x) {
    const int r0 = (int)(tl / tiles_c) * kQtR, c0 = (int)(tl % tiles_c) * kQtC;
    const int c = c0 + 8 * cg;
    float v[4][8];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = r0 + 4 * rg + j;
      if (r < rows && c < cols) {
        load8(in + (long long)r * cols + c, v[j]);
      } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) v[j][k] = 0.f;
      }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t w = q2(v[0][k], v[1][k], s) | (q2(v[2][k], v[3][k], s) << 16);
      tile[(8 * cg + k) * kQtWords + rg] = w;
    }
    __syncthreads();
    // 128 columns x 4 chunks of 16 bytes
#pragma unroll
    for (int e = threadIdx.x; e < kQtC * 4; e += kQuantThreads) {
      const int cc = e >> 2, qq = e & 3;
      const int oc = c0 + cc, orow = r0 + 16 * qq;
      if (oc < cols && orow < rows) {
        const uint2 lo = *(const uint2*)&tile[cc * kQtWords + 4 * qq];
        const uint2 hi = *(const uint2*)&tile[cc * kQtWords + 4 * qq + 2];
        *(uint4*)(out + (long long)oc * rows + orow) = make_uint4(lo.x, lo.y, hi.x, hi.y);
      }
    }
    __syncthreads();
  }
}

// Enqueues the absmax and quantisation passes of `count` blocks (each rows x
// cols) on `st`: block i reads in[i], writes out[i] and scales[i], with absmax
// word amax[i], which must hold 0 when the first pass runs. When every block
// qualifies for the vector kernels, each pass is one launch per 64 blocks
// (grid.y = block); otherwise each block takes the element-wise kernels.
// Returns the launch error, if any.
template <typename T>
inline cudaError_t launch_quantize_batch(const T* const* in, uint8_t* const* out, int count, int rows, int cols,
                                         int transpose, unsigned int* amax, float* scales, int sms, cudaStream_t st) {
  const long long n = (long long)rows * cols;
  const long long cap = (long long)sms * 8;
  bool a16 = n % 8 == 0, o16 = true, o8 = true;
  for (int i = 0; i < count; ++i) {
    a16 = a16 && ((uintptr_t)in[i] & 15) == 0;
    o16 = o16 && ((uintptr_t)out[i] & 15) == 0;
    o8 = o8 && ((uintptr_t)out[i] & 7) == 0;
  }
  const bool vec_abs = a16;
  const bool vec_q = !transpose && a16 && o8;
  const bool vec_t = transpose && a16 && o16 && rows % 16 == 0 && cols % 8 == 0;
  for (int b0 = 0; b0 < count; b0 += kQuantBatchMax) {
    const int cnt = count - b0 < kQuantBatchMax ? count - b0 : kQuantBatchMax;
    QuantBatch<T> qb;
    for (int i = 0; i < cnt; ++i) {
      qb.in[i] = in[b0 + i];
      qb.out[i] = out[b0 + i];
      qb.scale[i] = scales + b0 + i;
    }
    qb.amax = amax + b0;
    const long long per = cap / cnt > 1 ? cap / cnt : 1;  // CTAs per block: about 8 per SM in all
    if (vec_abs) {
      const long long n8 = n / 8;
      long long g = (n8 + kQuantThreads * 4 - 1) / (kQuantThreads * 4);
      g = g < 1 ? 1 : g > per ? per : g;
      k_absmax_v<T><<<dim3((unsigned)g, (unsigned)cnt), kQuantThreads, 0, st>>>(qb, n8);
    } else {
      long long g = (n + 255) / 256;
      g = g < 1 ? 1 : g > cap ? cap : g;
      for (int i = 0; i < cnt; ++i) k_absmax<T><<<(int)g, 256, 0, st>>>(qb.in[i], n, qb.amax + i);
    }
    if (vec_q) {
      const long long n8 = n / 8;
      long long g = (n8 + kQuantThreads * 2 - 1) / (kQuantThreads * 2);
      g = g < 1 ? 1 : g > per ? per : g;
      k_quant_e4m3_v<T><<<dim3((unsigned)g, (unsigned)cnt), kQuantThreads, 0, st>>>(qb, n8);
    } else if (vec_t) {
      const long long tiles = (long long)((cols + kQtC - 1) / kQtC) * ((rows + kQtR - 1) / kQtR);
      const long long g = tiles < per ? tiles : per;
      k_quant_e4m3_t<T><<<dim3((unsigned)g, (unsigned)cnt), kQuantThreads, 0, st>>>(qb, rows, cols);
    } else {
      long long g = (n + 255) / 256;
      g = g < 1 ? 1 : g > cap ? cap : g;
      for (int i = 0; i < cnt; ++i)
        k_quant_e4m3<T><<<(int)g, 256, 0, st>>>(qb.in[i], (__nv_fp8_e4m3*)qb.out[i], rows, cols, qb.amax + i,
                                                qb.scale[i], transpose);
    }
  }
  return cudaGetLastError();
}

}  // namespace bbx
