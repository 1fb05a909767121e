// HBM-streaming block kernels: add, n-ary reduce, elementwise, bias and
// column sums, casts / FP8 quantisation, softmax cross-entropy, Philox fill,
// and the rank<=4 permutation used by the contraction.
//
// All of them are grid-stride loops sized to a multiple of the SM count, use
// 128-bit loads/stores when the pointers allow it, and are bit-exact against
// the reference's CPU loops where the reference fixes the order of operations
// (add, left-fold reduce, relu, relu', hadamard, weighted sum, column sum).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cstdint>
#include "ptx.cuh"
#include "quant_ops.cuh"

namespace bbx {

enum UnaryOp : int {
  U_RELU = 0,        // dense_matrix_relu.cc:63-69
  U_RELU_DIF = 1,    // dense_matrix_relu_dif.cc:63-69 (1 if > 0 else 0)
  U_SIGMOID_REF = 2, // dense_matrix_sigmoid.cc:64-70: 1/(1+exp(v)) as the reference computes it
  U_SIGMOID = 3,     // 1/(1+exp(-v)), cutensor ew uop 0 (libraries/cutensor/ew.h:158-161)
  U_EXP = 4,
  U_SQUARE = 5,
  U_SQRT = 6,
  U_ADD_SCALAR = 7,  // v + param
  U_SCALE = 8,       // v * param
  U_RELU_LO = 9,     // relu(v) - bf16(relu(v)): the low part of a split activation (exact in f32)
};

enum BinaryOp : int {
  B_ADD = 0,          // dense_matrix_add.cc:67-73
  B_WEIGHTED = 1,     // dense_matrix_weighted_sum.cc:70-76: ca*a + cb*b
  B_HADAMARD = 2,     // dense_matrix_hadamard.cc:67-73
  B_MAX = 3,
  B_MIN = 4,
  B_SUB = 5,
  B_DIV = 6,
};

constexpr int kMaxReduceInputs = 32;

struct ReduceArgs {
  const float* in[kMaxReduceInputs];
};

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ float apply_unary(int op, float v, float p) {
  switch (op) {
    case U_RELU: return v > 0.f ? v : 0.f;
    case U_RELU_DIF: return v > 0.f ? 1.f : 0.f;
    case U_SIGMOID_REF: return __fdiv_rn(1.f, __fadd_rn(1.f, expf(v)));
    case U_SIGMOID: return __fdiv_rn(1.f, __fadd_rn(1.f, expf(-v)));
    case U_EXP: return expf(v);
    case U_SQUARE: return __fmul_rn(v, v);
    case U_SQRT: return sqrtf(v);
    case U_ADD_SCALAR: return __fadd_rn(v, p);
    case U_SCALE: return __fmul_rn(v, p);
    case U_RELU_LO: {
      const float r = v > 0.f ? v : 0.f;
      return __fsub_rn(r, __bfloat162float(__float2bfloat16_rn(r)));
    }
  }
  return v;
}

__device__ __forceinline__ float apply_binary(int op, float a, float b, float ca, float cb) {
  switch (op) {
    case B_ADD: return __fadd_rn(a, b);
    case B_WEIGHTED: return __fadd_rn(__fmul_rn(ca, a), __fmul_rn(cb, b));
    case B_HADAMARD: return __fmul_rn(a, b);
    case B_MAX: return a > b ? a : b;
    case B_MIN: return a < b ? a : b;
    case B_SUB: return __fsub_rn(a, b);
    case B_DIV: return __fdiv_rn(a, b);
  }
  return a;
}

// The same element functions as apply_unary / apply_binary (bit-identical),
// chosen once per call: `body` receives the function for `op`, so loops over
// elements carry no per-element dispatch.
template <typename Body>
__device__ __forceinline__ void with_unary(int op, float p, Body&& body) {
  switch (op) {
    case U_RELU: body([](float v) { return v > 0.f ? v : 0.f; }); break;
    case U_RELU_DIF: body([](float v) { return v > 0.f ? 1.f : 0.f; }); break;
    case U_SIGMOID_REF: body([](float v) { return __fdiv_rn(1.f, __fadd_rn(1.f, expf(v))); }); break;
    case U_SIGMOID: body([](float v) { return __fdiv_rn(1.f, __fadd_rn(1.f, expf(-v))); }); break;
    case U_EXP: body([](float v) { return expf(v); }); break;
    case U_SQUARE: body([](float v) { return __fmul_rn(v, v); }); break;
    case U_SQRT: body([](float v) { return sqrtf(v); }); break;
    case U_ADD_SCALAR: body([p](float v) { return __fadd_rn(v, p); }); break;
    case U_SCALE: body([p](float v) { return __fmul_rn(v, p); }); break;
    case U_RELU_LO:
      body([](float v) {
        const float r = v > 0.f ? v : 0.f;
        return __fsub_rn(r, __bfloat162float(__float2bfloat16_rn(r)));
      });
      break;
    default: body([](float v) { return v; }); break;
  }
}

template <typename Body>
__device__ __forceinline__ void with_binary(int op, float ca, float cb, Body&& body) {
  switch (op) {
    case B_ADD: body([](float a, float b) { return __fadd_rn(a, b); }); break;
    case B_WEIGHTED: body([ca, cb](float a, float b) { return __fadd_rn(__fmul_rn(ca, a), __fmul_rn(cb, b)); }); break;
    case B_HADAMARD: body([](float a, float b) { return __fmul_rn(a, b); }); break;
    case B_MAX: body([](float a, float b) { return a > b ? a : b; }); break;
    case B_MIN: body([](float a, float b) { return a < b ? a : b; }); break;
    case B_SUB: body([](float a, float b) { return __fsub_rn(a, b); }); break;
    case B_DIV: body([](float a, float b) { return __fdiv_rn(a, b); }); break;
    default: body([](float a, float) { return a; }); break;
  }
}

// ------------------------------------------------------------------ kernels
__global__ void k_unary(int op, const float* __restrict__ in, float* out, long long n, float p) {
  long long i4 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const bool vec = ((((uintptr_t)in) | ((uintptr_t)out)) & 15) == 0;
  if (vec) {
    const long long n4 = n >> 2;
    for (long long i = i4; i < n4; i += stride) {
      float4 v = ((const float4*)in)[i];
      v.x = apply_unary(op, v.x, p); v.y = apply_unary(op, v.y, p);
      v.z = apply_unary(op, v.z, p); v.w = apply_unary(op, v.w, p);
      ((float4*)out)[i] = v;
    }
    for (long long i = (n4 << 2) + i4; i < n; i += stride) out[i] = apply_unary(op, in[i], p);
  } else {
    for (long long i = i4; i < n; i += stride) out[i] = apply_unary(op, in[i], p);
  }
}

__global__ void k_binary(int op, const float* a, const float* b, float* c, long long n, float ca,
                         float cb) {
  long long i4 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const bool vec = ((((uintptr_t)a) | ((uintptr_t)b) | ((uintptr_t)c)) & 15) == 0;
  if (vec) {
    const long long n4 = n >> 2;
    for (long long i = i4; i < n4; i += stride) {
      float4 x = ((const float4*)a)[i];
      float4 y = ((const float4*)b)[i];
      float4 z;
      z.x = apply_binary(op, x.x, y.x, ca, cb); z.y = apply_binary(op, x.y, y.y, ca, cb);
      z.z = apply_binary(op, x.z, y.z, ca, cb); z.w = apply_binary(op, x.w, y.w, ca, cb);
      ((float4*)c)[i] = z;
    }
    for (long long i = (n4 << 2) + i4; i < n; i += stride) c[i] = apply_binary(op, a[i], b[i], ca, cb);
  } else {
    for (long long i = i4; i < n; i += stride) c[i] = apply_binary(op, a[i], b[i], ca, cb);
  }
}

// out = in[0] + in[1] + ... + in[n_in-1], left to right (the order of the
// reference's local reduce, src/operations/local_reduce_op.cc:23-91). With
// kahan != 0 the running sum carries a Kahan compensation term; with kahan == 0
// the result is bit-identical to the reference's pairwise left fold.
// `out` may alias in[0] (the reference marks matrix_add inputs in-place, {0,1}).
template <bool KAHAN>
__global__ void k_reduce(const __grid_constant__ ReduceArgs args, int n_in, float* out,
                         long long n) {
  long long i4 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  bool vec = (((uintptr_t)out) & 15) == 0;
  for (int j = 0; j < n_in; ++j) vec = vec && ((((uintptr_t)args.in[j]) & 15) == 0);
  const long long n4 = vec ? (n >> 2) : 0;
  for (long long i = i4; i < n4; i += stride) {
    float4 s = ((const float4*)args.in[0])[i];
    float4 comp = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int j = 1; j < n_in; ++j) {
      float4 x = ((const float4*)args.in[j])[i];
      if (KAHAN) {
        float y, t;
        y = __fsub_rn(x.x, comp.x); t = __fadd_rn(s.x, y); comp.x = __fsub_rn(__fsub_rn(t, s.x), y); s.x = t;
        y = __fsub_rn(x.y, comp.y); t = __fadd_rn(s.y, y); comp.y = __fsub_rn(__fsub_rn(t, s.y), y); s.y = t;
        y = __fsub_rn(x.z, comp.z); t = __fadd_rn(s.z, y); comp.z = __fsub_rn(__fsub_rn(t, s.z), y); s.z = t;
        y = __fsub_rn(x.w, comp.w); t = __fadd_rn(s.w, y); comp.w = __fsub_rn(__fsub_rn(t, s.w), y); s.w = t;
      } else {
        s.x = __fadd_rn(s.x, x.x); s.y = __fadd_rn(s.y, x.y);
        s.z = __fadd_rn(s.z, x.z); s.w = __fadd_rn(s.w, x.w);
      }
    }
    ((float4*)out)[i] = s;
  }
  for (long long i = (n4 << 2) + i4; i < n; i += stride) {
    float s = args.in[0][i], comp = 0.f;
    for (int j = 1; j < n_in; ++j) {
      float x = args.in[j][i];
      if (KAHAN) {
        float y = __fsub_rn(x, comp);
        float t = __fadd_rn(s, y);
        comp = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
      } else {
        s = __fadd_rn(s, x);
      }
    }
    out[i] = s;
  }
}

// out[r][c] = in[r][c] + bias[c]   (ffnn_activation_mult.cc:88-94)
__global__ void k_bias_add(const float* in, const float* __restrict__ bias, float* out, int rows,
                           int cols, int relu) {
  const long long n = (long long)rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    float v = __fadd_rn(in[i], bias[i % cols]);
    out[i] = (relu && v < 0.f) ? 0.f : v;
  }
}

// out[c] = (accumulate ? out[c] : 0) + sum_r in[r][c], rows summed in order
// (ffnn_back_mult.cc:86-90 sums rows 0..R-1 into the bias). One thread per
// column; consecutive threads read consecutive columns so each row read is
// coalesced; the row loop is unrolled to keep many loads in flight.
__global__ void k_colsum(const float* __restrict__ in, float* out, int rows, int cols, long long ld,
                         int accumulate) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = accumulate ? out[c] : 0.f;
  int r = 0;
  for (; r + 8 <= rows; r += 8) {
    float v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = in[(long long)(r + u) * ld + c];
#pragma unroll
    for (int u = 0; u < 8; ++u) s = __fadd_rn(s, v[u]);
  }
  for (; r < rows; ++r) s = __fadd_rn(s, in[(long long)r * ld + c]);
  out[c] = s;
}

__global__ void k_f32_to_bf16(const float* __restrict__ in, __nv_bfloat16* out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(in[i]);
}

// hi = bf16(relu(z)), lo = bf16(relu(z) - hi): hi + lo carries relu(z) to
// about 16 significant bits, so a tensor-core product of hi and of lo with
// the same bf16 operand sums to nearly the f32-operand product.
__global__ void k_relu_split(const float* __restrict__ z, __nv_bfloat16* hi, __nv_bfloat16* lo, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long i0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if ((((uintptr_t)z) & 15) == 0 && (((uintptr_t)hi | (uintptr_t)lo) & 7) == 0) {
    const long long n4 = n >> 2;
    for (long long i = i0; i < n4; i += stride) {
      const float4 v = ((const float4*)z)[i];
      const float a[4] = {v.x, v.y, v.z, v.w};
      __nv_bfloat16 h[4], l[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float r = a[u] > 0.f ? a[u] : 0.f;
        h[u] = __float2bfloat16_rn(r);
        l[u] = __float2bfloat16_rn(__fsub_rn(r, __bfloat162float(h[u])));
      }
      ((uint2*)hi)[i] = *(const uint2*)h;
      ((uint2*)lo)[i] = *(const uint2*)l;
    }
    for (long long i = (n4 << 2) + i0; i < n; i += stride) {
      const float r = z[i] > 0.f ? z[i] : 0.f;
      hi[i] = __float2bfloat16_rn(r);
      lo[i] = __float2bfloat16_rn(__fsub_rn(r, __bfloat162float(hi[i])));
    }
    return;
  }
  for (long long i = i0; i < n; i += stride) {
    const float r = z[i] > 0.f ? z[i] : 0.f;
    hi[i] = __float2bfloat16_rn(r);
    lo[i] = __float2bfloat16_rn(__fsub_rn(r, __bfloat162float(hi[i])));
  }
}

__global__ void k_bf16_to_f32(const __nv_bfloat16* __restrict__ in, float* out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = __bfloat162float(in[i]);
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC 2011). Counter = (i, 0, 0, 0) for output word group i,
// key = (seed_lo, seed_hi).
__host__ __device__ inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)M0 * c[0];
    uint64_t p1 = (uint64_t)M1 * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
    c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
    k0 += W0; k1 += W1;
  }
}

// Uniform in [lo, hi) from the top 24 bits of each Philox word; normal via
// Box-Muller on word pairs. dist: 0 uniform, 1 normal(mean=lo, std=hi).
template <typename T>
__global__ void k_fill_philox(T* out, long long n, unsigned long long seed, int dist, float lo,
                              float hi) {
  const long long groups = (n + 3) / 4;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < groups;
       g += (long long)gridDim.x * blockDim.x) {
    uint32_t c[4] = {(uint32_t)g, (uint32_t)(g >> 32), 0u, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    float v[4];
    if (dist == 0) {
#pragma unroll
      for (int j = 0; j < 4; ++j) v[j] = __fmaf_rn(hi - lo, (float)(c[j] >> 8) * (1.0f / 16777216.0f), lo);
    } else {
#pragma unroll
      for (int j = 0; j < 4; j += 2) {
        float u1 = ((c[j] >> 8) + 1) * (1.0f / 16777217.0f);
        float u2 = (c[j + 1] >> 8) * (1.0f / 16777216.0f);
        float r = sqrtf(-2.f * logf(u1));
        float sn, cs;
        sincospif(2.f * u2, &sn, &cs);
        v[j] = lo + hi * r * cs;
        v[j + 1] = lo + hi * r * sn;
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      long long i = g * 4 + j;
      if (i < n) {
        if constexpr (sizeof(T) == 4) out[i] = v[j];
        else out[i] = __float2bfloat16_rn(v[j]);
      }
    }
  }
}

// Softmax cross-entropy over rows of `logits` (rows x cols, pitch ld) against
// integer labels. Writes the per-row loss and, if grad != nullptr, the
// gradient (softmax - onehot) * grad_scale in the same layout (f32 or bf16).
// One warp per row.
template <typename TG>
__global__ void k_softmax_ce(const float* __restrict__ logits, const int* __restrict__ labels,
                             float* loss, TG* grad, int rows, int cols, long long ld,
                             float grad_scale) {
  const int warps_per_block = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  for (int r = blockIdx.x * warps_per_block + (threadIdx.x >> 5); r < rows;
       r += gridDim.x * warps_per_block) {
    const float* z = logits + (long long)r * ld;
    float mx = -INFINITY;
    for (int c = lane; c < cols; c += 32) mx = fmaxf(mx, z[c]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    float se = 0.f;
    for (int c = lane; c < cols; c += 32) se += expf(z[c] - mx);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
    const int y = labels[r];
    const float lse = mx + logf(se);
    if (lane == 0) loss[r] = lse - z[y];
    if (grad) {
      TG* g = grad + (long long)r * ld;
      const float inv = 1.f / se;
      for (int c = lane; c < cols; c += 32) {
        float p = expf(z[c] - mx) * inv;
        float v = (p - (c == y ? 1.f : 0.f)) * grad_scale;
        if constexpr (sizeof(TG) == 4) g[c] = v;
        else g[c] = __float2bfloat16_rn(v);
      }
    }
  }
}

// out[e] for e over the output dims: general rank<=4 gather with optional
// f32 -> bf16 cast. `ostride[d]` is the output stride of output dim d and
// `istride[d]` the input stride of the input dim that feeds output dim d;
// `odims` are the output extents (row-major flattening of the output index).
struct PermArgs {
  int rank;
  long long odims[4];
  long long ostride[4];
  long long istride[4];
};

template <typename TO>
__global__ void k_permute(const float* __restrict__ in, TO* out, const __grid_constant__ PermArgs a,
                          long long n) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    long long rem = e, src = 0, dst = 0;
    for (int d = a.rank - 1; d >= 0; --d) {
      long long idx = rem % a.odims[d];
      rem /= a.odims[d];
      src += idx * a.istride[d];
      dst += idx * a.ostride[d];
    }
    if constexpr (sizeof(TO) == 4) out[dst] = in[src];
    else out[dst] = __float2bfloat16_rn(in[src]);
  }
}

}  // namespace bbx

namespace bbx {

// ------------------------------------------------------------------ grouped streaming ops
// One launch processes a table of independent streaming block ops (the add /
// reduce / elementwise / cast commands of one DAG level). Work is split into
// chunks of kStreamChunk elements; chunk c belongs to the op whose
// [chunk_start, chunk_start + chunks) range contains it.
enum StreamKind : int { S_SUM = 0, S_UNARY = 1, S_BINARY = 2, S_CAST = 3 };
constexpr int kStreamMaxIn = 16;
constexpr long long kStreamChunk = 16384;  // elements (measured: 4.3 TB/s on a DAG level vs 4.2 at 8192)

struct StreamOp {
  int kind, op, in_dtype, out_dtype, n_in, kahan;
  long long n;
  const void* in[kStreamMaxIn];
  void* out;
  float p0, p1;
  long long chunk_start;
  int vec;  // 2: all pointers 16-byte aligned; 1: 16-byte (f32) / 8-byte (bf16) aligned; 0: scalar
  int tile; // bulk-staged plans: elements per item (chunk_start then counts items)
};

__device__ __forceinline__ void ld4(const void* p, int dt, long long i, float (&v)[4]) {
  if (dt == 0) {
    float4 x = *(const float4*)((const float*)p + i);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
  } else {
    uint2 x = *(const uint2*)((const __nv_bfloat16*)p + i);
    __nv_bfloat162 a = *(__nv_bfloat162*)&x.x, b = *(__nv_bfloat162*)&x.y;
    float2 fa = __bfloat1622float2(a), fb = __bfloat1622float2(b);
    v[0] = fa.x; v[1] = fa.y; v[2] = fb.x; v[3] = fb.y;
  }
}
__device__ __forceinline__ float ld1(const void* p, int dt, long long i) {
  return dt == 0 ? ((const float*)p)[i] : __bfloat162float(((const __nv_bfloat16*)p)[i]);
}
__device__ __forceinline__ void st4(void* p, int dt, long long i, const float (&v)[4]) {
  if (dt == 0) {
    *(float4*)((float*)p + i) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
    __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]);
    uint2 x;
    x.x = *(uint32_t*)&a;
    x.y = *(uint32_t*)&b;
    *(uint2*)((__nv_bfloat16*)p + i) = x;
  }
}
__device__ __forceinline__ void st1(void* p, int dt, long long i, float v) {
  if (dt == 0) ((float*)p)[i] = v;
  else ((__nv_bfloat16*)p)[i] = __float2bfloat16_rn(v);
}

// Unary / binary / cast element (sums are evaluated inline by the caller).
__device__ __forceinline__ float stream_eval(const StreamOp& o, const float* x) {
  switch (o.kind) {
    case S_UNARY: return apply_unary(o.op, x[0], o.p0);
    case S_BINARY: return apply_binary(o.op, x[0], x[1], o.p0, o.p1);
    default: return x[0];
  }
}

constexpr int kStreamInline = 8;
struct StreamInline {
  StreamOp ops[kStreamInline];
};

// ---- wide path: every pointer of the op 16-byte aligned, one 16-byte access
// per input per step (8 bf16 or 4 f32 elements)
template <int DT, int VW>
__device__ __forceinline__ void ldv(const void* p, long long i, float (&v)[VW]) {
  if constexpr (DT == 0) {
    const float4 x = *(const float4*)((const float*)p + i);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
  } else {
    const uint4 x = *(const uint4*)((const __nv_bfloat16*)p + i);
    const uint32_t w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float2 f = __bfloat1622float2(*(const __nv_bfloat162*)&w[q]);
      v[2 * q] = f.x;
      v[2 * q + 1] = f.y;
    }
  }
}

template <int DT, int VW>
__device__ __forceinline__ void stv(void* p, long long i, const float (&v)[VW]) {
  if constexpr (DT == 0) {
#pragma unroll
    for (int q = 0; q < VW; q += 4) *(float4*)((float*)p + i + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
  } else {
    uint32_t w[VW / 2];
#pragma unroll
    for (int q = 0; q < VW / 2; ++q) {
      const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
      w[q] = *(const uint32_t*)&h;
    }
    if constexpr (VW == 8) *(uint4*)((__nv_bfloat16*)p + i) = make_uint4(w[0], w[1], w[2], w[3]);
    else *(uint2*)((__nv_bfloat16*)p + i) = make_uint2(w[0], w[1]);
  }
}

// a += b in order (Kahan-compensated when asked), elementwise over VW lanes
template <int VW>
__device__ __forceinline__ void fold_in(float (&a)[VW], float (&comp)[VW], const float (&b)[VW], bool kahan) {
#pragma unroll
  for (int u = 0; u < VW; ++u) {
    if (kahan) {
      const float y = __fsub_rn(b[u], comp[u]);
      const float t = __fadd_rn(a[u], y);
      comp[u] = __fsub_rn(__fsub_rn(t, a[u]), y);
      a[u] = t;
    } else {
      a[u] = __fadd_rn(a[u], b[u]);
    }
  }
}

// Elements [e0, e1) of one op. Sums fold the inputs left to right exactly as
// the narrow path does; loads of up to four inputs are issued before they are
// folded, so each thread keeps several 16-byte loads in flight.
template <int IDT, int ODT, typename OpT>
__device__ __forceinline__ void stream_wide(const OpT& o, long long e0, long long e1) {
  constexpr int VW = IDT == 1 ? 8 : 4;
  const int kind = o.kind, nin = o.n_in, op = o.op;
  const bool kahan = o.kahan != 0;
  const float p0 = o.p0, p1 = o.p1;
  const void* const* in = o.in;  // read per use: a local copy indexed at run time would live in local memory
  void* const out = o.out;
  for (long long i = e0 + (long long)VW * threadIdx.x; i < e1; i += (long long)VW * blockDim.x) {
    if (i + VW <= e1) {
      float a[VW], r[VW];
      ldv<IDT, VW>(in[0], i, a);
      if (kind == S_SUM) {
        float comp[VW];
#pragma unroll
        for (int u = 0; u < VW; ++u) comp[u] = 0.f;
        int j = 1;
        for (; j + 3 < nin; j += 4) {
          float b0[VW], b1[VW], b2[VW], b3[VW];
          ldv<IDT, VW>(in[j], i, b0);
          ldv<IDT, VW>(in[j + 1], i, b1);
          ldv<IDT, VW>(in[j + 2], i, b2);
          ldv<IDT, VW>(in[j + 3], i, b3);
          fold_in(a, comp, b0, kahan);
          fold_in(a, comp, b1, kahan);
          fold_in(a, comp, b2, kahan);
          fold_in(a, comp, b3, kahan);
        }
        for (; j < nin; ++j) {
          float b0[VW];
          ldv<IDT, VW>(in[j], i, b0);
          fold_in(a, comp, b0, kahan);
        }
#pragma unroll
        for (int u = 0; u < VW; ++u) r[u] = a[u];
      } else if (kind == S_BINARY) {
        float b[VW];
        ldv<IDT, VW>(in[1], i, b);
#pragma unroll
        for (int u = 0; u < VW; ++u) r[u] = apply_binary(op, a[u], b[u], p0, p1);
      } else if (kind == S_UNARY) {
#pragma unroll
        for (int u = 0; u < VW; ++u) r[u] = apply_unary(op, a[u], p0);
      } else {
#pragma unroll
        for (int u = 0; u < VW; ++u) r[u] = a[u];
      }
      stv<ODT, VW>(out, i, r);
    } else {
      for (long long q = i; q < e1; ++q) {
        float x = ld1(in[0], IDT, q);
        if (kind == S_SUM) {
          float comp = 0.f;
          for (int j = 1; j < nin; ++j) {
            const float v = ld1(in[j], IDT, q);
            if (kahan) {
              const float y = __fsub_rn(v, comp), t = __fadd_rn(x, y);
              comp = __fsub_rn(__fsub_rn(t, x), y);
              x = t;
            } else {
              x = __fadd_rn(x, v);
            }
          }
        } else if (kind == S_BINARY) {
          x = apply_binary(op, x, ld1(in[1], IDT, q), p0, p1);
        } else if (kind == S_UNARY) {
          x = apply_unary(op, x, p0);
        }
        st1(out, ODT, q, x);
      }
    }
  }
}

template <typename TableT>
__device__ __forceinline__ void stream_group_body(const TableT* __restrict__ table, int count,
                                                  long long total_chunks);

// Table in global memory (plans, replayed inside CUDA graphs).
__global__ void __launch_bounds__(256) k_stream_group(const StreamOp* __restrict__ table, int count,
                                                      long long total_chunks) {
  stream_group_body(table, count, total_chunks);
}

// Up to kStreamInline ops carried in the kernel parameters (one-shot calls).
__global__ void __launch_bounds__(256) k_stream_group_inline(const __grid_constant__ StreamInline args,
                                                             int count, long long total_chunks) {
  stream_group_body(args.ops, count, total_chunks);
}

template <typename TableT>
__device__ __forceinline__ void stream_group_body(const TableT* __restrict__ table, int count,
                                                  long long total_chunks) {
  for (long long c = blockIdx.x; c < total_chunks; c += gridDim.x) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (table[mid].chunk_start <= c) lo = mid; else hi = mid - 1;
    }
    const StreamOp& o = table[lo];
    const long long e0 = (c - o.chunk_start) * kStreamChunk;
    const long long e1 = min(e0 + kStreamChunk, o.n);
    const int kind = o.kind, idt = o.in_dtype, odt = o.out_dtype, nin = o.n_in;
    if (o.vec == 2) {
      switch (idt * 2 + odt) {
        case 0: stream_wide<0, 0>(o, e0, e1); break;
        case 1: stream_wide<0, 1>(o, e0, e1); break;
        case 2: stream_wide<1, 0>(o, e0, e1); break;
        default: stream_wide<1, 1>(o, e0, e1); break;
      }
      continue;
    }
    if (o.vec) {
      for (long long i = e0 + 4 * threadIdx.x; i < e1; i += 4 * blockDim.x) {
        if (i + 4 <= e1) {
          float a[4], b[4], r[4];
          ld4(o.in[0], idt, i, a);
          if (kind == S_SUM) {
            float comp[4] = {0.f, 0.f, 0.f, 0.f};
            for (int j = 1; j < nin; ++j) {
              ld4(o.in[j], idt, i, b);
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                if (o.kahan) {
                  float y = __fsub_rn(b[u], comp[u]);
                  float t = __fadd_rn(a[u], y);
                  comp[u] = __fsub_rn(__fsub_rn(t, a[u]), y);
                  a[u] = t;
                } else {
                  a[u] = __fadd_rn(a[u], b[u]);
                }
              }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) r[u] = a[u];
          } else if (kind == S_BINARY) {
            ld4(o.in[1], idt, i, b);
#pragma unroll
            for (int u = 0; u < 4; ++u) r[u] = apply_binary(o.op, a[u], b[u], o.p0, o.p1);
          } else if (kind == S_UNARY) {
#pragma unroll
            for (int u = 0; u < 4; ++u) r[u] = apply_unary(o.op, a[u], o.p0);
          } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) r[u] = a[u];
          }
          st4(o.out, odt, i, r);
        } else {
          for (long long q = i; q < e1; ++q) {
            float x[2] = {ld1(o.in[0], idt, q), 0.f};
            if (kind == S_SUM) {
              float comp = 0.f;
              for (int j = 1; j < nin; ++j) {
                float v = ld1(o.in[j], idt, q);
                if (o.kahan) {
                  float y = __fsub_rn(v, comp), t = __fadd_rn(x[0], y);
                  comp = __fsub_rn(__fsub_rn(t, x[0]), y);
                  x[0] = t;
                } else {
                  x[0] = __fadd_rn(x[0], v);
                }
              }
              st1(o.out, odt, q, x[0]);
            } else {
              if (kind == S_BINARY) x[1] = ld1(o.in[1], idt, q);
              st1(o.out, odt, q, stream_eval(o, x));
            }
          }
        }
      }
    } else {
      for (long long q = e0 + threadIdx.x; q < e1; q += blockDim.x) {
        float x[2] = {ld1(o.in[0], idt, q), 0.f};
        if (kind == S_SUM) {
          float comp = 0.f;
          for (int j = 1; j < nin; ++j) {
            float v = ld1(o.in[j], idt, q);
            if (o.kahan) {
              float y = __fsub_rn(v, comp), t = __fadd_rn(x[0], y);
              comp = __fsub_rn(__fsub_rn(t, x[0]), y);
              x[0] = t;
            } else {
              x[0] = __fadd_rn(x[0], v);
            }
          }
          st1(o.out, odt, q, x[0]);
        } else {
          if (kind == S_BINARY) x[1] = ld1(o.in[1], idt, q);
          st1(o.out, odt, q, stream_eval(o, x));
        }
      }
    }
  }
}

}  // namespace bbx

namespace bbx {

// ---- bulk-staged path: used when every pointer of every op is 16-byte
// aligned. Work is dealt as items, one op's `tile` consecutive elements, with
// `tile` sized per op so that every item moves about kBulkSlot bytes (inputs +
// output) whatever its fan-in. One CTA per SM:
//  - a producer warp copies each item's input tiles into a shared-memory
//    stage with cp.async.bulk, one lane per input (kBulkStages stages,
//    completion on the stage's `full` mbarrier);
//  - kBulkConsumerWarps warps fold them in the same order as the register
//    paths above (bit-identical results), with the element function chosen
//    once per item (with_unary / with_binary), and store the output with
//    16-byte stores, handing the stage back (`empty` mbarrier) right away.
// Measured on the FFN and 2000-op DAG levels: 8 consumer warps beat 16, whole
// input tiles per copy beat 2-8 KiB pieces, and consumer stores beat staging
// the output tile for a bulk store (kBulkStoreTS, kept as an option). Fewer,
// larger stages win: 3 x 72 KiB against 3 x 64 KiB ran the 2000-op DAG's
// levels of adds at 6.89 against 6.47 TB/s (4 x 48 and 6 x 32 KiB were slower). The
// last (< 8-element) piece of an op, if any, is read and written with plain
// accesses.
constexpr int kBulkStages = 3;
constexpr int kBulkSlot = 73728;     // bytes per stage: input tiles + output tile
constexpr int kBulkConsumerWarps = 8;
constexpr int kBulkConsumers = kBulkConsumerWarps * 32;
constexpr int kBulkThreads = kBulkConsumers + 32;
// Shared memory after the stages: the full / empty barriers, each stage's op
// descriptor (a copy of its StreamOp, which the consumers read instead of the
// table in global memory) and, for plans of at most kBulkMaxStagedOps ops,
// every op's chunk_start, where the producer finds the op of an item. The
// binary search through the global table this replaces was a chain of
// dependent L2 reads per item, with the table evicted from L1 by the stages:
// measured on 2000-op random DAGs' streaming levels, adds 5.33 -> 6.49 TB/s,
// 2-16-input reduces 4.90 -> 5.73 TB/s.
constexpr int kBulkDescBytes = (int)sizeof(StreamOp);
static_assert(kBulkDescBytes % 16 == 0, "stage descriptors are copied in 16-byte pieces");
constexpr int kBulkSmem = kBulkStages * kBulkSlot + kBulkStages * 16 + kBulkStages * kBulkDescBytes;
constexpr int kBulkMaxStagedOps = 1280;
constexpr int kBulkSmemMax = kBulkSmem + 8 * kBulkMaxStagedOps;
static_assert(kBulkSmemMax <= 232448, "dynamic shared memory per CTA");
__host__ __device__ inline int bulk_smem_bytes(int count) {
  return kBulkSmem + (count <= kBulkMaxStagedOps ? 8 * count : 0);
}
constexpr bool kBulkStoreTS = false;   // output tiles by consumer stores (see stream_bulk_body)
constexpr uint32_t kBulkPiece = 65536;  // bytes per bulk load (one copy per input tile: splitting measured slower)

// Elements per item: a multiple of 64 whose input and output tiles fill at
// most one stage.
__host__ __device__ inline int bulk_tile(int n_in, int in_esz, int out_esz) {
  const int te = kBulkSlot / (n_in * in_esz + out_esz) / 64 * 64;
  return te < 64 ? 64 : te;
}

template <typename TableT>
__device__ __forceinline__ int stream_find_op(const TableT* table, int count, long long item) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (table[mid].chunk_start <= item) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Staged elements [e0, e0 + cnt) of one op: input j's tile at
// slot + j * tile elements. TS: the output tile goes to the stage (after the
// n_in input tiles) for a bulk store; else it is stored to global memory
// directly. Elements [e0 + cnt, e1) are read and written in global memory.
template <int IDT, int ODT, bool TS, typename OpT>
__device__ __forceinline__ void bulk_item(const OpT& o, uint8_t* slot, long long e0, int cnt, long long e1,
                                          int ctid) {
  constexpr int VW = IDT == 1 ? 8 : 4;
  constexpr int ESZ = IDT == 1 ? 2 : 4;
  const int kind = o.kind, nin = o.n_in, op = o.op, te = o.tile;
  const bool kahan = o.kahan != 0;
  const float p0 = o.p0, p1 = o.p1;
  void* const out = o.out;
  uint8_t* const oslot = slot + (size_t)nin * te * ESZ;
  auto put = [&](int li, const float (&r)[VW]) {
    if constexpr (TS) stv<ODT, VW>(oslot, li, r);
    else stv<ODT, VW>(out, e0 + li, r);
  };
  if (kind == S_SUM) {
    for (int li = ctid * VW; li < cnt; li += kBulkConsumers * VW) {
      float a[VW], comp[VW];
      ldv<IDT, VW>(slot, li, a);
#pragma unroll
      for (int u = 0; u < VW; ++u) comp[u] = 0.f;
      for (int j = 1; j < nin; ++j) {
        float b[VW];
        ldv<IDT, VW>(slot + (size_t)j * te * ESZ, li, b);
        fold_in(a, comp, b, kahan);
      }
      put(li, a);
    }
  } else if (kind == S_BINARY) {
    const uint8_t* const slot_b = slot + (size_t)te * ESZ;
    with_binary(op, p0, p1, [&](auto f) {
      for (int li = ctid * VW; li < cnt; li += kBulkConsumers * VW) {
        float a[VW], b[VW], r[VW];
        ldv<IDT, VW>(slot, li, a);
        ldv<IDT, VW>(slot_b, li, b);
#pragma unroll
        for (int u = 0; u < VW; ++u) r[u] = f(a[u], b[u]);
        put(li, r);
      }
    });
  } else {
    // unary, or a cast (the identity)
    with_unary(kind == S_UNARY ? op : -1, p0, [&](auto f) {
      for (int li = ctid * VW; li < cnt; li += kBulkConsumers * VW) {
        float a[VW], r[VW];
        ldv<IDT, VW>(slot, li, a);
#pragma unroll
        for (int u = 0; u < VW; ++u) r[u] = f(a[u]);
        put(li, r);
      }
    });
  }
  for (long long q = e0 + cnt + ctid; q < e1; q += kBulkConsumers) {
    float x = ld1(o.in[0], IDT, q);
    if (kind == S_SUM) {
      float comp = 0.f;
      for (int j = 1; j < nin; ++j) {
        const float v = ld1(o.in[j], IDT, q);
        if (kahan) {
          const float y = __fsub_rn(v, comp), t = __fadd_rn(x, y);
          comp = __fsub_rn(__fsub_rn(t, x), y);
          x = t;
        } else {
          x = __fadd_rn(x, v);
        }
      }
    } else if (kind == S_BINARY) {
      x = apply_binary(op, x, ld1(o.in[1], IDT, q), p0, p1);
    } else if (kind == S_UNARY) {
      x = apply_unary(op, x, p0);
    }
    st1(out, ODT, q, x);
  }
}

// Bounded wait that ignores the status word: used only to let copies already
// issued land before the CTA exits after an error.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kWaitBudgetCycles) return;
}

// Global bulk store from this CTA's shared memory (bulk-group completion);
// both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_store(void* gdst, const void* smem_src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_u32(smem_src)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kBulkConsumers) : "memory"); }
// Barrier over the consumer threads that also ANDs their flags: every consumer
// takes the same branch after a bounded wait, so none is left at a barrier.
__device__ __forceinline__ bool consumers_all(bool p) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)p), "n"(kBulkConsumers)
      : "memory");
  return r != 0;
}

// TS: output tiles leave by bulk store (the stage is handed back once the
// store has read it); else consumers store them and hand the stage back
// right away. Input tiles are copied in pieces of at most `piece` bytes so
// several bulk copies are in flight even for a one-input op.
template <bool TS, typename TableT>
__device__ __forceinline__ void stream_bulk_body(const TableT* table, int count, long long total_items,
                                                 uint32_t* status, uint32_t piece) {
  extern __shared__ __align__(128) uint8_t bulk_smem[];
  uint64_t* full = (uint64_t*)(bulk_smem + kBulkStages * kBulkSlot);
  uint64_t* empty = full + kBulkStages;
  StreamOp* desc = (StreamOp*)(empty + kBulkStages);       // [kBulkStages]: the op of the stage's item
  long long* starts = (long long*)(desc + kBulkStages);    // [count] when staged: every op's chunk_start
  const bool staged = count <= kBulkMaxStagedOps;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kBulkStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], TS ? 1 : kBulkConsumerWarps);
    }
    fence_mbar_init();
  }
  if (staged)
    for (int i = threadIdx.x; i < count; i += blockDim.x) starts[i] = table[i].chunk_start;
  __syncthreads();
  volatile uint32_t* st = status;
  if (warp == kBulkConsumerWarps) {
    // producer warp: lane 0 owns the barriers and the stage descriptors, lane j
    // issues input j's copies. A CTA's items come in increasing order, so the
    // op index only moves forward; lane 0 keeps the current op in registers and
    // reads the table only when the op changes.
    constexpr int kDescPieces = kBulkDescBytes / 16;
    uint4 cur[kDescPieces];
    int oi = -1;
    int k = 0;
    for (long long it = blockIdx.x; it < total_items; it += gridDim.x, ++k) {
      const int s = k % kBulkStages;
      const uint32_t ph = (uint32_t)(k / kBulkStages) & 1u;
      bool ok = true;
      if (lane == 0) ok = mbar_wait(&empty[s], ph ^ 1u, st, DEV_TIMEOUT_EMPTY);
      if (!__shfl_sync(0xffffffffu, ok, 0)) break;
      int noi;
      if (!staged) {
        noi = stream_find_op(table, count, it);
      } else if (oi < 0) {
        int lo = 0, hi = count - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (starts[mid] <= it) lo = mid; else hi = mid - 1;
        }
        noi = lo;
      } else {
        noi = oi;
        while (noi + 1 < count && starts[noi + 1] <= it) ++noi;
      }
      if (lane == 0) {
        if (noi != oi) {
          const uint4* src = (const uint4*)&table[noi];
#pragma unroll
          for (int q = 0; q < kDescPieces; ++q) cur[q] = src[q];
        }
        uint4* dst = (uint4*)&desc[s];
#pragma unroll
        for (int q = 0; q < kDescPieces; ++q) dst[q] = cur[q];
      }
      oi = noi;
      __syncwarp();
      const StreamOp& o = desc[s];
      const int esz = o.in_dtype == 1 ? 2 : 4;
      const long long e0 = (it - o.chunk_start) * (long long)o.tile;
      const long long e1 = min(e0 + (long long)o.tile, o.n);
      const uint32_t nb = (uint32_t)((e1 - e0) & ~7LL) * esz;  // a multiple of 8 elements: 16-byte multiples
      uint8_t* slot = bulk_smem + s * kBulkSlot;
      if (lane == 0) {
        // the descriptor is published by this arrive (release)
        if (nb) mbar_arrive_expect_tx(&full[s], nb * (uint32_t)o.n_in);
        else mbar_arrive(&full[s]);
      }
      __syncwarp();  // the expected bytes are registered before any copy is issued
      if (nb) {
        for (int j = lane; j < o.n_in; j += 32) {
          uint8_t* dst = slot + (size_t)j * o.tile * esz;
          const uint8_t* src = (const uint8_t*)o.in[j] + e0 * esz;
          for (uint32_t off = 0; off < nb; off += piece)
            bulk_load(dst + off, src + off, min(piece, nb - off), &full[s]);
        }
      }
    }
    // copies issued but never consumed (only after an error) land before exit
    if (lane == 0 && *st != DEV_OK)
      for (int q = (k > kBulkStages ? k - kBulkStages : 0); q < k; ++q)
        mbar_drain(&full[q % kBulkStages], (uint32_t)(q / kBulkStages) & 1u);
    return;
  }
  const int ctid = threadIdx.x;
  int k = 0;
  for (long long it = blockIdx.x; it < total_items; it += gridDim.x, ++k) {
    const int s = k % kBulkStages;
    const uint32_t ph = (uint32_t)(k / kBulkStages) & 1u;
    if (!consumers_all(mbar_wait(&full[s], ph, st, DEV_TIMEOUT_FULL))) break;
    const StreamOp& o = desc[s];
    const int esz = o.in_dtype == 1 ? 2 : 4, osz = o.out_dtype == 1 ? 2 : 4;
    const long long e0 = (it - o.chunk_start) * (long long)o.tile;
    const long long e1 = min(e0 + (long long)o.tile, o.n);
    const int cnt = (int)((e1 - e0) & ~7LL);
    uint8_t* slot = bulk_smem + s * kBulkSlot;
    switch (o.in_dtype * 2 + o.out_dtype) {
      case 0: bulk_item<0, 0, TS>(o, slot, e0, cnt, e1, ctid); break;
      case 1: bulk_item<0, 1, TS>(o, slot, e0, cnt, e1, ctid); break;
      case 2: bulk_item<1, 0, TS>(o, slot, e0, cnt, e1, ctid); break;
      default: bulk_item<1, 1, TS>(o, slot, e0, cnt, e1, ctid); break;
    }
    if constexpr (TS) {
      fence_proxy_async_smem();  // this thread's output-tile writes, visible to the bulk store
      consumer_sync();
      if (ctid == 0) {
        if (cnt) bulk_store((uint8_t*)o.out + e0 * osz, slot + (size_t)o.n_in * o.tile * esz, (uint32_t)cnt * osz);
        bulk_commit();
        // the previous item's store has finished reading its stage: hand it back
        bulk_wait_read_1();
        if (k > 0) mbar_arrive(&empty[(k - 1) % kBulkStages]);
      }
    } else {
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
  }
  if (TS && ctid == 0) {
    bulk_wait_read_all();
    bulk_wait_all();  // output tiles written before the CTA ends
  }
}

template <bool TS>
__global__ void __launch_bounds__(kBulkThreads, 1) k_stream_bulk(const StreamOp* __restrict__ table, int count,
                                                                  long long total_items, uint32_t* status,
                                                                  uint32_t piece) {
  stream_bulk_body<TS>(table, count, total_items, status, piece);
}

template <bool TS>
__global__ void __launch_bounds__(kBulkThreads, 1) k_stream_bulk_inline(const __grid_constant__ StreamInline args,
                                                                         int count, long long total_items,
                                                                         uint32_t* status, uint32_t piece) {
  stream_bulk_body<TS>(args.ops, count, total_items, status, piece);
}

}  // namespace bbx
