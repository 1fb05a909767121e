// FP32 SIMT block matmul: the "plain FP32" path. It computes exactly what the
// reference's CPU block matmul computes (src/ud_functions/impls/dense_matrix_mult.cc:78-82,
// row-major C = op(A) op(B) with transpose flags) in IEEE fp32 with fused
// multiply-adds, and also serves the batched-strided GEMM of the contraction
// (libraries/cutensor/contraction.h:439-461) and the cost-model MLP.
//
// Tile 128x128x8, 256 threads, 8x8 outputs per thread laid out as two 4x4
// quadrants 64 apart so shared-memory reads are float4 and conflict-free;
// double-buffered shared memory with register prefetch of the next k-slice.
#pragma once
#include <cstdint>

namespace bbx {

struct F32GemmArgs {
  const float* a;
  const float* b;
  float* c;
  const float* bias;       // optional, length n
  int m, n, k;
  long long lda, ldb, ldc;
  long long stride_a, stride_b, stride_c;  // batch strides (elements)
  int trans_a, trans_b;
  float alpha, beta;
  int relu;
};

constexpr int F32_BM = 128, F32_BN = 128, F32_BK = 8;

__global__ void __launch_bounds__(256) k_gemm_f32(const __grid_constant__ F32GemmArgs g) {
  __shared__ __align__(16) float As[2][F32_BK][F32_BM];
  __shared__ __align__(16) float Bs[2][F32_BK][F32_BN];

  const int bz = blockIdx.z;
  const float* A = g.a + bz * g.stride_a;
  const float* B = g.b + bz * g.stride_b;
  float* Cp = g.c + bz * g.stride_c;
  const int m0 = blockIdx.y * F32_BM;
  const int n0 = blockIdx.x * F32_BN;
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;

  // Each thread loads 4 elements of the A tile and 4 of the B tile per k-slice.
  // Non-transposed A (m,k at m*lda+k): thread -> row tid/2, k-quad (tid&1)*4.
  // Transposed A (m,k at k*lda+m):     thread -> k tid/32, m-quad (tid&31)*4.
  float ra[4], rb[4];
  auto load_a = [&](int k0) {
    if (!g.trans_a) {
      int r = tid >> 1, kq = (tid & 1) * 4;
      int gm = m0 + r;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        int gk = k0 + kq + u;
        ra[u] = (gm < g.m && gk < g.k) ? A[(long long)gm * g.lda + gk] : 0.f;
      }
    } else {
      int kk = tid >> 5, mq = (tid & 31) * 4;
      int gk = k0 + kk;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        int gm = m0 + mq + u;
        ra[u] = (gm < g.m && gk < g.k) ? A[(long long)gk * g.lda + gm] : 0.f;
      }
    }
  };
  auto store_a = [&](int buf) {
    if (!g.trans_a) {
      int r = tid >> 1, kq = (tid & 1) * 4;
#pragma unroll
      for (int u = 0; u < 4; ++u) As[buf][kq + u][r] = ra[u];
    } else {
      int kk = tid >> 5, mq = (tid & 31) * 4;
      *(float4*)&As[buf][kk][mq] = make_float4(ra[0], ra[1], ra[2], ra[3]);
    }
  };
  // Non-transposed B (k,n at k*ldb+n): thread -> k tid/32, n-quad (tid&31)*4.
  // Transposed B (k,n at n*ldb+k):     thread -> n tid/2, k-quad (tid&1)*4.
  auto load_b = [&](int k0) {
    if (!g.trans_b) {
      int kk = tid >> 5, nq = (tid & 31) * 4;
      int gk = k0 + kk;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        int gn = n0 + nq + u;
        rb[u] = (gn < g.n && gk < g.k) ? B[(long long)gk * g.ldb + gn] : 0.f;
      }
    } else {
      int r = tid >> 1, kq = (tid & 1) * 4;
      int gn = n0 + r;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        int gk = k0 + kq + u;
        rb[u] = (gn < g.n && gk < g.k) ? B[(long long)gn * g.ldb + gk] : 0.f;
      }
    }
  };
  auto store_b = [&](int buf) {
    if (!g.trans_b) {
      int kk = tid >> 5, nq = (tid & 31) * 4;
      *(float4*)&Bs[buf][kk][nq] = make_float4(rb[0], rb[1], rb[2], rb[3]);
    } else {
      int r = tid >> 1, kq = (tid & 1) * 4;
#pragma unroll
      for (int u = 0; u < 4; ++u) Bs[buf][kq + u][r] = rb[u];
    }
  };

  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

  const int ktiles = (g.k + F32_BK - 1) / F32_BK;
  load_a(0);
  load_b(0);
  store_a(0);
  store_b(0);
  __syncthreads();
  for (int kt = 0; kt < ktiles; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < ktiles) {
      load_a((kt + 1) * F32_BK);
      load_b((kt + 1) * F32_BK);
    }
#pragma unroll
    for (int kk = 0; kk < F32_BK; ++kk) {
      float4 a0 = *(const float4*)&As[buf][kk][ty * 4];
      float4 a1 = *(const float4*)&As[buf][kk][ty * 4 + 64];
      float4 b0 = *(const float4*)&Bs[buf][kk][tx * 4];
      float4 b1 = *(const float4*)&Bs[buf][kk][tx * 4 + 64];
      float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
    if (kt + 1 < ktiles) {
      store_a(buf ^ 1);
      store_b(buf ^ 1);
    }
    __syncthreads();
  }

#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int gm = m0 + ty * 4 + (i & 3) + (i >> 2) * 64;
    if (gm >= g.m) continue;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int gn = n0 + tx * 4 + (j & 3) + (j >> 2) * 64;
      if (gn >= g.n) continue;
      float v = g.alpha * acc[i][j];
      float* cp = Cp + (long long)gm * g.ldc + gn;
      if (g.beta != 0.f) v += g.beta * *cp;
      if (g.bias) v += g.bias[gn];
      if (g.relu) v = v > 0.f ? v : 0.f;
      *cp = v;
    }
  }
}

// ---------------------------------------------------------------------------
// Vector-load variant for aligned operands (the blocks of the plain FP32 path):
// 128x128 tile, BK = 16, 256 threads, the same 8x8 outputs per thread.
// Every global load is one 16-byte load along the operand's contiguous
// dimension; the K-contiguous operands (A row-major, B transposed) are stored
// transposed into shared memory, the MN-contiguous ones directly. Rows of the
// shared tiles are padded by 4 floats so the transposed stores spread over the
// banks and float4 reads stay 16-byte aligned. Two CTAs fit on an SM
// (33 KB shared memory, <= 128 registers). The epilogue stores float4 rows of
// C when C's rows allow it.
// Requirements (checked by the host): a, b 16-byte aligned; lda, ldb and the
// batch strides multiples of 4; the contiguous extent of each operand (k for
// row-major A / transposed B, m for transposed A, n for row-major B) a
// multiple of 4, so a 16-byte piece is either wholly inside the matrix or
// wholly outside.
constexpr int F32V_BK = 16, F32V_LD = F32_BM + 4;

__device__ __forceinline__ float4 ldg4_or_zero(const float* p, bool ok) {
  return ok ? __ldg((const float4*)p) : make_float4(0.f, 0.f, 0.f, 0.f);
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(256, 1) k_gemm_f32_v(const __grid_constant__ F32GemmArgs g) {
  __shared__ __align__(16) float As[2][F32V_BK][F32V_LD];
  __shared__ __align__(16) float Bs[2][F32V_BK][F32V_LD];

  const int bz = blockIdx.z;
  const float* A = g.a + bz * g.stride_a;
  const float* B = g.b + bz * g.stride_b;
  float* Cp = g.c + bz * g.stride_c;
  const int m0 = blockIdx.y * F32_BM;
  const int n0 = blockIdx.x * F32_BN;
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;

  // 128 x 16 (A) and 16 x 128 (B) tiles = 512 float4 each: two per thread.
  // K-contiguous: piece f -> row f / 4, k-quad (f % 4) * 4.
  // MN-contiguous: piece f -> k f / 32, quad (f % 32) * 4.
  float4 ra[2], rb[2];
  auto load = [&](int k0) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int f = tid + 256 * i;
      if (!TA) {
        const int gm = m0 + (f >> 2), gk = k0 + (f & 3) * 4;
        ra[i] = ldg4_or_zero(A + (long long)gm * g.lda + gk, gm < g.m && gk < g.k);
      } else {
        const int gk = k0 + (f >> 5), gm = m0 + (f & 31) * 4;
        ra[i] = ldg4_or_zero(A + (long long)gk * g.lda + gm, gk < g.k && gm < g.m);
      }
      if (!TB) {
        const int gk = k0 + (f >> 5), gn = n0 + (f & 31) * 4;
        rb[i] = ldg4_or_zero(B + (long long)gk * g.ldb + gn, gk < g.k && gn < g.n);
      } else {
        const int gn = n0 + (f >> 2), gk = k0 + (f & 3) * 4;
        rb[i] = ldg4_or_zero(B + (long long)gn * g.ldb + gk, gn < g.n && gk < g.k);
      }
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int f = tid + 256 * i;
      if (!TA) {
        const int r = f >> 2, kq = (f & 3) * 4;
        As[buf][kq][r] = ra[i].x; As[buf][kq + 1][r] = ra[i].y;
        As[buf][kq + 2][r] = ra[i].z; As[buf][kq + 3][r] = ra[i].w;
      } else {
        *(float4*)&As[buf][f >> 5][(f & 31) * 4] = ra[i];
      }
      if (!TB) {
        *(float4*)&Bs[buf][f >> 5][(f & 31) * 4] = rb[i];
      } else {
        const int r = f >> 2, kq = (f & 3) * 4;
        Bs[buf][kq][r] = rb[i].x; Bs[buf][kq + 1][r] = rb[i].y;
        Bs[buf][kq + 2][r] = rb[i].z; Bs[buf][kq + 3][r] = rb[i].w;
      }
    }
  };

  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

  const int ktiles = (g.k + F32V_BK - 1) / F32V_BK;
  load(0);
  store(0);
  __syncthreads();
  for (int kt = 0; kt < ktiles; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < ktiles) load((kt + 1) * F32V_BK);
#pragma unroll
    for (int kk = 0; kk < F32V_BK; ++kk) {
      const float4 a0 = *(const float4*)&As[buf][kk][ty * 4];
      const float4 a1 = *(const float4*)&As[buf][kk][ty * 4 + 64];
      const float4 b0 = *(const float4*)&Bs[buf][kk][tx * 4];
      const float4 b1 = *(const float4*)&Bs[buf][kk][tx * 4 + 64];
      const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
    if (kt + 1 < ktiles) store(buf ^ 1);
    __syncthreads();
  }

  const bool vec_c = ((((uintptr_t)Cp) & 15) == 0) && (g.ldc & 3) == 0 && (g.n & 3) == 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int gm = m0 + ty * 4 + (i & 3) + (i >> 2) * 64;
    if (gm >= g.m) continue;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int gn = n0 + tx * 4 + h * 64;
      if (gn >= g.n) continue;
      float v[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) v[q] = g.alpha * acc[i][4 * h + q];
      float* cp = Cp + (long long)gm * g.ldc + gn;
      if (vec_c) {  // n % 4 == 0: the four columns are all inside
        if (g.beta != 0.f) {
          const float4 o = *(const float4*)cp;
          v[0] += g.beta * o.x; v[1] += g.beta * o.y; v[2] += g.beta * o.z; v[3] += g.beta * o.w;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (g.bias) v[q] += g.bias[gn + q];
          if (g.relu) v[q] = v[q] > 0.f ? v[q] : 0.f;
        }
        *(float4*)cp = make_float4(v[0], v[1], v[2], v[3]);
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (gn + q >= g.n) break;
          float x = v[q];
          if (g.beta != 0.f) x += g.beta * cp[q];
          if (g.bias) x += g.bias[gn + q];
          if (g.relu) x = x > 0.f ? x : 0.f;
          cp[q] = x;
        }
      }
    }
  }
}

// True when k_gemm_f32_v's requirements hold for these operands.
inline bool f32_gemm_vector_ok(const F32GemmArgs& g) {
  auto a16 = [](const void* p) { return (((uintptr_t)p) & 15) == 0; };
  if (!a16(g.a) || !a16(g.b) || (g.lda & 3) || (g.ldb & 3) || (g.stride_a & 3) || (g.stride_b & 3)) return false;
  if (!g.trans_a && (g.k & 3)) return false;
  if (g.trans_a && (g.m & 3)) return false;
  if (!g.trans_b && (g.n & 3)) return false;
  if (g.trans_b && (g.k & 3)) return false;
  return true;
}

}  // namespace bbx
