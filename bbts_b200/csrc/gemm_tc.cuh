// Block matmul on the 5th-generation tensor cores (tcgen05) for sm_100a.
//
// One persistent kernel computes a *group* of independent block products
//     C_p = alpha_p * op(A_p) * op(B_p) (+ beta_p * C_p) (+ bias_p) (relu)
// for p = 0..P-1. This is the device side of the reference's block matmul ud
// (src/ud_functions/impls/dense_matrix_mult.cc:50-86: row-major C = op(A)op(B)
// with the transpose flags taken from params b0/b1) and of the FNN matmuls
// (applications/fnn/ffnn_activation_mult.cc:56-96 adds a column bias;
// ffnn_back_mult.cc:52-91 is the trans_a case).
//
// Layout: A_p is M x K (or K x M when trans_a), B_p is K x N (or N x K when
// trans_b), all row-major with arbitrary pitches that are multiples of 16 bytes.
// Operands whose K dimension is contiguous ("K-major") and operands whose M/N
// dimension is contiguous ("MN-major") are both read directly by TMA with the
// 128-byte swizzle; no transpose pass is needed.
//
// Roles inside a 192-thread CTA (320 with EP8):
//   warp 0      TMA producer (one elected lane) feeding a STAGES-deep smem ring
//   warp 1      TMEM allocator + MMA issuer (one elected lane)
//   warps 2..5  epilogue: tcgen05.ld from TMEM -> registers -> global (2..9 with
//               EP8: two warps per TMEM lane quarter, alternate 32-column chunks)
// The accumulator is double buffered in TMEM (2 x BN f32 columns), so the
// epilogue of tile t overlaps the main loop of tile t+1.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include "ptx.cuh"
#include "tile_order.h"

namespace bbx {

enum : int {
  EPI_RELU = 1,      // max(x, 0) after bias
  EPI_OUT_BF16 = 2,  // store bf16 instead of f32
  EPI_BIAS = 4,      // add bias[col]
  EPI_BETA = 8,      // read C and add beta * C
  EPI_TMA_STORE = 16,  // set by the host: C is written by TMA stores through tmap_c
  EPI_C_TRANS = 32,    // C is column-major: with EPI_TMA_STORE through tmap_c (boxes of 32 columns x 32
                       // rows of C), else by coalesced stores from registers
};

// One block product. 64-byte alignment is required by the tensor maps.
struct alignas(64) TcProblem {
  CUtensorMap tmap_a;  // 128 B
  CUtensorMap tmap_b;  // 128 B
  CUtensorMap tmap_c;  // 128 B, valid with EPI_TMA_STORE: 32-row x 64-byte boxes (row-major C) or
                       // 32 x 32-element boxes (column-major C), no swizzle
  void* c;
  const float* bias;
  long long ldc;       // elements
  int m, n, k;
  int tile_start;      // first global tile index of this problem
  int tiles_m, tiles_n;
  float alpha, beta;
  int flags;
  int pad_;
};

// Groups of up to kTcMaxInline problems travel in the kernel parameters (32 KB
// at most), tensor maps included: the TMA reads param-space maps fresh each
// launch, so these need no device table and no tensor-map acquire fence. A
// table map needs one per CTA and problem switch (about 0.3 us each, on the
// producer's path): moving config 1's 64-problem group into the parameters took
// it from 754 to 794 TFLOP/s.
constexpr int kTcMaxInline = 72;
static_assert(64 + kTcMaxInline * sizeof(TcProblem) <= 32764, "kernel parameters");

struct TcArgs {
  const TcProblem* table;  // device table, or nullptr to use `inline_probs`
  int num_problems;
  int total_tiles;
  uint32_t* status;        // device status word (0 = ok)
  TcProblem inline_probs[kTcMaxInline];
};

// Per-problem tile metadata (tile_start, tiles_m, tiles_n, k) is staged in
// shared memory for groups of up to kTcMetaMax problems, so locating a tile
// is an on-chip binary search instead of a chain of dependent global loads.
constexpr int kTcMetaMax = 512;
constexpr int kTcMetaBytes = kTcMetaMax * 16;
// Epilogue slots, one per epilogue warp, 1024-byte aligned: a 32 x 36 float
// staging buffer (the 144-byte pitch keeps 16-byte accesses conflict-free in
// both directions), or two alternating 32-row x 64-byte boxes for TMA stores of
// row-major C, or one 32 x 32-element box for column-major C.
constexpr int kTcEpiPitch = 36;
constexpr int kTcEpiSlot = 5120;
static_assert(32 * kTcEpiPitch * 4 <= kTcEpiSlot && 32 * 128 <= kTcEpiSlot && kTcEpiSlot % 1024 == 0, "epilogue slot");

// EP8: eight epilogue warps (two per TMEM lane quarter, taking alternate
// column chunks of the tile) and one shared-memory stage fewer. For groups of short
// main loops (K <= kTcEp8MaxK) the tile rate is set by the epilogue: measured
// on the contraction-only DAG, 4.08 -> 3.46 ms for its tensor groups; with
// long K the missing stage costs more than the extra warps give (the FP8 4096^3
// blocks: 2609 -> 2453 TFLOP/s), so the host picks it only for short K.
constexpr int kTcEp8MaxK = 512;
// The same for the 2-SM pair kernel's 256 x 256 tiles: config 1's 64 x 1024^3
// products 0.143 -> 0.128 ms. Not for longer K: with groups of K up to 2048 the
// 2000-op DAG's tensor groups ran 10 % faster alone but its makespan 2-4 %
// slower, and the FFN step (K = 2048) 3 % slower.
constexpr int kTc2Ep8MaxK = 1024;

template <int BN, bool A_MN, bool B_MN, bool FP8, bool EP8 = false>
struct TcCfg {
  static constexpr int BM = 128;
  static constexpr int BK_BYTES = 128;                // one 128-byte swizzle row of K
  static constexpr int ELEM = FP8 ? 1 : 2;
  static constexpr int BK = BK_BYTES / ELEM;          // 64 bf16 or 128 e4m3
  static constexpr int UMMA_K = FP8 ? 32 : 16;
  static constexpr int A_BYTES = BM * BK_BYTES;       // 16 KiB
  static constexpr int B_BYTES = BN * BK_BYTES;       // 32 or 16 KiB
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int STAGES = EP8 ? ((BN == 256) ? 3 : 5) : ((BN == 256) ? 4 : 6);
  static constexpr int TMEM_COLS = 2 * BN;            // double-buffered accumulator
  static constexpr int EPI_WARPS = EP8 ? 8 : 4;
  static constexpr int EPI_PARTS = EP8 ? 2 : 1;       // epilogue warps per TMEM lane quarter
  static constexpr int SMEM_BYTES =
      STAGES * STAGE_BYTES + 1024 /*align slack*/ + EPI_WARPS * kTcEpiSlot + 256 /*bars*/ + kTcMetaBytes;
  static constexpr int THREADS = 64 + 32 * EPI_WARPS;
  static constexpr int MN_BOX = 128 / ELEM;           // MN-major TMA box width (elements)
};

__device__ __forceinline__ const TcProblem* tc_problem(const TcArgs& args, int p) {
  return args.table ? (args.table + p) : (args.inline_probs + p);
}

// All threads of the CTA; visible after the prologue's __syncthreads.
__device__ __forceinline__ void tc_stage_meta(const TcArgs& args, int4* meta) {
  if (args.num_problems > kTcMetaMax) return;
  for (int i = threadIdx.x; i < args.num_problems; i += blockDim.x) {
    const TcProblem* pr = tc_problem(args, i);
    meta[i] = make_int4(pr->tile_start, pr->tiles_m, pr->tiles_n, pr->k);
  }
}

// Map a global tile index to (problem, tile_m, tile_n) and the problem's k.
// Tiles inside a problem are visited in bands of kTileBand = 16 tile-rows
// (band_tile, tile_order.h) so concurrently
// running CTAs share operand tiles in L2: a 4096^2 block's B panels are then
// read from DRAM once per problem (with bands of 8, twice; the pair kernel ran
// 1358 -> 1440 TFLOP/s on the 64 x 4096^3 step, same box and clock).
__device__ __forceinline__ void tc_locate(const TcArgs& args, const int4* meta, int t, int& p, int& tm, int& tn,
                                          int& k) {
  int lo = 0, hi = args.num_problems - 1;
  int4 e;
  if (args.num_problems <= kTcMetaMax) {
    while (lo < hi) {  // last problem with tile_start <= t
      const int mid = (lo + hi + 1) >> 1;
      if (meta[mid].x <= t) lo = mid; else hi = mid - 1;
    }
    e = meta[lo];
  } else {
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tc_problem(args, mid)->tile_start <= t) lo = mid; else hi = mid - 1;
    }
    const TcProblem* pr = tc_problem(args, lo);
    e = make_int4(pr->tile_start, pr->tiles_m, pr->tiles_n, pr->k);
  }
  p = lo;
  k = e.w;
  band_tile(t - e.x, e.y, e.z, tm, tn);
}

// Accumulator drain of one epilogue warp: its 32 rows (row0 .. row0+31, one
// TMEM lane each) x the tile's BN columns, 32 columns at a time.
//   1. each lane loads its row's 32 values (two tcgen05.ld, one wait), applies
//      alpha and the column bias and writes them to the warp's 32 x 36 buffer;
//   2. the warp writes the 32 rows back as contiguous segments -- f32: 8 lanes
//      x 16 B per 128-byte row segment, 4 rows per store; bf16: 4 lanes x 16 B,
//      8 rows per store -- adding beta * C, then ReLU, then converting.
// Row-per-lane stores would put every lane of a store in a different row (32
// half-sector writes per instruction); these write whole sectors. Warp-
// collective: every lane runs it; rows at or past m and columns at or past n
// are not written.
template <int BN, int PARTS = 1>
__device__ __forceinline__ void tc_epi_rows(const TcProblem* pr, uint32_t t_row, int row0, int lane, float* stage,
                                            int col_base, int part = 0) {
  const int flags = pr->flags;
  const float alpha = pr->alpha, beta = pr->beta;
  const long long ldc = pr->ldc;
  const int n = pr->n, m = pr->m;
  const bool has_bias = (flags & EPI_BIAS) != 0;
  const bool has_beta = (flags & EPI_BETA) != 0;
  const bool relu = (flags & EPI_RELU) != 0;
  if (flags & EPI_C_TRANS) {
    // column-major C without TMA stores: lane l holds row row0 + l, so for each
    // column the warp's 32 stores go to consecutive addresses (coalesced)
    const bool bf16 = (flags & EPI_OUT_BF16) != 0;
    const int row = row0 + lane;
#pragma unroll 1
    for (int c0 = 32 * part; c0 < BN; c0 += 32 * PARTS) {
      const int col = col_base + c0;
      if (col >= n || row0 >= m) break;  // warp-uniform
      uint32_t r0[16], r1[16];
      tmem_ld16_nowait(t_row + c0, r0);
      tmem_ld16_nowait(t_row + c0 + 16, r1);
      tmem_ld_wait();
      float v[32];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        v[i] = __uint_as_float(r0[i]) * alpha;
        v[16 + i] = __uint_as_float(r1[i]) * alpha;
      }
      if (has_bias) {
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (col + i < n) v[i] += pr->bias[col + i];
      }
      if (relu) {
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = fmaxf(v[i], 0.f);
      }
      if (row < m) {
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          if (col + i >= n) break;
          const long long idx = (long long)row + (long long)(col + i) * ldc;
          if (bf16) ((__nv_bfloat16*)pr->c)[idx] = __float2bfloat16_rn(v[i]);
          else ((float*)pr->c)[idx] = v[i];
        }
      }
    }
    return;
  }
  float* srow = stage + lane * kTcEpiPitch;
  // the buffer shares its slot with the TMA-store box of earlier tiles (a group
  // can mix problems with and without TMA stores): let those stores read it first
  if (lane == 0) bulk_wait_read_all();
  __syncwarp();
#pragma unroll 1
  for (int c = 2 * part; c < BN / 16; c += 2 * PARTS) {
    const int col0 = col_base + c * 16;
    if (col0 >= n) break;  // warp-uniform
    uint32_t r0[16], r1[16];
    tmem_ld16_nowait(t_row + c * 16, r0);
    tmem_ld16_nowait(t_row + (c + 1) * 16, r1);
    tmem_ld_wait();
    float x[32];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      x[i] = __uint_as_float(r0[i]) * alpha;
      x[16 + i] = __uint_as_float(r1[i]) * alpha;
    }
    if (has_bias) {
#pragma unroll
      for (int i = 0; i < 32; ++i)
        if (col0 + i < n) x[i] += pr->bias[col0 + i];
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) *(float4*)(srow + 4 * j) = make_float4(x[4 * j], x[4 * j + 1], x[4 * j + 2], x[4 * j + 3]);
    __syncwarp();
    if (flags & EPI_OUT_BF16) {
      const int rr = lane >> 2, cc = (lane & 3) * 8;
#pragma unroll
      for (int sidx = 0; sidx < 4; ++sidx) {
        const int r = sidx * 8 + rr, row = row0 + r, col = col0 + cc;
        if (row >= m || col >= n) continue;
        const float* sv = stage + r * kTcEpiPitch + cc;
        __nv_bfloat16* cp = (__nv_bfloat16*)pr->c + (long long)row * ldc + col;
        const float4 s0 = *(const float4*)sv, s1 = *(const float4*)(sv + 4);
        float v[8] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y, s1.z, s1.w};
        if (col + 8 <= n && ((((uintptr_t)cp) & 15) == 0)) {
          if (has_beta) {
            const uint4 o = *(const uint4*)cp;
            const __nv_bfloat162* h = (const __nv_bfloat162*)&o;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const float2 f = __bfloat1622float2(h[q]);
              v[2 * q] += beta * f.x;
              v[2 * q + 1] += beta * f.y;
            }
          }
          if (relu) {
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = fmaxf(v[q], 0.f);
          }
          uint4 pk;
          __nv_bfloat162* h = (__nv_bfloat162*)&pk;
#pragma unroll
          for (int q = 0; q < 4; ++q) h[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
          *(uint4*)cp = pk;
        } else {
          for (int q = 0; q < 8 && col + q < n; ++q) {
            float x = v[q];
            if (has_beta) x += beta * __bfloat162float(cp[q]);
            if (relu) x = fmaxf(x, 0.f);
            cp[q] = __float2bfloat16_rn(x);
          }
        }
      }
    } else {
      const int rr = lane >> 3, cc = (lane & 7) * 4;
#pragma unroll
      for (int sidx = 0; sidx < 8; ++sidx) {
        const int r = sidx * 4 + rr, row = row0 + r, col = col0 + cc;
        if (row >= m || col >= n) continue;
        const float* sv = stage + r * kTcEpiPitch + cc;
        float* cp = (float*)pr->c + (long long)row * ldc + col;
        const float4 s0 = *(const float4*)sv;
        float v[4] = {s0.x, s0.y, s0.z, s0.w};
        if (col + 4 <= n && ((((uintptr_t)cp) & 15) == 0)) {
          if (has_beta) {
            const float4 o = *(const float4*)cp;
            v[0] += beta * o.x; v[1] += beta * o.y; v[2] += beta * o.z; v[3] += beta * o.w;
          }
          if (relu) {
#pragma unroll
            for (int q = 0; q < 4; ++q) v[q] = fmaxf(v[q], 0.f);
          }
          *(float4*)cp = make_float4(v[0], v[1], v[2], v[3]);
        } else {
          for (int q = 0; q < 4 && col + q < n; ++q) {
            float x = v[q];
            if (has_beta) x += beta * cp[q];
            if (relu) x = fmaxf(x, 0.f);
            cp[q] = x;
          }
        }
      }
    }
    __syncwarp();  // the buffer is rewritten by the next 32 columns
  }
}

// Accumulator drain through TMA stores (problems with EPI_TMA_STORE: C's base
// and pitch meet the 16-byte rules, no beta * C). Row-major C: per 64 bytes of
// each of the warp's 32 rows (16 f32 or 32 bf16 columns), the lane of row r
// loads its values from TMEM, applies alpha, bias and ReLU, converts, and
// writes its 64 bytes into one of the warp's two alternating 32 x 64-byte
// boxes; one lane then issues the TMA store of the box, which clips rows >= m
// and columns >= n (the host takes this path only when a row of C is a whole
// number of 16-byte pieces, the granularity of the clip). A box is rewritten
// once the store issued from it has read it (cp.async.bulk.wait_group.read 1),
// so filling one box overlaps the store of the other; with a single box each
// 4 KB chunk waited for the previous store, which held the 2-SM headline
// kernel at 0.87 of the burst peak (0.92 with two boxes, same box). `box_sel`
// (per warp, kept across tiles) names the box to fill next; 2 means the last
// store read the whole 4 KB slot (column-major C). With EPI_C_TRANS
// (column-major C) the box is 32 columns x the warp's 32 rows, unswizzled, and
// m is the dimension a whole number of 16-byte pieces.
template <int BN, int PARTS = 1>
__device__ __forceinline__ void tc_epi_rows_tma(const TcProblem* pr, uint32_t t_row, int row0, int lane,
                                                uint8_t* box, int col_base, int& box_sel, int part = 0) {
  const int flags = pr->flags;
  const float alpha = pr->alpha;
  const int n = pr->n;
  const bool has_bias = (flags & EPI_BIAS) != 0;
  const bool relu = (flags & EPI_RELU) != 0;
  const bool bf16 = (flags & EPI_OUT_BF16) != 0;
  const int step = bf16 ? 64 : 32;  // columns per 128-byte row of the box
  if (row0 >= pr->m) return;  // warp-uniform: this warp's rows are all past the matrix, no box to store
  if (flags & EPI_C_TRANS) {
    box_sel = 2;  // its 4 KB box spans both 2 KB row-major boxes
    // column-major C: per 32 columns, the box holds column c's 32 rows (this
    // warp's) contiguously; lane l writes element l of every box row
#pragma unroll 1
    for (int c0 = 32 * part; c0 < BN; c0 += 32 * PARTS) {
      const int col = col_base + c0;
      if (col >= n) break;  // warp-uniform
      uint32_t r0[16], r1[16];
      tmem_ld16_nowait(t_row + c0, r0);
      tmem_ld16_nowait(t_row + c0 + 16, r1);
      tmem_ld_wait();
      float v[32];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        v[i] = __uint_as_float(r0[i]) * alpha;
        v[16 + i] = __uint_as_float(r1[i]) * alpha;
      }
      if (has_bias) {
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (col + i < n) v[i] += pr->bias[col + i];
      }
      if (relu) {
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = fmaxf(v[i], 0.f);
      }
      if (lane == 0) bulk_wait_read_all();  // the previous store has read the box
      __syncwarp();
      if (bf16) {
#pragma unroll
        for (int i = 0; i < 32; ++i) ((__nv_bfloat16*)box)[i * 32 + lane] = __float2bfloat16_rn(v[i]);
      } else {
#pragma unroll
        for (int i = 0; i < 32; ++i) ((float*)box)[i * 32 + lane] = v[i];
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) {
        tma_store_2d(&pr->tmap_c, box, row0, col);
        bulk_commit();
      }
    }
    return;
  }
  // row-major C: per 64 bytes of the warp's 32 rows (16 f32 / 32 bf16
  // columns) each lane writes its row's 64 bytes into one of two alternating
  // 32 x 64-byte boxes, and one lane stores the box with TMA; a box is
  // rewritten once the store issued from it has read it (wait_group.read 1:
  // the other box's store may still be reading)
  (void)step;
  const int half = bf16 ? 32 : 16;
  if (box_sel == 2) {  // the last store read the whole 4 KB box (column-major C): let it finish
    if (lane == 0) bulk_wait_read_all();
    box_sel = 0;
  }
#pragma unroll 1
  for (int c0 = half * part; c0 < BN; c0 += half * PARTS) {
    const int col = col_base + c0;
    if (col >= n) break;  // warp-uniform
    uint32_t r0[16], r1[16];
    tmem_ld16_nowait(t_row + c0, r0);
    if (bf16) tmem_ld16_nowait(t_row + c0 + 16, r1);
    tmem_ld_wait();
    uint4 q[4];
    if (bf16) {
      float v[32];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        v[i] = __uint_as_float(r0[i]) * alpha;
        v[16 + i] = __uint_as_float(r1[i]) * alpha;
      }
      if (has_bias) {
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (col + i < n) v[i] += pr->bias[col + i];
      }
      if (relu) {
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = fmaxf(v[i], 0.f);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        __nv_bfloat162 h[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) h[t] = __floats2bfloat162_rn(v[8 * j + 2 * t], v[8 * j + 2 * t + 1]);
        q[j] = make_uint4(*(uint32_t*)&h[0], *(uint32_t*)&h[1], *(uint32_t*)&h[2], *(uint32_t*)&h[3]);
      }
    } else {
      float v[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r0[i]) * alpha;
      if (has_bias) {
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (col + i < n) v[i] += pr->bias[col + i];
      }
      if (relu) {
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i], 0.f);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j)
        q[j] = make_uint4(__float_as_uint(v[4 * j]), __float_as_uint(v[4 * j + 1]), __float_as_uint(v[4 * j + 2]),
                          __float_as_uint(v[4 * j + 3]));
    }
    uint8_t* hb = box + box_sel * 2048;
    if (lane == 0) bulk_wait_read_1();
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 4; ++j) *(uint4*)(hb + lane * 64 + j * 16) = q[j];
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) {
      tma_store_2d(&pr->tmap_c, hb, col, row0);
      bulk_commit();
    }
    box_sel ^= 1;
  }
}

// Tile of CTA blockIdx.x in round `round` (snake order, snake_tile_of in
// tile_order.h). The producer, MMA and epilogue warps all walk this sequence.
__device__ __forceinline__ int snake_tile(int t0, int round, int total) {
  return snake_tile_of(t0, round, total, (int)blockIdx.x, (int)gridDim.x);
}

template <int BN, bool A_MN, bool B_MN, bool FP8, bool EP8>
__global__ void __launch_bounds__(EP8 ? 320 : 192, 1) tc_gemm_kernel(const __grid_constant__ TcArgs args) {
  using C = TcCfg<BN, A_MN, B_MN, FP8, EP8>;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte alignment for the 128B-swizzle atoms.
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* stage_base = smem;
  uint8_t* epi_base = smem + C::STAGES * C::STAGE_BYTES;  // 4 epilogue slots, 1024-byte aligned
  uint64_t* bars = (uint64_t*)(epi_base + C::EPI_WARPS * kTcEpiSlot);
  uint64_t* full_bar = bars;                       // [STAGES]
  uint64_t* empty_bar = bars + C::STAGES;          // [STAGES]
  uint64_t* tfull_bar = bars + 2 * C::STAGES;      // [2]
  uint64_t* tempty_bar = bars + 2 * C::STAGES + 2; // [2]
  uint32_t* tmem_slot = (uint32_t*)(bars + 2 * C::STAGES + 4);
  int4* meta = (int4*)((uint8_t*)bars + 256);  // [kTcMetaMax]
  volatile uint32_t* status = args.status;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  // epilogue warps 2..5: one slot each (staging buffer or TMA-store box)
  uint8_t* epi_buf = epi_base + (warp >= 2 ? (warp - 2) * kTcEpiSlot : 0);
  float* epi_stage = (float*)epi_buf;

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull_bar[b], 1);
      mbar_init(&tempty_bar[b], 32 * C::EPI_WARPS);
    }
    fence_mbar_init();
  }
  tc_stage_meta(args, meta);
  if (warp == 1) tmem_alloc(tmem_slot, C::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      int last_p = -1;
      for (int t0 = blockIdx.x, rr = 0; t0 < args.total_tiles && ok; t0 += gridDim.x, ++rr) {
        const int t = snake_tile(t0, rr, args.total_tiles);
        int p, tm, tn, kdim;
        tc_locate(args, meta, t, p, tm, tn, kdim);
        const TcProblem* pr = tc_problem(args, p);
        if (args.table && p != last_p) {
          tensormap_acquire(&pr->tmap_a);
          tensormap_acquire(&pr->tmap_b);
          last_p = p;
        }
        if (args.table && t + (int)gridDim.x < args.total_tiles) {
          // the next tile's tensor maps, if it starts a new problem
          int p2, tm2, tn2, k2;
          tc_locate(args, meta, t + gridDim.x, p2, tm2, tn2, k2);
          if (p2 != p) {
            prefetch_tensormap(&args.table[p2].tmap_a);
            prefetch_tensormap(&args.table[p2].tmap_b);
          }
        }
        const int kb_n = (kdim + C::BK - 1) / C::BK;
        for (int kb = 0; kb < kb_n; ++kb) {
          if (!mbar_wait(&empty_bar[s], ph ^ 1, status, DEV_TIMEOUT_EMPTY)) { ok = false; break; }
          uint8_t* sa = stage_base + s * C::STAGE_BYTES;
          uint8_t* sb = sa + C::A_BYTES;
          mbar_arrive_expect_tx(&full_bar[s], C::STAGE_BYTES);
          const int k0 = kb * C::BK;
          if constexpr (!A_MN) {
            tma_load_2d(sa, &pr->tmap_a, &full_bar[s], k0, tm * C::BM);
          } else {
#pragma unroll
            for (int j = 0; j < C::BM / C::MN_BOX; ++j)
              tma_load_2d(sa + j * (C::BK * 128), &pr->tmap_a, &full_bar[s],
                          tm * C::BM + j * C::MN_BOX, k0);
          }
          if constexpr (!B_MN) {
            tma_load_2d(sb, &pr->tmap_b, &full_bar[s], k0, tn * BN);
          } else {
#pragma unroll
            for (int j = 0; j < BN / C::MN_BOX; ++j)
              tma_load_2d(sb + j * (C::BK * 128), &pr->tmap_b, &full_bar[s],
                          tn * BN + j * C::MN_BOX, k0);
          }
          if (++s == C::STAGES) { s = 0; ph ^= 1; }
        }
      }
      // Drain: make sure every issued TMA has landed before the CTA may exit.
      for (int i = 0; i < C::STAGES; ++i) {
        if (!mbar_wait(&empty_bar[s], ph ^ 1, status, DEV_TIMEOUT_EMPTY)) break;
        if (++s == C::STAGES) { s = 0; ph ^= 1; }
      }
      if (*status != DEV_OK) {
        // Error path: the consumer stopped early, so give copies still in
        // flight a bounded grace period (~100 us) before the CTA exits.
        const long long t0 = clock64();
        while (clock64() - t0 < 200000) {}
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      constexpr uint32_t kFmt = FP8 ? 0u : 1u;  // e4m3 / bf16
      constexpr uint32_t idesc = make_idesc(C::BM, BN, kFmt, A_MN, B_MN);
      int s = 0;
      uint32_t ph = 0;
      int acc = 0;
      uint32_t acc_ph = 0;
      bool ok = true;
      for (int t0 = blockIdx.x, rr = 0; t0 < args.total_tiles && ok; t0 += gridDim.x, ++rr) {
        const int t = snake_tile(t0, rr, args.total_tiles);
        int p, tm, tn, kdim;
        tc_locate(args, meta, t, p, tm, tn, kdim);
        const int kb_n = (kdim + C::BK - 1) / C::BK;
        if (!mbar_wait(&tempty_bar[acc], acc_ph ^ 1, status, DEV_TIMEOUT_TMEM_EMPTY)) break;
        tc_fence_after();
        const uint32_t d_tmem = tmem_base + acc * BN;
        for (int kb = 0; kb < kb_n; ++kb) {
          if (!mbar_wait(&full_bar[s], ph, status, DEV_TIMEOUT_FULL)) { ok = false; break; }
          tc_fence_after();
          const uint32_t sa = smem_u32(stage_base + s * C::STAGE_BYTES);
          const uint32_t sb = sa + C::A_BYTES;
#pragma unroll
          for (int kk = 0; kk < C::BK / C::UMMA_K; ++kk) {
            uint64_t da, db;
            if constexpr (!A_MN) da = smem_desc_sw128(sa + kk * 32, 16, 1024);
            else da = smem_desc_sw128(sa + kk * (C::UMMA_K * 128), C::BK * 128, 1024);
            if constexpr (!B_MN) db = smem_desc_sw128(sb + kk * 32, 16, 1024);
            else db = smem_desc_sw128(sb + kk * (C::UMMA_K * 128), C::BK * 128, 1024);
            const uint32_t accum = (kb > 0 || kk > 0) ? 1u : 0u;
            if constexpr (FP8) umma_f8(d_tmem, da, db, idesc, accum);
            else umma_f16(d_tmem, da, db, idesc, accum);
          }
          umma_commit(&empty_bar[s]);  // frees the stage once these MMAs retire
          if (++s == C::STAGES) { s = 0; ph ^= 1; }
        }
        if (!ok) break;
        umma_commit(&tfull_bar[acc]);  // accumulator ready for the epilogue
        if (++acc == 2) { acc = 0; acc_ph ^= 1; }
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int lane_base = 32 * (warp & 3);
    int acc = 0;
    uint32_t acc_ph = 0;
    int last_p = -1;
    int box_sel = 0;
    for (int t0 = blockIdx.x, rr = 0; t0 < args.total_tiles; t0 += gridDim.x, ++rr) {
      const int t = snake_tile(t0, rr, args.total_tiles);
      int p, tm, tn, kdim;
      tc_locate(args, meta, t, p, tm, tn, kdim);
      const TcProblem* pr = tc_problem(args, p);
      if (args.table && p != last_p) {
        if (lane == 0 && (pr->flags & EPI_TMA_STORE)) tensormap_acquire(&pr->tmap_c);
        last_p = p;
      }
      // Warp-uniform outcome: tcgen05.ld below is warp-collective.
      const bool got = mbar_wait(&tfull_bar[acc], acc_ph, status, DEV_TIMEOUT_TMEM_FULL);
      if (!__all_sync(0xffffffffu, got)) break;
      tc_fence_after();
      // with EP8 warps 2..5 and 6..9 take alternate column chunks of the tile (even
      // and odd), so a problem whose n ends inside the tile splits its chunks evenly
      const int part = EP8 ? (warp - 2) >> 2 : 0;
      const uint32_t t_row = tmem_base + acc * BN + ((uint32_t)lane_base << 16);
      if (pr->flags & EPI_TMA_STORE)
        tc_epi_rows_tma<BN, C::EPI_PARTS>(pr, t_row, tm * C::BM + lane_base, lane, epi_buf, tn * BN, box_sel, part);
      else tc_epi_rows<BN, C::EPI_PARTS>(pr, t_row, tm * C::BM + lane_base, lane, epi_stage, tn * BN, part);
      tc_fence_before();
      mbar_arrive(&tempty_bar[acc]);
      if (++acc == 2) { acc = 0; acc_ph ^= 1; }
    }
    if (lane == 0) bulk_wait_all();  // this warp's TMA stores have landed before the CTA ends
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem_base, C::TMEM_COLS);
  }
}

// ============================================================================
// 2-SM variant: a cluster of two CTAs computes one 256 x 256 tile with
// tcgen05.mma.cta_group::2 (M = 256 split over the pair's TMEM, N = 256 split
// over the pair's shared memory). Each CTA TMA-loads only ITS half of A (128
// rows) and of B (128 rows / columns) -- no multicast -- so the operand bytes
// each SM pulls per FLOP are a third lower than the 1-SM 128 x 256 tile and the
// 32 KiB stages allow a 6-deep ring. Both CTAs' loads complete on the leader's
// full barrier; the leader's single MMA thread commits each stage back to the
// empty barriers of both CTAs and each accumulator to both CTAs' tfull
// barriers; both epilogues release the accumulator on the leader's tempty.
// bf16 only.
// ============================================================================
template <bool A_MN, bool B_MN, bool EP8 = false>
struct Tc2Cfg {
  static constexpr int BM = 256;  // rows per pair (128 per CTA)
  static constexpr int BN = 256;  // columns per pair (128 B rows per CTA)
  static constexpr int BK = 64;
  static constexpr int UMMA_K = 16;
  static constexpr int A_BYTES = 128 * 128;  // 128 rows x 128 B
  static constexpr int B_BYTES = 128 * 128;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  // EP8: eight epilogue warps per CTA (two per TMEM lane quarter, alternate
  // 32-column chunks) and one stage fewer, as in the 1-SM kernel
  static constexpr int STAGES = EP8 ? 5 : 6;
  static constexpr int TMEM_COLS = 512;
  static constexpr int EPI_WARPS = EP8 ? 8 : 4;
  static constexpr int EPI_PARTS = EP8 ? 2 : 1;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256 + kTcMetaBytes + EPI_WARPS * kTcEpiSlot;
  static constexpr int THREADS = 64 + 32 * EPI_WARPS;
};

template <bool A_MN, bool B_MN, bool EP8>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(EP8 ? 320 : 192, 1)
    tc_gemm2_kernel(const __grid_constant__ TcArgs args) {
  using C = Tc2Cfg<A_MN, B_MN, EP8>;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* stage_base = smem;
  uint8_t* epi_base = smem + C::STAGES * C::STAGE_BYTES;  // EPI_WARPS epilogue slots, 1024-byte aligned
  uint64_t* bars = (uint64_t*)(epi_base + C::EPI_WARPS * kTcEpiSlot);
  uint64_t* full_bar = bars;
  uint64_t* empty_bar = bars + C::STAGES;
  uint64_t* tfull_bar = bars + 2 * C::STAGES;
  uint64_t* tempty_bar = bars + 2 * C::STAGES + 2;
  uint32_t* tmem_slot = (uint32_t*)(bars + 2 * C::STAGES + 4);
  int4* meta = (int4*)((uint8_t*)bars + 256);  // [kTcMetaMax]
  volatile uint32_t* status = args.status;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  // epilogue warps 2..5: one slot each (staging buffer or TMA-store box)
  uint8_t* epi_buf = epi_base + (warp >= 2 ? (warp - 2) * kTcEpiSlot : 0);
  float* epi_stage = (float*)epi_buf;
  const uint32_t rank = cluster_ctarank();
  const bool leader = rank == 0;
  const int pair = blockIdx.x >> 1, num_pairs = gridDim.x >> 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull_bar[b], 1);
      mbar_init(&tempty_bar[b], 2 * 32 * C::EPI_WARPS);  // both CTAs' epilogue threads
    }
    fence_mbar_init();
  }
  tc_stage_meta(args, meta);
  if (warp == 1) tmem_alloc_2sm(tmem_slot, C::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  __syncwarp();
  cluster_sync();  // peer barriers initialised before any remote arrive / complete_tx
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ------------------------------------------------------------ producer (both CTAs)
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      int last_p = -1;
      for (int t0 = pair, rr = 0; t0 < args.total_tiles && ok; t0 += num_pairs, ++rr) {
        const int t = snake_tile_of(t0, rr, args.total_tiles, pair, num_pairs);
        int p, tm, tn, kdim;
        tc_locate(args, meta, t, p, tm, tn, kdim);
        const TcProblem* pr = tc_problem(args, p);
        if (args.table && p != last_p) {
          tensormap_acquire(&pr->tmap_a);
          tensormap_acquire(&pr->tmap_b);
          last_p = p;
        }
        if (args.table && t0 + num_pairs < args.total_tiles) {
          // the next tile's tensor maps, if it starts a new problem
          int p2, tm2, tn2, k2;
          tc_locate(args, meta, snake_tile_of(t0 + num_pairs, rr + 1, args.total_tiles, pair, num_pairs), p2, tm2,
                    tn2, k2);
          if (p2 != p) {
            prefetch_tensormap(&args.table[p2].tmap_a);
            prefetch_tensormap(&args.table[p2].tmap_b);
          }
        }
        const int kb_n = (kdim + C::BK - 1) / C::BK;
        for (int kb = 0; kb < kb_n; ++kb) {
          if (!mbar_wait(&empty_bar[s], ph ^ 1, status, DEV_TIMEOUT_EMPTY)) { ok = false; break; }
          uint8_t* sa = stage_base + s * C::STAGE_BYTES;
          uint8_t* sb = sa + C::A_BYTES;
          if (leader) mbar_arrive_expect_tx(&full_bar[s], 2 * C::STAGE_BYTES);
          const uint32_t bar = mapa_shared(smem_u32(&full_bar[s]), 0);
          const int k0 = kb * C::BK;
          const int row_a = tm * C::BM + (int)rank * 128;
          const int row_b = tn * C::BN + (int)rank * 128;
          if constexpr (!A_MN) {
            tma_load_2d_2sm(sa, &pr->tmap_a, bar, k0, row_a);
          } else {
            tma_load_2d_2sm(sa, &pr->tmap_a, bar, row_a, k0);
            tma_load_2d_2sm(sa + C::BK * 128, &pr->tmap_a, bar, row_a + 64, k0);
          }
          if constexpr (!B_MN) {
            tma_load_2d_2sm(sb, &pr->tmap_b, bar, k0, row_b);
          } else {
            tma_load_2d_2sm(sb, &pr->tmap_b, bar, row_b, k0);
            tma_load_2d_2sm(sb + C::BK * 128, &pr->tmap_b, bar, row_b + 64, k0);
          }
          if (++s == C::STAGES) { s = 0; ph ^= 1; }
        }
      }
      for (int i = 0; i < C::STAGES; ++i) {
        if (!mbar_wait(&empty_bar[s], ph ^ 1, status, DEV_TIMEOUT_EMPTY)) break;
        if (++s == C::STAGES) { s = 0; ph ^= 1; }
      }
      if (*status != DEV_OK) {
        const long long t0 = clock64();
        while (clock64() - t0 < 200000) {}
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer (leader CTA only)
    if (leader && lane == 0) {
      constexpr uint32_t idesc = make_idesc(256, 256, 1u, A_MN, B_MN);
      int s = 0;
      uint32_t ph = 0;
      int acc = 0;
      uint32_t acc_ph = 0;
      bool ok = true;
      for (int t0 = pair, rr = 0; t0 < args.total_tiles && ok; t0 += num_pairs, ++rr) {
        const int t = snake_tile_of(t0, rr, args.total_tiles, pair, num_pairs);
        int p, tm, tn, kdim;
        tc_locate(args, meta, t, p, tm, tn, kdim);
        const int kb_n = (kdim + C::BK - 1) / C::BK;
        if (!mbar_wait(&tempty_bar[acc], acc_ph ^ 1, status, DEV_TIMEOUT_TMEM_EMPTY)) break;
        tc_fence_after();
        const uint32_t d_tmem = tmem_base + acc * C::BN;
        for (int kb = 0; kb < kb_n; ++kb) {
          if (!mbar_wait(&full_bar[s], ph, status, DEV_TIMEOUT_FULL)) { ok = false; break; }
          tc_fence_after();
          const uint32_t sa = smem_u32(stage_base + s * C::STAGE_BYTES);
          const uint32_t sb = sa + C::A_BYTES;
#pragma unroll
          for (int kk = 0; kk < C::BK / C::UMMA_K; ++kk) {
            uint64_t da, db;
            if constexpr (!A_MN) da = smem_desc_sw128(sa + kk * 32, 16, 1024);
            else da = smem_desc_sw128(sa + kk * (C::UMMA_K * 128), C::BK * 128, 1024);
            if constexpr (!B_MN) db = smem_desc_sw128(sb + kk * 32, 16, 1024);
            else db = smem_desc_sw128(sb + kk * (C::UMMA_K * 128), C::BK * 128, 1024);
            umma_f16_2sm(d_tmem, da, db, idesc, (kb > 0 || kk > 0) ? 1u : 0u);
          }
          umma_commit_2sm(&empty_bar[s], 0x3);
          if (++s == C::STAGES) { s = 0; ph ^= 1; }
        }
        if (!ok) break;
        umma_commit_2sm(&tfull_bar[acc], 0x3);
        if (++acc == 2) { acc = 0; acc_ph ^= 1; }
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue (both CTAs)
    const int lane_base = 32 * (warp & 3);
    const uint32_t tempty_leader0 = mapa_shared(smem_u32(&tempty_bar[0]), 0);
    const uint32_t tempty_leader1 = mapa_shared(smem_u32(&tempty_bar[1]), 0);
    int acc = 0;
    uint32_t acc_ph = 0;
    int last_p = -1;
    int box_sel = 0;
    for (int t0 = pair, rr = 0; t0 < args.total_tiles; t0 += num_pairs, ++rr) {
      const int t = snake_tile_of(t0, rr, args.total_tiles, pair, num_pairs);
      int p, tm, tn, kdim;
      tc_locate(args, meta, t, p, tm, tn, kdim);
      const TcProblem* pr = tc_problem(args, p);
      if (args.table && p != last_p) {
        if (lane == 0 && (pr->flags & EPI_TMA_STORE)) tensormap_acquire(&pr->tmap_c);
        last_p = p;
      }
      const bool got = mbar_wait(&tfull_bar[acc], acc_ph, status, DEV_TIMEOUT_TMEM_FULL);
      if (!__all_sync(0xffffffffu, got)) break;
      tc_fence_after();
      const uint32_t t_row = tmem_base + acc * C::BN + ((uint32_t)lane_base << 16);
      const int row0 = tm * C::BM + (int)rank * 128 + lane_base;
      const int part = EP8 ? (warp - 2) >> 2 : 0;
      if (pr->flags & EPI_TMA_STORE)
        tc_epi_rows_tma<C::BN, C::EPI_PARTS>(pr, t_row, row0, lane, epi_buf, tn * C::BN, box_sel, part);
      else tc_epi_rows<C::BN, C::EPI_PARTS>(pr, t_row, row0, lane, epi_stage, tn * C::BN, part);
      tc_fence_before();
      mbar_arrive_cluster(acc == 0 ? tempty_leader0 : tempty_leader1);
      if (++acc == 2) { acc = 0; acc_ph ^= 1; }
    }
    if (lane == 0) bulk_wait_all();  // this warp's TMA stores have landed before the CTA ends
  }

  // the leader's MMAs read the peer's shared memory: neither CTA may release
  // TMEM or exit before both are done
  tc_fence_before();
  __syncthreads();
  __syncwarp();
  cluster_sync();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc_2sm(tmem_base, C::TMEM_COLS);
  }
}

}  // namespace bbx
