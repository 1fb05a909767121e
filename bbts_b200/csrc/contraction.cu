// einsum contraction of the reference's "cutensor" block library
// (libraries/cutensor/contraction.h): out = alpha * sum(lhs * rhs) over the
// modes absent from the output, on column-major rank<=4 FP32 tensors.
//
// Lowering (stream-ordered temporaries for the per-call entry point; arena
// slots in the DAG executor):
//   1. classify every mode as I (lhs+out), N (rhs+out), K (lhs+rhs, summed),
//      B (all three, batch), L (lhs only, summed) or R (rhs only, summed) --
//      the same classes the reference's cpu_op plan uses (contraction.h:229-253);
//   2. gather lhs into Lc[b][m][k] and rhs into Rc[b][n][k] (k contiguous,
//      pitch padded to 16 bytes for the tensor-core path, L/R modes summed in
//      the gather);
//   3. batched matmul Ct[b][n][m] = alpha * Rc[b] * Lc[b]^T: SIMT FP32 or
//      tcgen05 BF16 with f32 accumulation;
//   4. if the output's mode order is (I..., N..., B...), Ct already is the
//      column-major output and step 3 wrote it in place; otherwise gather Ct
//      into the output order.
// Inside every group, modes are flattened column-major (first mode fastest),
// I/N/B in output order and K in lhs order.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <vector>
#include "bbts_b200.h"
#include "common.h"
#include "contraction.h"
#include "ptx.cuh"

namespace bbx {

__device__ __forceinline__ void gather_one(const float* __restrict__ in, void* out, int out_bf16,
                                           const GatherArgs& a, long long e) {
  long long rem = e, src = 0, dst = 0;
  for (int d = a.rank_o - 1; d >= 0; --d) {
    long long idx = rem % a.odims[d];
    rem /= a.odims[d];
    src += idx * a.istride[d];
    dst += idx * a.ostride[d];
  }
  float v;
  if (a.rank_s == 0) {
    v = in[src];
  } else {
    long long ns = 1;
    for (int d = 0; d < a.rank_s; ++d) ns *= a.sdims[d];
    v = 0.f;
    for (long long s = 0; s < ns; ++s) {
      long long r = s, off = 0;
      for (int d = 0; d < a.rank_s; ++d) {
        off += (r % a.sdims[d]) * a.sstride[d];
        r /= a.sdims[d];
      }
      v += in[src + off];
    }
  }
  if (out_bf16) ((__nv_bfloat16*)out)[dst] = __float2bfloat16_rn(v);
  else ((float*)out)[dst] = v;
}

__global__ void k_gather_sum(const float* __restrict__ in, void* out, int out_bf16,
                             const __grid_constant__ GatherArgs a, long long n) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    gather_one(in, out, out_bf16, a, e);
}

constexpr long long kGatherChunk = 4096;

// Row path: after merging, the innermost output mode is unit-stride in both the
// source and the destination and nothing is summed. Work items are (row,
// segment) pairs, a segment being up to kGatherSeg elements of one row, so
// short rows and rows as long as a whole tensor both spread over warps. Each
// warp carries kRowsPerWarp items at once, so every lane keeps that many
// independent loads in flight.
constexpr int kRowsPerWarp = 4;

static bool row_mode_ok(const GatherArgs& a) {
  const int last = a.rank_o - 1;
  return a.rank_s == 0 && last >= 0 && a.istride[last] == 1 && a.ostride[last] == 1 && a.odims[last] >= 16;
}

void simplify_gather(GatherArgs* a) {
  if (a->rank_o <= 1) return;
  long long od[4], is[4], os[4];  // fastest first
  int r = 1;
  od[0] = a->odims[a->rank_o - 1];
  is[0] = a->istride[a->rank_o - 1];
  os[0] = a->ostride[a->rank_o - 1];
  for (int d = a->rank_o - 2; d >= 0; --d) {
    if (a->istride[d] == is[r - 1] * od[r - 1] && a->ostride[d] == os[r - 1] * od[r - 1]) {
      od[r - 1] *= a->odims[d];  // (i_d, i_f) -> i_d * n_f + i_f on both sides
    } else {
      od[r] = a->odims[d];
      is[r] = a->istride[d];
      os[r] = a->ostride[d];
      ++r;
    }
  }
  a->rank_o = r;
  for (int q = 0; q < r; ++q) {
    a->odims[q] = od[r - 1 - q];
    a->istride[q] = is[r - 1 - q];
    a->ostride[q] = os[r - 1 - q];
  }
}

static void set_row_mode(GatherRec* r) {
  r->row_mode = row_mode_ok(r->a) ? 1 : 0;
  if (!r->row_mode) {
    r->row_len = r->segs = r->items_per_chunk = 0;
    return;
  }
  r->row_len = r->a.odims[r->a.rank_o - 1];
  r->segs = (r->row_len + kGatherSeg - 1) / kGatherSeg;
  r->items_per_chunk = std::max<long long>(32, 4 * kGatherChunk / std::min(r->row_len, kGatherSeg));
}

static long long row_items(const GatherRec& r) { return (r.n / r.row_len) * r.segs; }

__device__ __forceinline__ void gather_rows(const GatherRec& rec, long long item0, long long item1) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  // the record's fields in registers: stores to the destination could alias
  // the record as far as the compiler knows, which would reload it every item
  const int outer = rec.a.rank_o - 1;  // dims 0 .. outer-1 index rows, dim `outer` runs along a row
  long long odims[3], istr[3], ostr[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    odims[d] = d < outer ? rec.a.odims[d] : 1;
    istr[d] = d < outer ? rec.a.istride[d] : 0;
    ostr[d] = d < outer ? rec.a.ostride[d] : 0;
  }
  const float* __restrict__ src = rec.src;
  void* const dst = rec.dst;
  const bool bf16 = rec.dst_bf16 != 0;
  const long long row_len = rec.row_len, segs = rec.segs;
  for (long long it = item0 + (long long)warp * kRowsPerWarp; it < item1; it += (long long)nwarps * kRowsPerWarp) {
    long long so[kRowsPerWarp], dso[kRowsPerWarp];
    int len[kRowsPerWarp];
    int maxlen = 0;
#pragma unroll
    for (int u = 0; u < kRowsPerWarp; ++u) {
      so[u] = dso[u] = 0;
      len[u] = 0;
      const long long item = it + u;
      if (item < item1) {
        const long long row = item / segs, start = (item - row * segs) * kGatherSeg;
        long long rem = row, s = start, t = start;
#pragma unroll
        for (int d = 2; d >= 0; --d) {
          if (d < outer) {
            const long long idx = rem % odims[d];
            rem /= odims[d];
            s += idx * istr[d];
            t += idx * ostr[d];
          }
        }
        so[u] = s;
        dso[u] = t;
        len[u] = (int)min(kGatherSeg, row_len - start);
        maxlen = max(maxlen, len[u]);
      }
    }
    // four 32-element steps per pass: 16 independent loads per lane in flight
    for (int x0 = lane; x0 < maxlen; x0 += 128) {
      float v[kRowsPerWarp][4];
#pragma unroll
      for (int u = 0; u < kRowsPerWarp; ++u)
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (x0 + 32 * q < len[u]) v[u][q] = __ldg(src + so[u] + x0 + 32 * q);
#pragma unroll
      for (int u = 0; u < kRowsPerWarp; ++u) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int x = x0 + 32 * q;
          if (x < len[u]) {
            if (bf16) ((__nv_bfloat16*)dst)[dso[u] + x] = __float2bfloat16_rn(v[u][q]);
            else ((float*)dst)[dso[u] + x] = v[u][q];
          }
        }
      }
    }
  }
}

// One gather record on the row path (the per-call contraction).
__global__ void k_gather_rows1(const __grid_constant__ GatherRec r, long long chunks) {
  const long long items = (r.n / r.row_len) * r.segs;
  for (long long c = blockIdx.x; c < chunks; c += gridDim.x) {
    const long long i0 = c * r.items_per_chunk;
    gather_rows(r, i0, min(i0 + r.items_per_chunk, items));
  }
}

// Many gathers in one launch: chunk c belongs to the record whose
// [chunk_start, next chunk_start) range holds it.
// A CTA's chunks come in increasing order, so after a binary search for the
// first one the record index only moves forward. Four CTAs per SM (64
// registers, a few spilled): the row loop's loads are latency-bound, and the
// 2000-op DAG's input gathers went 0.83 -> 0.59 ms against three CTAs at 80.
__global__ void __launch_bounds__(256, 4) k_gather_group(const GatherRec* __restrict__ recs, int count, long long total_chunks) {
  int lo = -1;
  for (long long c = blockIdx.x; c < total_chunks; c += gridDim.x) {
    if (lo < 0) {
      int hi = count - 1;
      lo = 0;
      while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (recs[mid].chunk_start <= c) lo = mid; else hi = mid - 1;
      }
    } else {
      while (lo + 1 < count && recs[lo + 1].chunk_start <= c) ++lo;
    }
    const GatherRec& r = recs[lo];
    if (r.row_mode) {
      const long long i0 = (c - r.chunk_start) * r.items_per_chunk;
      gather_rows(r, i0, min(i0 + r.items_per_chunk, (r.n / r.row_len) * r.segs));
      continue;
    }
    const long long e0 = (c - r.chunk_start) * kGatherChunk;
    const long long e1 = min(e0 + kGatherChunk, r.n);
    for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x) gather_one(r.src, r.dst, r.dst_bf16, r.a, e);
  }
}

// ---- bulk-staged row gather: every record on the row path, its source 16-byte
// aligned and every destination row 16-byte aligned (the tensor-core staging
// blocks, whose pitches are padded to 16 bytes). One CTA per SM:
//  - a producer warp deals items (one row segment of up to kGatherSeg
//    elements) kGBItems to a stage: lane u finds item u's record and row,
//    and copies the segment's whole 16-byte blocks into the stage with one
//    cp.async.bulk, completing on the stage's `full` mbarrier;
//  - kGBConsumerWarps warps convert each staged segment and store it (8-byte
//    bf16 / 16-byte f32 stores where the source row is 16-byte aligned, else
//    element by element); the at most 3 + 3 elements before the first and
//    after the last whole block are read from global memory directly.
// The loads leave the consumers' critical path (the row kernel above issues
// element loads and waits on them).
constexpr int kGBStages = 3;
constexpr int kGBItems = 16;
constexpr int kGBItemBytes = (int)kGatherSeg * 4;
constexpr int kGBSlot = kGBItems * kGBItemBytes;  // 64 KiB
constexpr int kGBConsumerWarps = 8;
constexpr int kGBThreads = 32 * (kGBConsumerWarps + 1);
constexpr int kGBMaxRecs = 1024;
struct GBItem {
  long long so, dso, c0, c1;  // source / destination element of the segment; its whole blocks [c0, c1)
  const float* src;           // the record's source and destination (consumers read no record)
  void* dst;
  int len, bf16;              // elements (0: no item); destination bf16
};
constexpr int kGBSmemBase = kGBStages * kGBSlot + kGBStages * 16 + kGBStages * kGBItems * (int)sizeof(GBItem);
__host__ __device__ inline int gb_smem_bytes(int count) { return kGBSmemBase + 8 * count; }
static_assert(kGBSmemBase + 8 * kGBMaxRecs <= 232448, "dynamic shared memory per CTA");
static_assert(kGBItems <= 32 && kGBItemBytes >= (int)kGatherSeg * 4, "one segment per producer lane and slot");

__global__ void __launch_bounds__(kGBThreads, 1) k_gather_bulk(const GatherRec* __restrict__ recs, int count,
                                                                long long total_items, uint32_t* status) {
  extern __shared__ __align__(128) uint8_t gb_smem[];
  uint64_t* full = (uint64_t*)(gb_smem + kGBStages * kGBSlot);
  uint64_t* empty = full + kGBStages;
  GBItem* items = (GBItem*)(empty + kGBStages);                     // [kGBStages][kGBItems]
  long long* starts = (long long*)(items + kGBStages * kGBItems);   // [count]: each record's first item
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int q = 0; q < kGBStages; ++q) {
      mbar_init(&full[q], 1);
      mbar_init(&empty[q], kGBConsumerWarps);
    }
    fence_mbar_init();
  }
  for (int i = threadIdx.x; i < count; i += blockDim.x) starts[i] = recs[i].chunk_start;
  __syncthreads();
  volatile uint32_t* st = status;
  const long long step = (long long)gridDim.x * kGBItems;
  if (warp == kGBConsumerWarps) {
    // ------------------------------------------------------------ producer
    int k = 0;
    for (long long base = (long long)blockIdx.x * kGBItems; base < total_items; base += step, ++k) {
      const int s = k % kGBStages;
      const uint32_t ph = (uint32_t)(k / kGBStages) & 1u;
      bool ok = true;
      if (lane == 0) ok = mbar_wait(&empty[s], ph ^ 1u, st, DEV_TIMEOUT_EMPTY);
      if (!__shfl_sync(0xffffffffu, ok, 0)) break;
      const long long item = base + lane;
      GBItem it{0, 0, 0, 0, nullptr, nullptr, 0, 0};
      uint32_t bytes = 0;
      const float* src = nullptr;
      if (lane < kGBItems && item < total_items) {
        int lo = 0, hi = count - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (starts[mid] <= item) lo = mid; else hi = mid - 1;
        }
        const GatherRec& R = recs[lo];
        const GatherSeg g = gather_segment(R, item - starts[lo]);
        it.so = g.so;
        it.dso = g.dso;
        it.c0 = g.c0;
        it.c1 = g.c1;
        it.len = g.len;
        it.src = R.src;
        it.dst = R.dst;
        it.bf16 = R.dst_bf16;
        bytes = (uint32_t)(it.c1 - it.c0) * 4u;
        src = R.src;
      }
      if (lane < kGBItems) items[s * kGBItems + lane] = it;
      const uint32_t total = __reduce_add_sync(0xffffffffu, bytes);
      __syncwarp();  // the item descriptors are written before lane 0's arrive publishes them
      if (lane == 0) {
        if (total) mbar_arrive_expect_tx(&full[s], total);
        else mbar_arrive(&full[s]);
      }
      __syncwarp();  // the expected bytes are registered before any copy is issued
      if (bytes) bulk_load(gb_smem + s * kGBSlot + lane * kGBItemBytes, src + it.c0, bytes, &full[s]);
    }
    // copies issued but never consumed (only after an error) land before exit
    if (lane == 0 && *st != DEV_OK) {
      const long long t0 = clock64();
      while (clock64() - t0 < 200000) {}
    }
    return;
  }
  // -------------------------------------------------------------- consumers
  int k = 0;
  for (long long base = (long long)blockIdx.x * kGBItems; base < total_items; base += step, ++k) {
    const int s = k % kGBStages;
    const uint32_t ph = (uint32_t)(k / kGBStages) & 1u;
    if (!__all_sync(0xffffffffu, mbar_wait(&full[s], ph, st, DEV_TIMEOUT_FULL))) break;
    for (int u = warp; u < kGBItems; u += kGBConsumerWarps) {
      const GBItem it = items[s * kGBItems + u];
      if (it.len == 0) continue;
      const float* __restrict__ src = it.src;
      const bool bf16 = it.bf16 != 0;
      const float* sp = (const float*)(gb_smem + s * kGBSlot + u * kGBItemBytes);
      const int nw = (int)(it.c1 - it.c0);  // staged elements
      if (it.c0 == it.so) {
        // the row is 16-byte aligned: staged element j is output element j
        for (int q = lane; q < nw / 4; q += 32) {
          const float4 v = *(const float4*)(sp + 4 * q);
          const long long o = it.dso + 4 * q;
          if (bf16) {
            const __nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), b = __floats2bfloat162_rn(v.z, v.w);
            *(uint2*)((__nv_bfloat16*)it.dst + o) = make_uint2(*(const uint32_t*)&a, *(const uint32_t*)&b);
          } else {
            *(float4*)((float*)it.dst + o) = v;
          }
        }
        for (int y = nw + lane; y < it.len; y += 32) {  // the tail after the last whole block
          const float v = __ldg(src + it.so + y);
          if (bf16) ((__nv_bfloat16*)it.dst)[it.dso + y] = __float2bfloat16_rn(v);
          else ((float*)it.dst)[it.dso + y] = v;
        }
      } else {
        for (int y = lane; y < it.len; y += 32) {
          const long long x = it.so + y;
          const float v = (x >= it.c0 && x < it.c1) ? sp[x - it.c0] : __ldg(src + x);
          if (bf16) ((__nv_bfloat16*)it.dst)[it.dso + y] = __float2bfloat16_rn(v);
          else ((float*)it.dst)[it.dso + y] = v;
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
}

static int launch_gather(const float* in, void* out, bool bf16, const GatherArgs& args, long long n,
                         cudaStream_t st) {
  if (n == 0) return BBX_OK;
  GatherArgs a = args;
  simplify_gather(&a);
  if (row_mode_ok(a)) {
    GatherRec r{};  // travels by value in the kernel parameters
    r.a = a;
    r.src = in;
    r.dst = out;
    r.dst_bf16 = bf16 ? 1 : 0;
    r.n = n;
    set_row_mode(&r);
    const long long chunks = (row_items(r) + r.items_per_chunk - 1) / r.items_per_chunk;
    k_gather_rows1<<<(int)std::min<long long>(chunks, 148 * 8), 256, 0, st>>>(r, chunks);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(BBX_ERR_CUDA, "k_gather_rows1: %s", cudaGetErrorString(e));
    return BBX_OK;
  }
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_gather_sum<<<(int)blocks, 256, 0, st>>>(in, out, bf16 ? 1 : 0, a, n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(BBX_ERR_CUDA, "k_gather_sum: %s", cudaGetErrorString(e));
  return BBX_OK;
}

enum { CI = 0, CN = 1, CB = 2, CK = 3, CL = 4, CR = 5 };

int lower_contraction(int rank_l, const long long* dims_l, const int* modes_l, int rank_r,
                      const long long* dims_r, const int* modes_r, int rank_o, const int* modes_o,
                      bool bf16, ContractionLowering* L) {
  if (rank_l < 0 || rank_l > 4 || rank_r < 0 || rank_r > 4 || rank_o < 0 || rank_o > 4)
    return set_error(BBX_ERR_INVALID, "ranks must be in [0,4] (MAXRANK of the cutensor format)");
  constexpr int MAXM = 16;
  long long ext[MAXM];
  bool inl[MAXM] = {}, inr[MAXM] = {}, ino[MAXM] = {};
  for (int i = 0; i < MAXM; ++i) ext[i] = -1;
  long long strl[MAXM] = {}, strr[MAXM] = {};
  long long s = 1;
  for (int d = 0; d < rank_l; ++d) {
    int m = modes_l[d];
    if (m < 0 || m >= MAXM || inl[m]) return set_error(BBX_ERR_INVALID, "bad lhs mode %d", m);
    inl[m] = true; ext[m] = dims_l[d]; strl[m] = s; s *= dims_l[d];
  }
  s = 1;
  for (int d = 0; d < rank_r; ++d) {
    int m = modes_r[d];
    if (m < 0 || m >= MAXM || inr[m]) return set_error(BBX_ERR_INVALID, "bad rhs mode %d", m);
    if (ext[m] >= 0 && ext[m] != dims_r[d])
      return set_error(BBX_ERR_INVALID, "mode %d has extent %lld in lhs and %lld in rhs", m, ext[m], dims_r[d]);
    inr[m] = true; ext[m] = dims_r[d]; strr[m] = s; s *= dims_r[d];
  }
  for (int d = 0; d < rank_o; ++d) {
    int m = modes_o[d];
    if (m < 0 || m >= MAXM || ino[m]) return set_error(BBX_ERR_INVALID, "bad out mode %d", m);
    if (!inl[m] && !inr[m]) return set_error(BBX_ERR_INVALID, "output mode %d is not an input mode", m);
    ino[m] = true;
  }
  auto cls = [&](int m) {
    if (inl[m] && inr[m]) return ino[m] ? (int)CB : (int)CK;
    if (inl[m]) return ino[m] ? (int)CI : (int)CL;
    return ino[m] ? (int)CN : (int)CR;
  };
  std::vector<int> gI, gN, gB, gK, gL, gR;
  for (int d = 0; d < rank_o; ++d) {
    int c = cls(modes_o[d]);
    (c == CI ? gI : c == CN ? gN : gB).push_back(modes_o[d]);
  }
  for (int d = 0; d < rank_l; ++d) {
    int c = cls(modes_l[d]);
    if (c == CK) gK.push_back(modes_l[d]);
    if (c == CL) gL.push_back(modes_l[d]);
  }
  for (int d = 0; d < rank_r; ++d)
    if (cls(modes_r[d]) == CR) gR.push_back(modes_r[d]);
  auto prod = [&](const std::vector<int>& g) { long long p = 1; for (int m : g) p *= ext[m]; return p; };
  memset(L, 0, sizeof(*L));
  L->nb = prod(gB);
  L->nm = prod(gI);
  L->nn = prod(gN);
  const long long nk = prod(gK);
  L->empty = L->nb == 0 || L->nm == 0 || L->nn == 0;
  if (L->empty) return BBX_OK;
  if (L->nm > (1ll << 31) - 1 || L->nn > (1ll << 31) - 1 || nk > (1ll << 31) - 1)
    return set_error(BBX_ERR_INVALID, "contraction group too large");
  L->kdim = nk > 0 ? nk : 1;  // no contracted mode: an outer product, k = 1
  L->pk = bf16 ? ((L->kdim + 7) / 8) * 8 : L->kdim;
  L->pm = bf16 ? ((L->nm + 7) / 8) * 8 : L->nm;
  L->pn = bf16 ? ((L->nn + 7) / 8) * 8 : L->nn;
  // staging major-ness (tensor-core lowering only): MN-major when the source's
  // fastest mode is one of the operand's M (lhs) / N (rhs) modes
  L->lc_mn = bf16 && rank_l > 0 && cls(modes_l[0]) == CI;
  L->rc_mn = bf16 && rank_r > 0 && cls(modes_r[0]) == CN;
  L->lc_elems = L->nb * (L->lc_mn ? L->kdim * L->pm : L->nm * L->pk);
  L->rc_elems = L->nb * (L->rc_mn ? L->kdim * L->pn : L->nn * L->pk);

  // Column-major group flattening: stride of each mode inside its group.
  auto group_strides = [&](const std::vector<int>& g, long long base, long long* st_of) {
    long long p = base;
    for (int m : g) { st_of[m] = p; p *= ext[m]; }
  };
  // Gather arguments: output modes listed outermost first (B, then M or N, then K).
  auto make_gather = [&](const std::vector<int>& outer, const std::vector<int>& mid,
                         const std::vector<int>& inner, const std::vector<int>& summed,
                         const long long* src_stride, long long mid_n, long long pitch, GatherArgs* a) {
    long long dst_of[MAXM] = {};
    group_strides(inner, 1, dst_of);
    group_strides(mid, pitch, dst_of);
    group_strides(outer, pitch * mid_n, dst_of);
    std::vector<int> order;  // outermost first; inside a group the last mode is outermost
    for (int i = (int)outer.size() - 1; i >= 0; --i) order.push_back(outer[i]);
    for (int i = (int)mid.size() - 1; i >= 0; --i) order.push_back(mid[i]);
    for (int i = (int)inner.size() - 1; i >= 0; --i) order.push_back(inner[i]);
    memset(a, 0, sizeof(*a));
    a->rank_o = (int)order.size();
    for (int d = 0; d < a->rank_o; ++d) {
      a->odims[d] = ext[order[d]];
      a->istride[d] = src_stride[order[d]];
      a->ostride[d] = dst_of[order[d]];
    }
    a->rank_s = (int)summed.size();
    for (int d = 0; d < a->rank_s; ++d) {
      a->sdims[d] = ext[summed[d]];
      a->sstride[d] = src_stride[summed[d]];
    }
    if (a->rank_o == 0) { a->rank_o = 1; a->odims[0] = 1; }  // empty groups behave as extent 1
  };
  // K-major: [b][m][k] = outer B, mid M (pitch pk), inner K; MN-major:
  // [b][k][m] = outer B, mid K (pitch pm), inner M
  if (L->lc_mn) make_gather(gB, gK, gI, gL, strl, L->kdim, L->pm, &L->ga);
  else make_gather(gB, gI, gK, gL, strl, L->nm, L->pk, &L->ga);
  if (L->rc_mn) make_gather(gB, gK, gN, gR, strr, L->kdim, L->pn, &L->gb);
  else make_gather(gB, gN, gK, gR, strr, L->nn, L->pk, &L->gb);
  L->nl = L->nb * L->nm * L->kdim;
  L->nr = L->nb * L->nn * L->kdim;

  // Direct write when the output order is I..., N..., B...
  L->direct = true;
  int last = -1;
  for (int d = 0; d < rank_o; ++d) {
    int c = cls(modes_o[d]);
    int rank_c = c == CI ? 0 : c == CN ? 1 : 2;
    if (rank_c < last) L->direct = false;
    last = rank_c;
  }
  // Ct[b][n][m] -> column-major output in modes_o order
  long long src_of[MAXM] = {};
  group_strides(gI, 1, src_of);
  group_strides(gN, L->nm, src_of);
  group_strides(gB, L->nm * L->nn, src_of);
  long long p = 1, ostr[MAXM] = {};
  for (int d = 0; d < rank_o; ++d) { ostr[modes_o[d]] = p; p *= ext[modes_o[d]]; }
  L->go.rank_o = rank_o;
  for (int d = 0; d < rank_o; ++d) {
    int m = modes_o[rank_o - 1 - d];
    L->go.odims[d] = ext[m];
    L->go.istride[d] = src_of[m];
    L->go.ostride[d] = ostr[m];
  }
  if (L->go.rank_o == 0) { L->go.rank_o = 1; L->go.odims[0] = 1; }
  L->no = p;
  return BBX_OK;
}

ContractionGemm contraction_gemm(const ContractionLowering& L, const void* lc, const void* rc, void* ct, long long b) {
  ContractionGemm g{};
  const char* lb = (const char*)lc + 2 * b * (L.lc_mn ? L.kdim * L.pm : L.nm * L.pk);  // this batch's Lc
  const char* rb = (const char*)rc + 2 * b * (L.rc_mn ? L.kdim * L.pn : L.nn * L.pk);  // this batch's Rc
  g.c = (char*)ct + 4 * b * L.nn * L.nm;
  g.k = (int)L.kdim;
  g.ldc = L.nm;
  if (L.nm > L.nn) {
    // A = Lc (m = nm), B = Rc (n = nn), C column-major
    g.a = lb;
    g.trans_a = L.lc_mn ? 1 : 0;  // Lc[k][m]: MN-major; Lc[m][k]: K-major
    g.lda = L.lc_mn ? L.pm : L.pk;
    g.b = rb;
    g.trans_b = L.rc_mn ? 0 : 1;  // Rc[k][n]: op(B) stored as is; Rc[n][k]: transposed
    g.ldb = L.rc_mn ? L.pn : L.pk;
    g.m = (int)L.nm;
    g.n = (int)L.nn;
    g.flags = BBX_EPI_C_COLMAJOR;
    return g;
  }
  // A = Rc (m = nn), B = Lc (n = nm), C row-major
  g.a = rb;
  g.trans_a = L.rc_mn ? 1 : 0;  // Rc[k][n]: A stored k x n, MN-major; Rc[n][k]: K-major
  g.lda = L.rc_mn ? L.pn : L.pk;
  g.b = lb;
  g.trans_b = L.lc_mn ? 0 : 1;  // Lc[k][m]: op(B) = k x m stored as is; Lc[m][k]: transposed
  g.ldb = L.lc_mn ? L.pm : L.pk;
  g.m = (int)L.nn;
  g.n = (int)L.nm;
  g.flags = 0;
  return g;
}

struct GatherPlan {
  GatherRec* d = nullptr;
  int count = 0;
  long long total = 0;
  bool bulk = false;  // k_gather_bulk: `total` counts row segments, chunk_start each record's first
};

// Every record on the row path with a 16-byte aligned source and 16-byte
// aligned destination rows (base and every row stride).
static bool bulk_ok(const GatherRec& r) {
  if (!r.row_mode || (((uintptr_t)r.src) & 15) || (((uintptr_t)r.dst) & 15)) return false;
  const long long esz = r.dst_bf16 ? 2 : 4;
  for (int d = 0; d + 1 < r.a.rank_o; ++d)
    if ((r.a.ostride[d] * esz) & 15) return false;
  return true;
}

int gather_bulk_init() {
  cudaError_t e = cudaFuncSetAttribute(k_gather_bulk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       gb_smem_bytes(kGBMaxRecs));
  return e == cudaSuccess ? BBX_OK : set_error(BBX_ERR_CUDA, "k_gather_bulk attribute: %s", cudaGetErrorString(e));
}

int gather_plan_create(const GatherRec* recs, int count, GatherPlan** out, bool allow_bulk) {
  if (!recs || count <= 0 || !out) return set_error(BBX_ERR_INVALID, "bad gather plan");
  std::vector<GatherRec> h(recs, recs + count);
  bool bulk = allow_bulk && count <= kGBMaxRecs;
  for (auto& r : h) {
    simplify_gather(&r.a);
    set_row_mode(&r);
    bulk = bulk && bulk_ok(r);
  }
  long long chunks = 0;
  for (auto& r : h) {
    r.chunk_start = chunks;
    if (bulk) chunks += row_items(r);
    else if (r.row_mode) chunks += (row_items(r) + r.items_per_chunk - 1) / r.items_per_chunk;
    else chunks += (r.n + kGatherChunk - 1) / kGatherChunk;
  }
  auto* p = new GatherPlan();
  p->count = count;
  p->total = chunks;
  p->bulk = bulk;
  cudaError_t e = cudaMalloc(&p->d, sizeof(GatherRec) * count);
  if (e == cudaSuccess) e = cudaMemcpy(p->d, h.data(), sizeof(GatherRec) * count, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    if (p->d) cudaFree(p->d);
    delete p;
    return set_error(BBX_ERR_CUDA, "gather plan upload: %s", cudaGetErrorString(e));
  }
  *out = p;
  return BBX_OK;
}

int gather_plan_launch(GatherPlan* p, void* stream) {
  if (!p || p->total == 0) return BBX_OK;
  if (p->bulk) {
    uint32_t* status = nullptr;
    int sms = 148;
    int rc = device_status_and_sms(&status, &sms);
    if (rc) return rc;
    const long long grid = std::min<long long>((p->total + kGBItems - 1) / kGBItems, sms);
    k_gather_bulk<<<(int)grid, kGBThreads, gb_smem_bytes(p->count), (cudaStream_t)stream>>>(p->d, p->count,
                                                                                          p->total, status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(BBX_ERR_CUDA, "k_gather_bulk: %s", cudaGetErrorString(e));
    return BBX_OK;
  }
  long long grid = std::min<long long>(p->total, 148 * 8);
  k_gather_group<<<(int)grid, 256, 0, (cudaStream_t)stream>>>(p->d, p->count, p->total);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(BBX_ERR_CUDA, "k_gather_group: %s", cudaGetErrorString(e));
  return BBX_OK;
}

void gather_plan_destroy(GatherPlan* p) {
  if (!p) return;
  if (p->d) cudaFree(p->d);
  delete p;
}

}  // namespace bbx

using namespace bbx;

extern "C" int bbx_contraction(const float* lhs, int rank_l, const long long* dims_l,
                               const int* modes_l, const float* rhs, int rank_r,
                               const long long* dims_r, const int* modes_r, float* out, int rank_o,
                               const int* modes_o, float alpha, int precision, void* stream) {
  if (!lhs || !rhs || !out) return set_error(BBX_ERR_INVALID, "null tensor");
  if (precision != BBX_F32 && precision != BBX_BF16)
    return set_error(BBX_ERR_UNSUPPORTED, "contraction precision %d", precision);
  const bool bf16 = precision == BBX_BF16;
  ContractionLowering L;
  int rc = lower_contraction(rank_l, dims_l, modes_l, rank_r, dims_r, modes_r, rank_o, modes_o, bf16, &L);
  if (rc) return rc;
  if (L.empty) return BBX_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const int esz = bf16 ? 2 : 4;
  void *Lc = nullptr, *Rc = nullptr;
  float* Ct = nullptr;
  cudaError_t e;
  e = cudaMallocAsync(&Lc, (size_t)(L.lc_elems * esz + 16), st);
  if (e != cudaSuccess) return set_error(BBX_ERR_CUDA, "cudaMallocAsync: %s", cudaGetErrorString(e));
  e = cudaMallocAsync(&Rc, (size_t)(L.rc_elems * esz + 16), st);
  if (e != cudaSuccess) { cudaFreeAsync(Lc, st); return set_error(BBX_ERR_CUDA, "cudaMallocAsync: %s", cudaGetErrorString(e)); }
  if (!L.direct) {
    e = cudaMallocAsync((void**)&Ct, (size_t)(L.nb * L.nn * L.nm * 4), st);
    if (e != cudaSuccess) { cudaFreeAsync(Lc, st); cudaFreeAsync(Rc, st); return set_error(BBX_ERR_CUDA, "cudaMallocAsync: %s", cudaGetErrorString(e)); }
  }
  float* C = L.direct ? out : Ct;
  rc = launch_gather(lhs, Lc, bf16, L.ga, L.nl, st);
  if (!rc) rc = launch_gather(rhs, Rc, bf16, L.gb, L.nr, st);
  if (!rc) {
    const long long pitch = L.pk;
    if (!bf16) {
      rc = bbx_matmul_f32((const float*)Rc, (const float*)Lc, C, (int)L.nn, (int)L.nm, (int)L.kdim, pitch,
                          pitch, L.nm, 0, 1, alpha, 0.f, nullptr, 0, (int)L.nb, L.nn * pitch, L.nm * pitch,
                          L.nn * L.nm, stream);
    } else {
      std::vector<bbx_tc_problem_t> probs((size_t)L.nb);
      for (long long b = 0; b < L.nb; ++b) {
        bbx_tc_problem_t& q = probs[(size_t)b];
        memset(&q, 0, sizeof(q));
        const ContractionGemm g = contraction_gemm(L, Lc, Rc, C, b);
        q.a = g.a; q.b = g.b; q.c = g.c;
        q.m = g.m; q.n = g.n; q.k = g.k;
        q.trans_a = g.trans_a; q.trans_b = g.trans_b;
        q.lda = g.lda; q.ldb = g.ldb; q.ldc = g.ldc;
        q.flags = g.flags;
        q.alpha = alpha; q.beta = 0.f;
      }
      rc = bbx_matmul_tc(BBX_BF16, probs.data(), (int)L.nb, 0, stream);
    }
  }
  if (!rc && !L.direct) rc = launch_gather(Ct, out, false, L.go, L.no, st);
  cudaFreeAsync(Lc, st);
  cudaFreeAsync(Rc, st);
  if (Ct) cudaFreeAsync(Ct, st);
  return rc;
}
