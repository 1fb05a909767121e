// Lowering of the cutensor plugin's einsum contraction (libraries/cutensor/
// contraction.h) into gathers + one batched matmul, shared by the per-call
// entry point (bbx_contraction) and the DAG executor (which groups the gathers
// and matmuls of a whole wave into single launches).
#pragma once
#include <cstdint>
#include "tile_order.h"  // BBX_HD

namespace bbx {

// out[dst(e)] = sum over the summed modes of in[src(e) + off(s)], for e over
// the output modes (outermost first, row-major flattening of e).
struct GatherArgs {
  int rank_o;
  long long odims[4], istride[4], ostride[4];
  int rank_s;
  long long sdims[4], sstride[4];
};

// Lc <- lhs and Rc <- rhs, then Ct[b][n][m] = alpha Rc Lc^T; if !direct,
// out <- Ct through `go`. Staging layouts (bf16 lowering): each operand is
// K-major (Lc[b][m][k], Rc[b][n][k], pitch pk) or MN-major (Lc[b][k][m] pitch
// pm, Rc[b][k][n] pitch pn), whichever keeps its source's fastest mode
// fastest, so the gather streams; the tensor cores read either layout. The
// FP32 lowering is always K-major.
struct ContractionLowering {
  bool empty;          // an output extent is 0: nothing to do
  bool direct;         // Ct is the output itself
  bool lc_mn, rc_mn;   // Lc / Rc staged MN-major
  long long nb, nm, nn, kdim, pk, pm, pn;
  long long lc_elems, rc_elems;  // staging sizes in elements, padding included
  long long nl, nr;    // elements gathered into Lc / Rc (unpadded)
  long long no;        // output elements (for the final gather)
  GatherArgs ga, gb, go;
};

// The batched GEMM of a bf16 lowering as tensor-core problem fields for batch
// b. C = Ct[b] holds the output n-major (f32, element (m, n) at m + n * nm).
// When nm > nn the GEMM is M = nm, N = nn with A = Lc, B = Rc and a
// column-major C (BBX_EPI_C_COLMAJOR), so the long dimension fills the
// 128-row tiles; otherwise M = nn, N = nm with A = Rc, B = Lc and C row-major
// with ldc = nm.
struct ContractionGemm {
  const void* a;
  const void* b;
  void* c;
  int m, n, k, trans_a, trans_b, flags;
  long long lda, ldb, ldc;
};
ContractionGemm contraction_gemm(const ContractionLowering& L, const void* lc, const void* rc, void* ct, long long b);

// Returns 0 or a BBX_ERR_* code (message via set_error).
int lower_contraction(int rank_l, const long long* dims_l, const int* modes_l, int rank_r,
                      const long long* dims_r, const int* modes_r, int rank_o, const int* modes_o,
                      bool bf16, ContractionLowering* out);

// One gather of a grouped gather launch.
struct GatherRec {
  GatherArgs a;
  const float* src;
  void* dst;
  int dst_bf16;
  int row_mode;            // set by gather_plan_create: innermost mode contiguous on both sides
  long long n;
  long long chunk_start;   // set by gather_plan_create
  long long row_len;       // row mode: elements per row (the innermost extent, after merging)
  long long segs;          // row mode: segments of kGatherSeg elements per row
  long long items_per_chunk;  // row mode: (row, segment) items per chunk
};

// Elements per work item of the row path: one segment of a row.
constexpr long long kGatherSeg = 1024;

// Row segment `local` (row-major over the record's rows, then segments) of a
// row-path record: the source and destination element of its first element,
// its length, and the whole 16-byte blocks [c0, c1) of its source range, in
// elements (the source base is 16-byte aligned; c1 == c0 when none fits).
struct GatherSeg {
  long long so, dso, c0, c1;
  int len;
};
BBX_HD GatherSeg gather_segment(const GatherRec& R, long long local) {
  const int outer = R.a.rank_o - 1;
  const long long row = local / R.segs, start = (local - row * R.segs) * kGatherSeg;
  long long rem = row, s = start, t = start;
  for (int d = outer - 1; d >= 0; --d) {
    const long long idx = rem % R.a.odims[d];
    rem /= R.a.odims[d];
    s += idx * R.a.istride[d];
    t += idx * R.a.ostride[d];
  }
  GatherSeg g;
  g.so = s;
  g.dso = t;
  g.len = (int)(R.row_len - start < kGatherSeg ? R.row_len - start : kGatherSeg);
  g.c0 = (s + 3) & ~3LL;
  g.c1 = (s + g.len) & ~3LL;
  if (g.c1 < g.c0) g.c1 = g.c0;
  return g;
}

// Merges adjacent output modes that are contiguous in both the source and the
// destination (a padded or permuted copy then runs as long rows).
void simplify_gather(GatherArgs* a);

struct GatherPlan;
// allow_bulk: use the bulk-staged kernel when every record qualifies. It holds
// about 200 KB of shared memory per SM, so it cannot run beside a tensor-core
// launch; the row kernel, which needs none, can.
int gather_plan_create(const GatherRec* recs, int count, GatherPlan** out, bool allow_bulk = true);
int gather_plan_launch(GatherPlan* p, void* stream);
void gather_plan_destroy(GatherPlan* p);
// Opts the bulk gather kernel into its shared memory (once per device, outside any capture).
int gather_bulk_init();
// The device's status word (bounded waits report into it) and SM count (abi_kernels.cu).
int device_status_and_sms(uint32_t** status, int* sms);

}  // namespace bbx
