// Lowering of the cutensor plugin's einsum contraction (libraries/cutensor/
// contraction.h) into gathers + one batched matmul, shared by the per-call
// entry point (bbx_contraction) and the DAG executor (which groups the gathers
// and matmuls of a whole wave into single launches).
#pragma once
#include <cstdint>

namespace bbx {

// out[dst(e)] = sum over the summed modes of in[src(e) + off(s)], for e over
// the output modes (outermost first, row-major flattening of e).
struct GatherArgs {
  int rank_o;
  long long odims[4], istride[4], ostride[4];
  int rank_s;
  long long sdims[4], sstride[4];
};

// Lc[b][m][k] (pitch pk) <- lhs, Rc[b][n][k] <- rhs; Ct[b][n][m] = alpha Rc Lc^T;
// if !direct, out <- Ct through `go`.
struct ContractionLowering {
  bool empty;          // an output extent is 0: nothing to do
  bool direct;         // Ct is the output itself
  long long nb, nm, nn, kdim, pk;
  long long nl, nr;    // elements gathered into Lc / Rc (unpadded)
  long long no;        // output elements (for the final gather)
  GatherArgs ga, gb, go;
};

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
  int pad_;
  long long n;
  long long chunk_start;
};

struct GatherPlan;
int gather_plan_create(const GatherRec* recs, int count, GatherPlan** out);
int gather_plan_launch(GatherPlan* p, void* stream);
void gather_plan_destroy(GatherPlan* p);

}  // namespace bbx
