// The remaining block ops of the reference's "cutensor" plugin, on
// column-major FP32 tensors of rank <= 4 (libraries/cutensor/cu.h:60-169):
//   reduction     out = alpha * fold_{add|max|min|mul} over the dropped modes
//                 (libraries/cutensor/reduction.h:13-21 params, :42-111 semantics)
//   ew            out = permute(alpha * uop(in))        (ew.h:13-21, :131-190)
//   ewb           out = op(alpha * lhs, beta * rhs) with broadcast (ewb.h:13-46, :122-204)
//   ewb_castable  out = op(lhs, rhs), same shape         (ewb_castable.h:24-91)
//   expand        out = zeros, then a box copied in      (expand.h:1-110)
// Two HBM-streaming kernels cover them: a strided map over the output
// (unary / binary with per-input strides, 0 for broadcast) and a strided fold.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include "bbts_b200.h"
#include "common.h"

namespace bbx {

struct CuMapArgs {
  int rank;                 // output modes, column-major (mode 0 fastest)
  long long odims[4];
  long long sa[4], sb[4];   // strides of a / b per output mode (0 = broadcast)
  long long oa, ob, oo;     // base offsets
  long long ostride[4];     // output strides per mode
  int kind;                 // 0 unary(a), 1 binary(a, b)
  int op;
  float p, alpha, beta;
};

__device__ __forceinline__ float cu_unary(int op, float v, float p) {
  switch (op) {
    case 0: { float e = expf(v); return e / (1.f + e); }  // sigmoid as e^v / (1 + e^v)
    case 1: return expf(v);
    case 2: return v * v;
    case 3: return v > 0.f ? v : 0.f;                     // fmax(v, 0)
    case 4: return v < 0.f ? 0.f : 1.f;                   // relu' of the plugin: 1 at 0
    case 5: return sqrtf(v);
    case 6: return v + p;
  }
  return v;
}

__device__ __forceinline__ float cu_binary(int op, float l, float r) {
  switch (op) {
    case 0: return l + r;
    case 1: return l > r ? l : r;
    case 2: return l > r ? r : l;
    case 3: return l * r;
    case 4: return l - r;
    case 5: return l / r;
  }
  return l;
}

__global__ void k_cu_map(const float* __restrict__ a, const float* __restrict__ b, float* out,
                         const __grid_constant__ CuMapArgs g, long long n) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    long long rem = e, ia = g.oa, ib = g.ob, io = g.oo;
    for (int d = 0; d < g.rank; ++d) {
      long long idx = rem % g.odims[d];
      rem /= g.odims[d];
      ia += idx * g.sa[d];
      ib += idx * g.sb[d];
      io += idx * g.ostride[d];
    }
    float v;
    // scalings are rounded on their own (no FMA contraction), as the plugin's
    // CPU path scales each operand before the binary op (ewb.h:166-184)
    if (g.kind == 0) v = __fmul_rn(g.alpha, cu_unary(g.op, a[ia], g.p));
    else v = cu_binary(g.op, __fmul_rn(g.alpha, a[ia]), __fmul_rn(g.beta, b[ib]));
    out[io] = v;
  }
}

// The reduction's castable scalar ops (libraries/cutensor/utils.h:32-35); min
// is `l < r ? l : r`, which differs from ewb's min on signed zeros and NaN.
__device__ __forceinline__ float cu_fold_op(int op, float l, float r) {
  switch (op) {
    case 0: return l + r;
    case 1: return l > r ? l : r;
    case 2: return l < r ? l : r;
    default: return l * r;
  }
}

struct CuFoldArgs {
  int rank_o;
  long long odims[4], ostride_in[4];  // kept modes: output extent and input stride
  int rank_a;
  long long adims[4], astride[4];     // dropped modes folded, in input order (first fastest)
  int op;
  float alpha;
};

__global__ void k_cu_fold(const float* __restrict__ in, float* out, const __grid_constant__ CuFoldArgs g,
                          long long n) {
  long long na = 1;
  for (int d = 0; d < g.rank_a; ++d) na *= g.adims[d];
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    long long rem = e, base = 0;
    for (int d = 0; d < g.rank_o; ++d) {
      long long idx = rem % g.odims[d];
      rem /= g.odims[d];
      base += idx * g.ostride_in[d];
    }
    float acc = 0.f;
    for (long long s = 0; s < na; ++s) {
      long long r = s, off = 0;
      for (int d = 0; d < g.rank_a; ++d) {
        off += (r % g.adims[d]) * g.astride[d];
        r /= g.adims[d];
      }
      float v = in[base + off];
      acc = s == 0 ? v : cu_fold_op(g.op, acc, v);
    }
    out[e] = g.alpha * acc;
  }
}

static int grid_of(long long n) {
  long long b = (n + 255) / 256;
  return (int)std::max<long long>(1, std::min<long long>(b, 148 * 16));
}

static void colmajor_strides(int rank, const long long* dims, long long* st) {
  long long s = 1;
  for (int d = 0; d < rank; ++d) { st[d] = s; s *= dims[d]; }
}

}  // namespace bbx

using namespace bbx;

extern "C" {

int bbx_cu_reduction(const float* in, int rank, const long long* dims, int op, float alpha, const int* ordering,
                     int rank_out, float* out, void* stream) {
  if (!in || !out || rank < 0 || rank > 4 || rank_out < 0 || rank_out > rank)
    return set_error(BBX_ERR_INVALID, "bad reduction arguments");
  if (op < 0 || op > 3) return set_error(BBX_ERR_INVALID, "reduction op must be 0 add, 1 max, 2 min, 3 mul");
  long long st[4] = {0, 0, 0, 0};
  colmajor_strides(rank, dims, st);
  CuFoldArgs g;
  memset(&g, 0, sizeof(g));
  bool kept[4] = {false, false, false, false};
  long long n = 1;
  for (int r = 0; r < rank_out; ++r) {
    int m = ordering[r];
    if (m < 0 || m >= rank || kept[m]) return set_error(BBX_ERR_INVALID, "bad reduction ordering");
    kept[m] = true;
    g.odims[r] = dims[m];
    g.ostride_in[r] = st[m];
    n *= dims[m];
  }
  g.rank_o = rank_out;
  for (int d = 0; d < rank; ++d)
    if (!kept[d]) {
      g.adims[g.rank_a] = dims[d];
      g.astride[g.rank_a] = st[d];
      ++g.rank_a;
    }
  g.op = op;
  g.alpha = alpha;
  if (n == 0) return BBX_OK;
  k_cu_fold<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(in, out, g, n);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? BBX_OK : set_error(BBX_ERR_CUDA, "k_cu_fold: %s", cudaGetErrorString(e));
}

int bbx_cu_ew(const float* in, int rank, const long long* dims, int uop, float scalar, float alpha,
              const int* ordering, float* out, void* stream) {
  if (!in || !out || rank < 0 || rank > 4) return set_error(BBX_ERR_INVALID, "bad ew arguments");
  if (uop < 0 || uop > 6) return set_error(BBX_ERR_INVALID, "is not a valid unary op");
  long long st[4] = {0, 0, 0, 0};
  colmajor_strides(rank, dims, st);
  CuMapArgs g;
  memset(&g, 0, sizeof(g));
  g.rank = rank;
  long long n = 1;
  unsigned seen = 0;
  // output mode r is input mode ordering[r]
  for (int r = 0; r < rank; ++r) {
    int m = ordering[r];
    if (m < 0 || m >= rank || (seen & (1u << m))) return set_error(BBX_ERR_INVALID, "ew ordering is not a permutation");
    seen |= 1u << m;
    g.odims[r] = dims[m];
    g.sa[r] = st[m];
  }
  long long os = 1;
  for (int r = 0; r < rank; ++r) { g.ostride[r] = os; os *= g.odims[r]; n *= g.odims[r]; }
  g.kind = 0;
  g.op = uop;
  g.p = scalar;
  g.alpha = alpha;
  if (rank == 0) { g.rank = 0; n = 1; }
  k_cu_map<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(in, nullptr, out, g, n);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? BBX_OK : set_error(BBX_ERR_CUDA, "k_cu_map: %s", cudaGetErrorString(e));
}

int bbx_cu_ewb(const float* lhs, int rank_l, const long long* dims_l, const int* ord_l, const float* rhs,
               int rank_r, const long long* dims_r, const int* ord_r, int op, float alpha, float beta, float* out,
               int* rank_out, long long* dims_out, void* stream) {
  if (!lhs || !rhs || !out || rank_l < 0 || rank_l > 4 || rank_r < 0 || rank_r > 4)
    return set_error(BBX_ERR_INVALID, "bad ewb arguments");
  if (op < 0 || op > 5) return set_error(BBX_ERR_INVALID, "ewb op must be 0..5");
  int ro = 0;
  for (int r = 0; r < rank_l; ++r) ro = std::max(ro, ord_l[r] + 1);
  for (int r = 0; r < rank_r; ++r) ro = std::max(ro, ord_r[r] + 1);
  if (ro > 4) return set_error(BBX_ERR_INVALID, "ewb output rank > 4");
  long long od[4] = {1, 1, 1, 1};
  bool set_by_l[4] = {false, false, false, false};
  long long sl[4] = {0, 0, 0, 0}, sr[4] = {0, 0, 0, 0};
  long long s = 1;
  for (int r = 0; r < rank_l; ++r) {
    if (ord_l[r] < 0 || set_by_l[ord_l[r]]) return set_error(BBX_ERR_INVALID, "bad ewb ordering");
    od[ord_l[r]] = dims_l[r];
    set_by_l[ord_l[r]] = true;
    sl[ord_l[r]] = s;
    s *= dims_l[r];
  }
  s = 1;
  bool set_by_r[4] = {false, false, false, false};
  for (int r = 0; r < rank_r; ++r) {
    if (ord_r[r] < 0 || set_by_r[ord_r[r]]) return set_error(BBX_ERR_INVALID, "bad ewb ordering");
    set_by_r[ord_r[r]] = true;
    if (set_by_l[ord_r[r]] && od[ord_r[r]] != dims_r[r])
      return set_error(BBX_ERR_INVALID, "ewb extents disagree on mode %d", ord_r[r]);
    od[ord_r[r]] = dims_r[r];
    sr[ord_r[r]] = s;
    s *= dims_r[r];
  }
  CuMapArgs g;
  memset(&g, 0, sizeof(g));
  g.rank = ro;
  long long n = 1, os = 1;
  for (int d = 0; d < ro; ++d) {
    g.odims[d] = od[d];
    g.sa[d] = sl[d];
    g.sb[d] = sr[d];
    g.ostride[d] = os;
    os *= od[d];
    n *= od[d];
  }
  g.kind = 1;
  g.op = op;
  g.alpha = alpha;
  g.beta = beta;
  if (rank_out) *rank_out = ro;
  if (dims_out)
    for (int d = 0; d < ro; ++d) dims_out[d] = od[d];
  k_cu_map<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(lhs, rhs, out, g, n);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? BBX_OK : set_error(BBX_ERR_CUDA, "k_cu_map: %s", cudaGetErrorString(e));
}

int bbx_cu_expand(const float* in, const int* params5, int rank, float* out, void* stream) {
  if (!in || !out || !params5 || rank < 0 || rank > 4) return set_error(BBX_ERR_INVALID, "bad expand arguments");
  long long nout = 1;
  CuMapArgs g;
  memset(&g, 0, sizeof(g));
  g.rank = rank;
  long long si = 1, so = 1;
  long long n = 1;
  for (int i = 0; i < rank; ++i) {
    const int sz_in = params5[5 * i], sz_out = params5[5 * i + 1], num = params5[5 * i + 2];
    const int start_in = params5[5 * i + 3], start_out = params5[5 * i + 4];
    if (sz_in < 0 || sz_out < 0 || num < 0 || start_in < 0 || start_out < 0 || start_in + num > sz_in ||
        start_out + num > sz_out)
      return set_error(BBX_ERR_INVALID, "expand box out of range on mode %d", i);
    g.odims[i] = num;
    g.sa[i] = si;
    g.ostride[i] = so;
    g.oa += (long long)start_in * si;
    g.oo += (long long)start_out * so;
    si *= sz_in;
    so *= sz_out;
    nout *= sz_out;
    n *= num;
  }
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float) * nout, st);
  if (e != cudaSuccess) return set_error(BBX_ERR_CUDA, "expand memset: %s", cudaGetErrorString(e));
  g.kind = 0;
  g.op = 7;  // identity: a plain copy keeps signed zeros and NaN payloads
  g.p = 0.f;
  g.alpha = 1.f;
  if (n == 0) return BBX_OK;
  k_cu_map<<<grid_of(n), 256, 0, st>>>(in, nullptr, out, g, n);
  e = cudaGetLastError();
  return e == cudaSuccess ? BBX_OK : set_error(BBX_ERR_CUDA, "k_cu_map: %s", cudaGetErrorString(e));
}

}  // extern "C"
