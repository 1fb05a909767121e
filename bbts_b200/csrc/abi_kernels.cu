// C-ABI entry points for the block kernels (declared in include/bbts_b200.h).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include <algorithm>

#include "bbts_b200.h"
#include "common.h"
#include "contraction.h"
#include "gemm_f32.cuh"
#include "gemm_tc.cuh"
#include "stream_ops.cuh"

namespace bbx {

// ------------------------------------------------------------------ errors
static thread_local std::string t_last_error;

int set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_last_error = buf;
  return code;
}

const std::string& last_error() { return t_last_error; }

#define BBX_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return set_error(BBX_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                       __FILE__, __LINE__);                                             \
  } while (0)

#define BBX_CHECK_LAUNCH(name)                                                          \
  do {                                                                                  \
    cudaError_t e_ = cudaGetLastError();                                                \
    if (e_ != cudaSuccess)                                                              \
      return set_error(BBX_ERR_CUDA, "launch of %s failed: %s", name, cudaGetErrorString(e_)); \
  } while (0)

// ------------------------------------------------------------------ per-device state
struct DeviceState {
  bool ready = false;
  int sms = 148;
  uint32_t* status = nullptr;       // kernel status word
  uint32_t attr_done = 0;          // bitmask of tcgen05 kernels with smem attribute set
};
static std::mutex g_dev_mu;
static DeviceState g_dev[64];

template <int BN, bool AMN, bool BMN, bool FP8, bool EP8 = false>
static int set_tc_attr() {
  BBX_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<BN, AMN, BMN, FP8, EP8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                TcCfg<BN, AMN, BMN, FP8, EP8>::SMEM_BYTES));
  return BBX_OK;
}

template <bool EP8>
static int set_tc_attrs() {
  int rc = 0;
  rc |= set_tc_attr<256, false, false, false, EP8>(); rc |= set_tc_attr<256, false, true, false, EP8>();
  rc |= set_tc_attr<256, true, false, false, EP8>();  rc |= set_tc_attr<256, true, true, false, EP8>();
  rc |= set_tc_attr<128, false, false, false, EP8>(); rc |= set_tc_attr<128, false, true, false, EP8>();
  rc |= set_tc_attr<128, true, false, false, EP8>();  rc |= set_tc_attr<128, true, true, false, EP8>();
  rc |= set_tc_attr<256, false, false, true, EP8>();  rc |= set_tc_attr<256, false, true, true, EP8>();
  rc |= set_tc_attr<256, true, false, true, EP8>();   rc |= set_tc_attr<256, true, true, true, EP8>();
  rc |= set_tc_attr<128, false, false, true, EP8>();  rc |= set_tc_attr<128, false, true, true, EP8>();
  rc |= set_tc_attr<128, true, false, true, EP8>();   rc |= set_tc_attr<128, true, true, true, EP8>();
  return rc;
}

template <bool AMN, bool BMN, bool EP8>
static int set_tc2_attr() {
  BBX_CUDA(cudaFuncSetAttribute(tc_gemm2_kernel<AMN, BMN, EP8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                Tc2Cfg<AMN, BMN, EP8>::SMEM_BYTES));
  return BBX_OK;
}

template <bool EP8>
static int set_tc2_attrs() {
  int rc = 0;
  rc |= set_tc2_attr<false, false, EP8>(); rc |= set_tc2_attr<false, true, EP8>();
  rc |= set_tc2_attr<true, false, EP8>();  rc |= set_tc2_attr<true, true, EP8>();
  return rc;
}

static int launch_tc2(bool amn, bool bmn, bool ep8, const TcArgs& args, int grid, cudaStream_t st) {
  if (grid < 2) grid = 2;
#define TC2_CASE(A_, B_, E_)                                                                  \
  if (amn == A_ && bmn == B_ && ep8 == E_) {                                                  \
    tc_gemm2_kernel<A_, B_, E_><<<grid, Tc2Cfg<A_, B_, E_>::THREADS, Tc2Cfg<A_, B_, E_>::SMEM_BYTES, st>>>(args); \
    BBX_CHECK_LAUNCH("tc_gemm2_kernel");                                                      \
    return BBX_OK;                                                                            \
  }
  TC2_CASE(false, false, false) TC2_CASE(false, true, false) TC2_CASE(true, false, false) TC2_CASE(true, true, false)
  TC2_CASE(false, false, true) TC2_CASE(false, true, true) TC2_CASE(true, false, true) TC2_CASE(true, true, true)
#undef TC2_CASE
  return set_error(BBX_ERR_UNSUPPORTED, "no 2-SM variant");
}

static int init_tc_attributes() {
  int rc = 0;
  rc |= set_tc_attrs<false>();
  rc |= set_tc_attrs<true>();
  rc |= set_tc2_attrs<false>();
  rc |= set_tc2_attrs<true>();
  for (auto f : {(const void*)k_stream_bulk<false>, (const void*)k_stream_bulk<true>,
                 (const void*)k_stream_bulk_inline<false>, (const void*)k_stream_bulk_inline<true>})
    rc |= cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kBulkSmemMax) != cudaSuccess;
  rc |= gather_bulk_init() != BBX_OK;
  return rc ? BBX_ERR_CUDA : BBX_OK;
}

int device_state(DeviceState** out) {
  int dev = 0;
  BBX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(BBX_ERR_INVALID, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_dev_mu);
  DeviceState& d = g_dev[dev];
  if (!d.ready) {
    BBX_CUDA(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
    // a failed earlier set-up keeps its status buffer: allocate it only once
    if (!d.status) BBX_CUDA(cudaMalloc(&d.status, 256));
    BBX_CUDA(cudaMemset(d.status, 0, 256));
    // Dynamic shared-memory opt-in for every tcgen05 variant, once, here: never
    // inside a stream capture.
    int rc = init_tc_attributes();
    if (rc) return rc;
    d.attr_done = 0xFFFFFFFFu;
    d.ready = true;
  }
  *out = &d;
  return BBX_OK;
}

int device_status_and_sms(uint32_t** status, int* sms) {
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  *status = d->status;
  *sms = d->sms;
  return BBX_OK;
}

static inline int grid_for(long long work_items, int threads, int sms) {
  long long blocks = (work_items + threads - 1) / threads;
  long long cap = (long long)sms * 8;  // 8 resident blocks of 256 threads per SM
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

// ------------------------------------------------------------------ tensor maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int get_encode_fn(EncodeTiledFn* fn) {
  static EncodeTiledFn cached = nullptr;
  static std::once_flag once;
  static cudaError_t err = cudaSuccess;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    err = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
    if (err == cudaSuccess && q == cudaDriverEntryPointSuccess) cached = (EncodeTiledFn)p;
  });
  if (!cached)
    return set_error(BBX_ERR_CUDA, "cuTensorMapEncodeTiled unavailable (%s)", cudaGetErrorString(err));
  *fn = cached;
  return BBX_OK;
}

// 2-D map over a row-major matrix with `rows` rows of `cols` elements and pitch
// `ld` elements; box = box_cols x box_rows, 128-byte swizzle, zero OOB fill.
static int make_map(CUtensorMap* map, const void* base, int dtype, long long rows, long long cols,
                    long long ld, int box_cols, int box_rows, bool swizzle = true) {
  EncodeTiledFn enc;
  int rc = get_encode_fn(&enc);
  if (rc) return rc;
  const int esz = dtype == BBX_E4M3 ? 1 : dtype == BBX_F32 ? 4 : 2;
  CUtensorMapDataType dt = dtype == BBX_E4M3  ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                           : dtype == BBX_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                              : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(ld * esz)};
  cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(BBX_ERR_INVALID,
                     "cuTensorMapEncodeTiled failed (%d): rows=%lld cols=%lld ld=%lld box=%dx%d",
                     (int)r, rows, cols, ld, box_cols, box_rows);
  return BBX_OK;
}

// ------------------------------------------------------------------ tcgen05 dispatch
template <int BN, bool AMN, bool BMN, bool FP8, bool EP8>
static int launch_tc_variant(const TcArgs& args, int grid, cudaStream_t st, DeviceState* d,
                             int bit) {
  using C = TcCfg<BN, AMN, BMN, FP8, EP8>;
  auto kern = tc_gemm_kernel<BN, AMN, BMN, FP8, EP8>;
  if (!(d->attr_done & (1u << bit))) {
    BBX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM_BYTES));
    d->attr_done |= (1u << bit);
  }
  kern<<<grid, C::THREADS, C::SMEM_BYTES, st>>>(args);
  BBX_CHECK_LAUNCH("tc_gemm_kernel");
  return BBX_OK;
}

static int launch_tc(int bn, bool amn, bool bmn, bool fp8, bool ep8, const TcArgs& args, int grid,
                     cudaStream_t st, DeviceState* d) {
  const int bit = (ep8 ? 16 : 0) | (bn == 256 ? 8 : 0) | (amn ? 4 : 0) | (bmn ? 2 : 0) | (fp8 ? 1 : 0);
#define TC_CASE(BN_, A_, B_, F_)                                                                   \
  if (bn == BN_ && amn == A_ && bmn == B_ && fp8 == F_)                                            \
    return ep8 ? launch_tc_variant<BN_, A_, B_, F_, true>(args, grid, st, d, bit)                  \
               : launch_tc_variant<BN_, A_, B_, F_, false>(args, grid, st, d, bit);
  TC_CASE(256, false, false, false) TC_CASE(256, false, true, false)
  TC_CASE(256, true, false, false) TC_CASE(256, true, true, false)
  TC_CASE(128, false, false, false) TC_CASE(128, false, true, false)
  TC_CASE(128, true, false, false) TC_CASE(128, true, true, false)
  TC_CASE(256, false, false, true) TC_CASE(256, false, true, true)
  TC_CASE(256, true, false, true) TC_CASE(256, true, true, true)
  TC_CASE(128, false, false, true) TC_CASE(128, false, true, true)
  TC_CASE(128, true, false, true) TC_CASE(128, true, true, true)
#undef TC_CASE
  return set_error(BBX_ERR_UNSUPPORTED, "no tcgen05 variant for tile_n=%d", bn);
}

// Validates one public problem and fills the device record (minus tile_start).
// bn = 128 / 256: the 1-SM kernels (128 x bn tiles); bn = 512: the 2-SM pair
// kernel (256 x 256 tiles, each CTA loading 128-row halves of A and B).
static int build_problem(int in_dtype, const bbx_tc_problem_t& q, int bn_code, TcProblem* out) {
  const bool pair = bn_code == 512;
  const int bn = pair ? 128 : bn_code;  // rows of a K-major B box
  if (!q.a || !q.b || !q.c) return set_error(BBX_ERR_INVALID, "null operand pointer");
  if (q.m <= 0 || q.n <= 0 || q.k <= 0)
    return set_error(BBX_ERR_INVALID, "bad shape m=%d n=%d k=%d", q.m, q.n, q.k);
  const int esz = in_dtype == BBX_E4M3 ? 1 : 2;
  if ((((uintptr_t)q.a) | ((uintptr_t)q.b)) & 15)
    return set_error(BBX_ERR_INVALID, "tensor-core operands must be 16-byte aligned");
  if (((q.lda * esz) & 15) || ((q.ldb * esz) & 15))
    return set_error(BBX_ERR_INVALID, "operand pitches must be multiples of 16 bytes (lda=%lld ldb=%lld)",
                     q.lda, q.ldb);
  const bool amn = q.trans_a != 0, bmn = q.trans_b == 0;
  const int bk = 128 / esz, mnbox = 128 / esz;
  std::memset(out, 0, sizeof(TcProblem));
  int rc;
  // A: op(A) is m x k. Not transposed -> stored m x k (K-major); transposed -> k x m (MN-major).
  if (!amn) {
    if (q.lda < q.k) return set_error(BBX_ERR_INVALID, "lda < k");
    rc = make_map(&out->tmap_a, q.a, in_dtype, q.m, q.k, q.lda, bk, 128);
  } else {
    if (q.lda < q.m) return set_error(BBX_ERR_INVALID, "lda < m");
    rc = make_map(&out->tmap_a, q.a, in_dtype, q.k, q.m, q.lda, mnbox, bk);
  }
  if (rc) return rc;
  // B: op(B) is k x n. Not transposed -> stored k x n (MN-major); transposed -> n x k (K-major).
  if (!bmn) {
    if (q.ldb < q.k) return set_error(BBX_ERR_INVALID, "ldb < k");
    rc = make_map(&out->tmap_b, q.b, in_dtype, q.n, q.k, q.ldb, bk, bn);
  } else {
    if (q.ldb < q.n) return set_error(BBX_ERR_INVALID, "ldb < n");
    rc = make_map(&out->tmap_b, q.b, in_dtype, q.k, q.n, q.ldb, mnbox, bk);
  }
  if (rc) return rc;
  const bool c_col = (q.flags & BBX_EPI_C_COLMAJOR) != 0;
  if (q.ldc < (c_col ? q.m : q.n)) return set_error(BBX_ERR_INVALID, c_col ? "ldc < m" : "ldc < n");
  if ((q.flags & BBX_EPI_BIAS) && !q.bias) return set_error(BBX_ERR_INVALID, "bias flag without bias");
  out->c = q.c;
  out->bias = q.bias;
  out->ldc = q.ldc;
  out->m = q.m;
  out->n = q.n;
  out->k = q.k;
  out->tiles_m = pair ? (q.m + 255) / 256 : (q.m + 127) / 128;
  out->tiles_n = pair ? (q.n + 255) / 256 : (q.n + bn - 1) / bn;
  out->alpha = q.alpha;
  out->beta = q.beta;
  out->flags = q.flags & (EPI_RELU | EPI_OUT_BF16 | EPI_BIAS | EPI_BETA);
  const bool c_bf16 = (out->flags & EPI_OUT_BF16) != 0;
  const int c_esz = c_bf16 ? 2 : 4;
  if (c_col) {
    // column-major C: stored n rows of m. With the 16-byte rules met, each
    // epilogue warp stores its 32 rows of C as TMA boxes of 32 columns x 32
    // m-elements (no swizzle); otherwise by coalesced stores from registers.
    if (out->flags & EPI_BETA) return set_error(BBX_ERR_UNSUPPORTED, "column-major C with beta");
    out->flags |= EPI_C_TRANS;
    if ((((uintptr_t)q.c) & 15) == 0 && ((q.ldc * c_esz) & 15) == 0 && ((q.m * c_esz) & 15) == 0) {
      rc = make_map(&out->tmap_c, q.c, c_bf16 ? BBX_BF16 : BBX_F32, q.n, q.m, q.ldc, 32, 32, false);
      if (rc) return rc;
      out->flags |= EPI_TMA_STORE;
    }
    return BBX_OK;
  }
  // C through TMA stores when its base, pitch and row length meet the 16-byte
  // rules and the epilogue does not read C: 32-row boxes of 64 bytes (16 f32 /
  // 32 bf16), unswizzled, two per epilogue warp in turn. A TMA store clips the box at the tensor's edge in whole 16-byte
  // pieces of a row (measured: with m = 1031 f32 rows stored column-major,
  // element 1031 of a 16-byte piece holding 1028..1031 was written), so a row
  // length that is not a multiple of 16 bytes would write into the pitch
  // padding: such C goes through the staged stores.
  if (!(out->flags & EPI_BETA) && (((uintptr_t)q.c) & 15) == 0 && ((q.ldc * c_esz) & 15) == 0 &&
      ((q.n * c_esz) & 15) == 0) {
    rc = make_map(&out->tmap_c, q.c, c_bf16 ? BBX_BF16 : BBX_F32, q.m, q.n, q.ldc, 64 / c_esz, 32, false);
    if (rc) return rc;
    out->flags |= EPI_TMA_STORE;
  }
  return BBX_OK;
}

// Default tile: the 2-SM 256 x 256 pair for bf16 groups whose problems are all
// at least 256 x 256 and that fill every SM pair at least twice (measured
// 6-7% above the 1-SM 128 x 256 tile on 4096^3 blocks); otherwise 128 x 256,
// or 128 x 128 when no problem is wider than 128.
int pick_tile_n(const bbx_tc_problem_t* probs, int count, int in_dtype) {
  int maxn = 0, minmn = 1 << 30;
  long long pair_tiles = 0;
  for (int i = 0; i < count; ++i) {
    maxn = std::max(maxn, probs[i].n);
    minmn = std::min(minmn, std::min(probs[i].m, probs[i].n));
    pair_tiles += (long long)((probs[i].m + 255) / 256) * ((probs[i].n + 255) / 256);
  }
  DeviceState* d = nullptr;
  const int sms = device_state(&d) == BBX_OK ? d->sms : 148;
  if (in_dtype == BBX_BF16 && minmn >= 256 && pair_tiles >= 2LL * (sms / 2)) return 512;
  return maxn > 128 ? 256 : 128;
}

// Layout class shared by every problem of a group (one kernel variant per launch).
static int group_layout(const bbx_tc_problem_t* probs, int count, bool* amn, bool* bmn) {
  *amn = probs[0].trans_a != 0;
  *bmn = probs[0].trans_b == 0;
  for (int i = 1; i < count; ++i)
    if ((probs[i].trans_a != 0) != *amn || (probs[i].trans_b == 0) != *bmn)
      return set_error(BBX_ERR_INVALID, "all problems of a group must share transpose flags");
  return BBX_OK;
}

}  // namespace bbx

using namespace bbx;

struct bbx_tc_plan {
  int dtype = BBX_BF16;
  int bn = 256;
  bool ep8 = false;  // eight epilogue warps (every problem's K <= kTcEp8MaxK, kTc2Ep8MaxK for the pair)
  bool amn = false, bmn = true;
  int count = 0;
  int total_tiles = 0;
  int device = 0;
  TcProblem* d_table = nullptr;
  std::vector<TcProblem> host;  // kept for inline launches (count <= kTcMaxInline)
};

extern "C" {

const char* bbx_version(void) { return "bbts_b200 0.1 (sm_100a)"; }

int bbx_last_error(char* buf, size_t len) {
  const std::string& e = last_error();
  if (buf && len) {
    size_t n = std::min(len - 1, e.size());
    memcpy(buf, e.data(), n);
    buf[n] = 0;
  }
  return (int)e.size();
}

int bbx_num_sms(void) {
  DeviceState* d;
  if (device_state(&d)) return -1;
  return d->sms;
}

int bbx_check_device_status(void* stream, uint32_t* code_out) {
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  BBX_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  uint32_t code = 0;
  BBX_CUDA(cudaMemcpy(&code, d->status, 4, cudaMemcpyDeviceToHost));
  if (code_out) *code_out = code;
  if (code) {
    BBX_CUDA(cudaMemset(d->status, 0, 4));
    return set_error(BBX_ERR_DEVICE, "a kernel reported device status %u (bounded wait expired)", code);
  }
  return BBX_OK;
}

int bbx_matmul_f32(const float* a, const float* b, float* c, int m, int n, int k, long long lda,
                   long long ldb, long long ldc, int trans_a, int trans_b, float alpha, float beta,
                   const float* bias, int relu, int batch, long long stride_a, long long stride_b,
                   long long stride_c, void* stream) {
  if (!a || !b || !c) return set_error(BBX_ERR_INVALID, "null pointer");
  if (m <= 0 || n <= 0 || k < 0 || batch <= 0 || batch > 65535)
    return set_error(BBX_ERR_INVALID, "bad shape m=%d n=%d k=%d batch=%d", m, n, k, batch);
  F32GemmArgs g;
  g.a = a; g.b = b; g.c = c; g.bias = bias;
  g.m = m; g.n = n; g.k = k;
  g.lda = lda; g.ldb = ldb; g.ldc = ldc;
  g.stride_a = stride_a; g.stride_b = stride_b; g.stride_c = stride_c;
  g.trans_a = trans_a; g.trans_b = trans_b;
  g.alpha = alpha; g.beta = beta; g.relu = relu;
  dim3 grid((n + F32_BN - 1) / F32_BN, (m + F32_BM - 1) / F32_BM, batch);
  if (grid.y > 65535) return set_error(BBX_ERR_INVALID, "m too large");
  cudaStream_t st = (cudaStream_t)stream;
  if (f32_gemm_vector_ok(g)) {
    if (!trans_a && !trans_b) k_gemm_f32_v<false, false><<<grid, 256, 0, st>>>(g);
    else if (!trans_a) k_gemm_f32_v<false, true><<<grid, 256, 0, st>>>(g);
    else if (!trans_b) k_gemm_f32_v<true, false><<<grid, 256, 0, st>>>(g);
    else k_gemm_f32_v<true, true><<<grid, 256, 0, st>>>(g);
    BBX_CHECK_LAUNCH("k_gemm_f32_v");
    return BBX_OK;
  }
  k_gemm_f32<<<grid, 256, 0, st>>>(g);
  BBX_CHECK_LAUNCH("k_gemm_f32");
  return BBX_OK;
}

int bbx_tc_plan_create(int in_dtype, const bbx_tc_problem_t* problems, int count, int tile_n,
                       bbx_tc_plan_t** out) {
  if (!out || !problems || count <= 0) return set_error(BBX_ERR_INVALID, "bad plan arguments");
  if (in_dtype != BBX_BF16 && in_dtype != BBX_E4M3)
    return set_error(BBX_ERR_UNSUPPORTED, "tensor-core input dtype must be bf16 or e4m3");
  if (tile_n == 0) tile_n = pick_tile_n(problems, count, in_dtype);
  if (tile_n != 128 && tile_n != 256 && tile_n != 512)
    return set_error(BBX_ERR_INVALID, "tile_n must be 128, 256 or 512 (2-SM 256x256 pair)");
  if (tile_n == 512 && in_dtype != BBX_BF16) return set_error(BBX_ERR_UNSUPPORTED, "the 2-SM tile is bf16 only");
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  auto* p = new bbx_tc_plan();
  p->dtype = in_dtype;
  p->bn = tile_n;
  p->count = count;
  cudaGetDevice(&p->device);
  rc = group_layout(problems, count, &p->amn, &p->bmn);
  if (rc) { delete p; return rc; }
  p->host.resize(count);
  // The persistent grid strides over the concatenated tile list, so CTA c runs
  // tiles c, c + grid, ... (in odd rounds the kernel hands the round's tiles
  // out in reverse). Problems go in descending order of a tile's cost (stable):
  // its k-blocks plus its 32-column epilogue chunks, the two phases a tile is
  // paced by. Each round of `grid` consecutive tiles then holds tiles of
  // similar cost and the cheapest come last, which evens out the work per CTA
  // when a group mixes short and long K loops or narrow and wide problems
  // (measured against descending K alone on the contraction-only 600-op DAG's
  // tensor groups, with the snake rounds: 2.94 -> 2.86 ms).
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  auto tcost = [&](int x) {
    const int bnn = tile_n == 128 ? 128 : 256;
    return (problems[x].k + 63) / 64 + (std::min(problems[x].n, bnn) + 31) / 32;
  };
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return tcost(x) > tcost(y); });
  int tiles = 0;
  for (int i = 0; i < count; ++i) {
    rc = build_problem(in_dtype, problems[order[i]], tile_n, &p->host[i]);
    if (rc) { delete p; return rc; }
    p->host[i].tile_start = tiles;
    tiles += p->host[i].tiles_m * p->host[i].tiles_n;
  }
  p->total_tiles = tiles;
  int max_k = 0;
  for (int i = 0; i < count; ++i) max_k = std::max(max_k, problems[i].k);
  p->ep8 = max_k <= (tile_n == 512 ? kTc2Ep8MaxK : kTcEp8MaxK);
  if (count > kTcMaxInline) {
    cudaError_t e = cudaMalloc(&p->d_table, sizeof(TcProblem) * count);
    if (e != cudaSuccess) { delete p; return set_error(BBX_ERR_CUDA, "cudaMalloc(plan table): %s", cudaGetErrorString(e)); }
    e = cudaMemcpy(p->d_table, p->host.data(), sizeof(TcProblem) * count, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { cudaFree(p->d_table); delete p; return set_error(BBX_ERR_CUDA, "plan upload: %s", cudaGetErrorString(e)); }
  }
  *out = p;
  return BBX_OK;
}

int bbx_tc_plan_launch(bbx_tc_plan_t* p, void* stream) {
  if (!p) return set_error(BBX_ERR_INVALID, "null plan");
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  TcArgs args;
  memset(&args, 0, sizeof(args));
  args.table = p->d_table;
  args.num_problems = p->count;
  args.total_tiles = p->total_tiles;
  args.status = d->status;
  if (!p->d_table)
    for (int i = 0; i < p->count; ++i) args.inline_probs[i] = p->host[i];
  if (p->bn == 512) {
    // one CTA pair (cluster of 2) per 256 x 256 tile, persistent over the tile list
    const int grid = 2 * std::min(p->total_tiles, d->sms / 2);
    return launch_tc2(p->amn, p->bmn, p->ep8, args, grid, (cudaStream_t)stream);
  }
  const int grid = std::min(p->total_tiles, d->sms);
  return launch_tc(p->bn, p->amn, p->bmn, p->dtype == BBX_E4M3, p->ep8, args, grid,
                   (cudaStream_t)stream, d);
}

int bbx_tc_plan_tile_n(const bbx_tc_plan_t* p) { return p ? p->bn : 0; }

int bbx_tc_plan_destroy(bbx_tc_plan_t* p) {
  if (!p) return BBX_OK;
  if (p->d_table) cudaFree(p->d_table);
  delete p;
  return BBX_OK;
}

int bbx_matmul_tc(int in_dtype, const bbx_tc_problem_t* problems, int count, int tile_n,
                  void* stream) {
  if (count <= 0 || !problems) return set_error(BBX_ERR_INVALID, "no problems");
  if (tile_n == 0) tile_n = pick_tile_n(problems, count, in_dtype);
  // Problems travel in the kernel parameters, kTcMaxInline per launch: no
  // device table, no host-to-device copy, so the call is safe to capture in a
  // CUDA graph. Large groups that are launched repeatedly should use a plan.
  for (int i = 0; i < count; i += kTcMaxInline) {
    const int c = std::min(kTcMaxInline, count - i);
    bbx_tc_plan_t* p = nullptr;
    int rc = bbx_tc_plan_create(in_dtype, problems + i, c, tile_n, &p);
    if (rc) return rc;
    rc = bbx_tc_plan_launch(p, stream);
    bbx_tc_plan_destroy(p);  // inline plans own no device memory
    if (rc) return rc;
  }
  return BBX_OK;
}

int bbx_add_f32(const float* a, const float* b, float* c, long long n, void* stream) {
  return bbx_binary_f32(BBX_B_ADD, a, b, c, n, 1.f, 1.f, stream);
}

int bbx_binary_f32(int op, const float* a, const float* b, float* c, long long n, float ca,
                   float cb, void* stream) {
  if (op < 0 || op > B_DIV) return set_error(BBX_ERR_INVALID, "unknown binary op %d", op);
  if (n == 0) return BBX_OK;
  if (!a || !b || !c || n < 0) return set_error(BBX_ERR_INVALID, "bad binary arguments");
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  k_binary<<<grid_for((n + 3) / 4, 256, d->sms), 256, 0, (cudaStream_t)stream>>>(op, a, b, c, n, ca, cb);
  BBX_CHECK_LAUNCH("k_binary");
  return BBX_OK;
}

int bbx_unary_f32(int op, const float* in, float* out, long long n, float param, void* stream) {
  if (op < 0 || op > U_RELU_LO) return set_error(BBX_ERR_INVALID, "unknown unary op %d", op);
  if (n == 0) return BBX_OK;
  if (!in || !out || n < 0) return set_error(BBX_ERR_INVALID, "bad unary arguments");
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  k_unary<<<grid_for((n + 3) / 4, 256, d->sms), 256, 0, (cudaStream_t)stream>>>(op, in, out, n, param);
  BBX_CHECK_LAUNCH("k_unary");
  return BBX_OK;
}

int bbx_reduce_f32(const float* const* inputs, int n_in, float* out, long long n, int kahan,
                   void* stream) {
  if (!inputs || !out || n_in < 1 || n < 0) return set_error(BBX_ERR_INVALID, "bad reduce arguments");
  for (int i = 0; i < n_in; ++i)
    if (!inputs[i]) return set_error(BBX_ERR_INVALID, "null reduce input %d", i);
  if (n == 0) return BBX_OK;
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // Chunks of up to 32 inputs; later chunks fold into `out` first, which keeps
  // the left-to-right order (out = ((in0+...+in31) + in32) + ...). With Kahan
  // the compensation restarts at chunk boundaries.
  int done = 0;
  while (done < n_in) {
    ReduceArgs ra;
    int cnt = 0;
    if (done > 0) ra.in[cnt++] = out;
    while (cnt < kMaxReduceInputs && done < n_in) ra.in[cnt++] = inputs[done++];
    if (cnt == 1) {
      if (ra.in[0] != out) BBX_CUDA(cudaMemcpyAsync(out, ra.in[0], n * 4, cudaMemcpyDeviceToDevice, st));
      continue;
    }
    const int grid = grid_for((n + 3) / 4, 256, d->sms);
    if (kahan) k_reduce<true><<<grid, 256, 0, st>>>(ra, cnt, out, n);
    else k_reduce<false><<<grid, 256, 0, st>>>(ra, cnt, out, n);
    BBX_CHECK_LAUNCH("k_reduce");
  }
  return BBX_OK;
}

int bbx_bias_add_f32(const float* in, const float* bias, float* out, int rows, int cols, int relu,
                     void* stream) {
  if (!in || !bias || !out || rows < 0 || cols <= 0) return set_error(BBX_ERR_INVALID, "bad bias_add arguments");
  if (rows == 0) return BBX_OK;
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  k_bias_add<<<grid_for((long long)rows * cols, 256, d->sms), 256, 0, (cudaStream_t)stream>>>(in, bias, out, rows, cols, relu);
  BBX_CHECK_LAUNCH("k_bias_add");
  return BBX_OK;
}

int bbx_colsum_f32(const float* in, float* out, int rows, int cols, long long ld, int accumulate,
                   void* stream) {
  if (!in || !out || rows < 0 || cols <= 0 || ld < cols) return set_error(BBX_ERR_INVALID, "bad colsum arguments");
  k_colsum<<<(cols + 127) / 128, 128, 0, (cudaStream_t)stream>>>(in, out, rows, cols, ld, accumulate);
  BBX_CHECK_LAUNCH("k_colsum");
  return BBX_OK;
}

int bbx_cast(int src_dtype, const void* in, int dst_dtype, void* out, long long n, void* stream) {
  if (!in || !out || n < 0) return set_error(BBX_ERR_INVALID, "bad cast arguments");
  if (n == 0) return BBX_OK;
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  const int grid = grid_for(n, 256, d->sms);
  cudaStream_t st = (cudaStream_t)stream;
  if (src_dtype == BBX_F32 && dst_dtype == BBX_BF16) {
    k_f32_to_bf16<<<grid, 256, 0, st>>>((const float*)in, (__nv_bfloat16*)out, n);
  } else if (src_dtype == BBX_BF16 && dst_dtype == BBX_F32) {
    k_bf16_to_f32<<<grid, 256, 0, st>>>((const __nv_bfloat16*)in, (float*)out, n);
  } else if (src_dtype == dst_dtype) {
    BBX_CUDA(cudaMemcpyAsync(out, in, n * (src_dtype == BBX_F32 ? 4 : src_dtype == BBX_BF16 ? 2 : 1),
                             cudaMemcpyDeviceToDevice, st));
    return BBX_OK;
  } else {
    return set_error(BBX_ERR_UNSUPPORTED, "cast %d -> %d", src_dtype, dst_dtype);
  }
  BBX_CHECK_LAUNCH("cast");
  return BBX_OK;
}

int bbx_relu_split(const float* z, void* hi, void* lo, long long n, void* stream) {
  if (!z || !hi || !lo || n < 0) return set_error(BBX_ERR_INVALID, "bad relu_split arguments");
  if (n == 0) return BBX_OK;
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  k_relu_split<<<grid_for((n + 3) / 4, 256, d->sms), 256, 0, (cudaStream_t)stream>>>(
      z, (__nv_bfloat16*)hi, (__nv_bfloat16*)lo, n);
  BBX_CHECK_LAUNCH("relu_split");
  return BBX_OK;
}

int bbx_quantize_e4m3(int src_dtype, const void* in, void* out, int rows, int cols, int transpose,
                      float* scale_out, void* stream) {
  if (!in || !out || !scale_out || rows <= 0 || cols <= 0) return set_error(BBX_ERR_INVALID, "bad quantize arguments");
  if (src_dtype != BBX_F32 && src_dtype != BBX_BF16) return set_error(BBX_ERR_UNSUPPORTED, "quantize source dtype");
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // the absmax word is stream-ordered scratch of this call, so quantisations
  // on different streams never share it
  unsigned int* amax = nullptr;
  BBX_CUDA(cudaMallocAsync((void**)&amax, 4, st));
  BBX_CUDA(cudaMemsetAsync(amax, 0, 4, st));
  uint8_t* o = (uint8_t*)out;
  cudaError_t le;
  if (src_dtype == BBX_F32) {
    const float* i = (const float*)in;
    le = launch_quantize_batch(&i, &o, 1, rows, cols, transpose, amax, scale_out, d->sms, st);
  } else {
    const __nv_bfloat16* i = (const __nv_bfloat16*)in;
    le = launch_quantize_batch(&i, &o, 1, rows, cols, transpose, amax, scale_out, d->sms, st);
  }
  cudaFreeAsync(amax, st);
  if (le != cudaSuccess) return set_error(BBX_ERR_CUDA, "quantize_e4m3: %s", cudaGetErrorString(le));
  return BBX_OK;
}

int bbx_quantize_e4m3_batched(int src_dtype, const void* const* in, void* const* out, int count, int rows, int cols,
                              int transpose, float* scales_out, void* stream) {
  if (count == 0) return BBX_OK;
  if (!in || !out || !scales_out || rows <= 0 || cols <= 0 || count < 0)
    return set_error(BBX_ERR_INVALID, "bad batched quantize arguments");
  if (src_dtype != BBX_F32 && src_dtype != BBX_BF16) return set_error(BBX_ERR_UNSUPPORTED, "quantize source dtype");
  for (int i = 0; i < count; ++i)
    if (!in[i] || !out[i]) return set_error(BBX_ERR_INVALID, "null block pointer %d", i);
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // one absmax word per block, stream-ordered scratch of this call
  unsigned int* amax = nullptr;
  BBX_CUDA(cudaMallocAsync((void**)&amax, sizeof(unsigned int) * count, st));
  BBX_CUDA(cudaMemsetAsync(amax, 0, sizeof(unsigned int) * count, st));
  cudaError_t le = src_dtype == BBX_F32
                       ? launch_quantize_batch((const float* const*)in, (uint8_t* const*)out, count, rows, cols,
                                               transpose, amax, scales_out, d->sms, st)
                       : launch_quantize_batch((const __nv_bfloat16* const*)in, (uint8_t* const*)out, count, rows,
                                               cols, transpose, amax, scales_out, d->sms, st);
  cudaFreeAsync(amax, st);
  if (le != cudaSuccess) return set_error(BBX_ERR_CUDA, "quantize_e4m3_batched: %s", cudaGetErrorString(le));
  return BBX_OK;
}

int bbx_fill_philox(int dtype, void* out, long long n, unsigned long long seed, int dist, float a,
                    float b, void* stream) {
  if (!out || n < 0 || (dist != 0 && dist != 1)) return set_error(BBX_ERR_INVALID, "bad fill arguments");
  if (n == 0) return BBX_OK;
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  const int grid = grid_for((n + 3) / 4, 256, d->sms);
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == BBX_F32) k_fill_philox<float><<<grid, 256, 0, st>>>((float*)out, n, seed, dist, a, b);
  else if (dtype == BBX_BF16) k_fill_philox<__nv_bfloat16><<<grid, 256, 0, st>>>((__nv_bfloat16*)out, n, seed, dist, a, b);
  else return set_error(BBX_ERR_UNSUPPORTED, "fill dtype %d", dtype);
  BBX_CHECK_LAUNCH("k_fill_philox");
  return BBX_OK;
}

int bbx_softmax_ce_f32(const float* logits, const int* labels, float* loss, float* grad, int rows,
                       int cols, long long ld, float grad_scale, void* stream) {
  return bbx_softmax_ce(logits, labels, loss, grad, BBX_F32, rows, cols, ld, grad_scale, stream);
}

int bbx_softmax_ce(const float* logits, const int* labels, float* loss, void* grad, int grad_dtype, int rows,
                   int cols, long long ld, float grad_scale, void* stream) {
  if (!logits || !labels || !loss || rows < 0 || cols <= 0 || ld < cols)
    return set_error(BBX_ERR_INVALID, "bad softmax_ce arguments");
  if (grad_dtype != BBX_F32 && grad_dtype != BBX_BF16) return set_error(BBX_ERR_UNSUPPORTED, "softmax_ce grad dtype");
  if (rows == 0) return BBX_OK;
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  const int warps = 8;
  int grid = std::min((rows + warps - 1) / warps, d->sms * 8);
  if (grad_dtype == BBX_F32)
    k_softmax_ce<float><<<grid, warps * 32, 0, (cudaStream_t)stream>>>(logits, labels, loss, (float*)grad, rows, cols,
                                                                      ld, grad_scale);
  else
    k_softmax_ce<__nv_bfloat16><<<grid, warps * 32, 0, (cudaStream_t)stream>>>(
        logits, labels, loss, (__nv_bfloat16*)grad, rows, cols, ld, grad_scale);
  BBX_CHECK_LAUNCH("k_softmax_ce");
  return BBX_OK;
}

int bbx_permute(const float* in, int rank, const long long* in_dims, const int* perm, int dst_dtype,
                void* out, void* stream) {
  if (!in || !out || !in_dims || !perm || rank < 1 || rank > 4)
    return set_error(BBX_ERR_INVALID, "bad permute arguments");
  if (dst_dtype != BBX_F32 && dst_dtype != BBX_BF16) return set_error(BBX_ERR_UNSUPPORTED, "permute dtype");
  PermArgs pa;
  memset(&pa, 0, sizeof(pa));
  pa.rank = rank;
  long long istr[4];
  long long s = 1;
  for (int d = rank - 1; d >= 0; --d) { istr[d] = s; s *= in_dims[d]; }
  const long long n = s;
  unsigned seen = 0;
  for (int d = 0; d < rank; ++d) {
    if (perm[d] < 0 || perm[d] >= rank || (seen & (1u << perm[d])))
      return set_error(BBX_ERR_INVALID, "perm is not a permutation");
    seen |= 1u << perm[d];
    pa.odims[d] = in_dims[perm[d]];
    pa.istride[d] = istr[perm[d]];
  }
  s = 1;
  for (int d = rank - 1; d >= 0; --d) { pa.ostride[d] = s; s *= pa.odims[d]; }
  if (n == 0) return BBX_OK;
  DeviceState* dv;
  int rc = device_state(&dv);
  if (rc) return rc;
  const int grid = grid_for(n, 256, dv->sms);
  if (dst_dtype == BBX_F32) k_permute<float><<<grid, 256, 0, (cudaStream_t)stream>>>(in, (float*)out, pa, n);
  else k_permute<__nv_bfloat16><<<grid, 256, 0, (cudaStream_t)stream>>>(in, (__nv_bfloat16*)out, pa, n);
  BBX_CHECK_LAUNCH("k_permute");
  return BBX_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ grouped streaming ops
struct bbx_stream_plan {
  StreamOp* d_table = nullptr;
  int count = 0;
  long long total_chunks = 0;  // items when bulk
  bool bulk = false;
};

namespace bbx {
// *bulk: every op qualifies for the bulk-staged kernel (all pointers 16-byte
// aligned); the table then counts items of bulk_tile elements instead of
// kStreamChunk chunks.
static int build_stream_table(const bbx_stream_op_t* ops, int count, std::vector<StreamOp>* out,
                              long long* total, bool* bulk, bool allow_bulk = true) {
  static_assert(kStreamMaxIn == BBX_STREAM_MAX_IN, "stream op fan-in mismatch");
  out->resize(count);
  // Blocks stride over the chunk list (block b takes chunks b, b + grid, ...),
  // and a chunk costs about (inputs + 1) x its bytes: ops go in descending
  // fan-in, then size, so each round of `grid` chunks has similar cost. The ops
  // of one launch are independent, so the order changes no result.
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  auto fan_in = [&](int i) { return ops[i].kind == S_SUM ? ops[i].n_in : (ops[i].kind == S_BINARY ? 2 : 1); };
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    if (fan_in(x) != fan_in(y)) return fan_in(x) > fan_in(y);
    return ops[x].n > ops[y].n;
  });
  long long chunks = 0;
  for (int k = 0; k < count; ++k) {
    const int i = order[k];
    const bbx_stream_op_t& q = ops[i];
    StreamOp& o = (*out)[k];
    memset(&o, 0, sizeof(o));
    if (q.kind < S_SUM || q.kind > S_CAST) return set_error(BBX_ERR_INVALID, "stream op %d: kind %d", i, q.kind);
    const int need = q.kind == S_SUM ? q.n_in : (q.kind == S_BINARY ? 2 : 1);
    if (need < 1 || need > kStreamMaxIn) return set_error(BBX_ERR_INVALID, "stream op %d: %d inputs", i, need);
    if ((q.in_dtype != BBX_F32 && q.in_dtype != BBX_BF16) || (q.out_dtype != BBX_F32 && q.out_dtype != BBX_BF16))
      return set_error(BBX_ERR_UNSUPPORTED, "stream op %d: dtype", i);
    if (q.n < 0) return set_error(BBX_ERR_INVALID, "stream op %d: n < 0", i);
    if (q.n > 0 && !q.out) return set_error(BBX_ERR_INVALID, "stream op %d: null output", i);
    uintptr_t align = (uintptr_t)q.out;
    for (int j = 0; j < need; ++j) {
      if (q.n > 0 && !q.in[j]) return set_error(BBX_ERR_INVALID, "stream op %d: null input %d", i, j);
      o.in[j] = q.in[j];
      align |= (uintptr_t)q.in[j];
    }
    o.kind = q.kind; o.op = q.op; o.in_dtype = q.in_dtype; o.out_dtype = q.out_dtype;
    o.n_in = need; o.kahan = q.kahan; o.n = q.n; o.out = q.out; o.p0 = q.p0; o.p1 = q.p1;
    // 2: every pointer 16-byte aligned (the wide path); 1: the 4-element path
    const uintptr_t need_align = (q.in_dtype == BBX_F32 || q.out_dtype == BBX_F32) ? 15 : 7;
    o.vec = (align & 15) == 0 ? 2 : (align & need_align) == 0 ? 1 : 0;
    o.chunk_start = chunks;
    chunks += (q.n + kStreamChunk - 1) / kStreamChunk;
  }
  *total = chunks;
  bool all16 = true;
  for (const StreamOp& o : *out) all16 = all16 && (o.n == 0 || o.vec == 2);
  *bulk = all16 && allow_bulk;
  if (*bulk) {
    long long items = 0;
    for (StreamOp& o : *out) {
      o.tile = bulk_tile(o.n_in, o.in_dtype == BBX_BF16 ? 2 : 4, o.out_dtype == BBX_BF16 ? 2 : 4);
      o.chunk_start = items;
      items += (o.n + o.tile - 1) / o.tile;
    }
    *total = items;
  }
  return BBX_OK;
}
}  // namespace bbx

extern "C" {

int bbx_stream_plan_create(const bbx_stream_op_t* ops, int count, bbx_stream_plan_t** out) {
  return bbx_stream_plan_create_kernel(ops, count, BBX_STREAM_KERNEL_AUTO, out);
}

int bbx_stream_plan_create_kernel(const bbx_stream_op_t* ops, int count, int kernel, bbx_stream_plan_t** out) {
  if (!ops || count <= 0 || !out) return set_error(BBX_ERR_INVALID, "bad stream plan arguments");
  if (kernel != BBX_STREAM_KERNEL_AUTO && kernel != BBX_STREAM_KERNEL_REGISTER)
    return set_error(BBX_ERR_INVALID, "stream plan kernel %d", kernel);
  std::vector<StreamOp> table;
  long long total = 0;
  bool bulk = false;
  int rc = build_stream_table(ops, count, &table, &total, &bulk, kernel == BBX_STREAM_KERNEL_AUTO);
  if (rc) return rc;
  auto* p = new bbx_stream_plan();
  p->count = count;
  p->total_chunks = total;
  p->bulk = bulk;
  cudaError_t e = cudaMalloc(&p->d_table, sizeof(StreamOp) * count);
  if (e == cudaSuccess) e = cudaMemcpy(p->d_table, table.data(), sizeof(StreamOp) * count, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    if (p->d_table) cudaFree(p->d_table);
    delete p;
    return set_error(BBX_ERR_CUDA, "stream plan upload: %s", cudaGetErrorString(e));
  }
  *out = p;
  return BBX_OK;
}

int bbx_stream_plan_launch(bbx_stream_plan_t* p, void* stream) {
  if (!p) return set_error(BBX_ERR_INVALID, "null stream plan");
  if (p->total_chunks == 0) return BBX_OK;
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  if (p->bulk) {
    const long long grid = std::min<long long>(p->total_chunks, (long long)d->sms);
    k_stream_bulk<kBulkStoreTS><<<(int)grid, kBulkThreads, bulk_smem_bytes(p->count), (cudaStream_t)stream>>>(
        p->d_table, p->count, p->total_chunks, d->status, kBulkPiece);
    BBX_CHECK_LAUNCH("k_stream_bulk");
    return BBX_OK;
  }
  long long grid = std::min<long long>(p->total_chunks, (long long)d->sms * 8);
  k_stream_group<<<(int)grid, 256, 0, (cudaStream_t)stream>>>(p->d_table, p->count, p->total_chunks);
  BBX_CHECK_LAUNCH("k_stream_group");
  return BBX_OK;
}

int bbx_stream_plan_bulk(const bbx_stream_plan_t* p) {
  if (!p) return set_error(BBX_ERR_INVALID, "null stream plan");
  return p->bulk ? 1 : 0;
}

int bbx_stream_plan_destroy(bbx_stream_plan_t* p) {
  if (!p) return BBX_OK;
  if (p->d_table) cudaFree(p->d_table);
  delete p;
  return BBX_OK;
}

int bbx_stream_group(const bbx_stream_op_t* ops, int count, void* stream) {
  if (!ops || count <= 0) return set_error(BBX_ERR_INVALID, "bad stream group arguments");
  DeviceState* d;
  int rc = device_state(&d);
  if (rc) return rc;
  // Ops travel in the kernel parameters, kStreamInline per launch (capture-safe).
  for (int i = 0; i < count; i += kStreamInline) {
    const int c = std::min(kStreamInline, count - i);
    std::vector<StreamOp> table;
    long long total = 0;
    bool bulk = false;
    rc = build_stream_table(ops + i, c, &table, &total, &bulk);
    if (rc) return rc;
    if (total == 0) continue;
    StreamInline args;
    memset(&args, 0, sizeof(args));
    for (int j = 0; j < c; ++j) args.ops[j] = table[j];
    if (bulk) {
      const long long grid = std::min<long long>(total, (long long)d->sms);
      k_stream_bulk_inline<kBulkStoreTS><<<(int)grid, kBulkThreads, bulk_smem_bytes(c), (cudaStream_t)stream>>>(
          args, c, total, d->status, kBulkPiece);
      BBX_CHECK_LAUNCH("k_stream_bulk_inline");
      continue;
    }
    long long grid = std::min<long long>(total, (long long)d->sms * 8);
    k_stream_group_inline<<<(int)grid, 256, 0, (cudaStream_t)stream>>>(args, c, total);
    BBX_CHECK_LAUNCH("k_stream_group_inline");
  }
  return BBX_OK;
}

}  // extern "C"
