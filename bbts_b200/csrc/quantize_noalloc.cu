// Allocation-free FP8-E4M3 per-block quantisation.
//
// Some callers of this library cannot allocate device memory while they run:
// code that executes under an external memory manager which owns every byte
// of the GPU (a serving framework's pooled allocator that forbids outside
// cudaMalloc), code on a latency-critical path where cudaMalloc / cudaFree
// would synchronise the device, and code that must keep a fixed footprint
// known at start-up. bbx_quantize_e4m3 keeps its absmax word in scratch that
// the library allocates on first use; this variant takes its scratch from the
// fixed array below instead, so a call never allocates.
//
// Scratch: kNoAllocMaxBlocks absmax words (4 KiB) in a file-scope __device__
// array. Every GPU that loads the library holds this array until the process
// exits. The array is shared by every call on a device and keeps the previous
// call's contents, so each call clears the words it uses first; two calls
// whose work overlaps on the GPU (different streams, no ordering between them)
// race on the same words and must not be issued.
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <mutex>
#include "bbts_b200.h"
#include "common.h"
#include "quant_ops.cuh"

namespace bbx {

constexpr int kNoAllocMaxBlocks = 1024;

// One absmax word per block of a call.
static __device__ __align__(256) unsigned int g_noalloc_absmax[kNoAllocMaxBlocks];

// Device address of g_noalloc_absmax per device. In host code the symbol name
// is only a host-side stand-in, so the address is looked up once per device
// (with that device current) and passed to the kernels.
static std::mutex g_noalloc_mu;
static unsigned int* g_noalloc_ptr[64] = {};
static int g_noalloc_sms[64] = {};

static int noalloc_scratch(unsigned int** ptr, int* sms) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(BBX_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return set_error(BBX_ERR_INVALID, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_absmax);
    if (e != cudaSuccess || !p)
      return set_error(BBX_ERR_CUDA, "cudaGetSymbolAddress(no-alloc scratch): %s", cudaGetErrorString(e));
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return set_error(BBX_ERR_CUDA, "cudaDeviceGetAttribute: %s", cudaGetErrorString(e));
    g_noalloc_ptr[dev] = (unsigned int*)p;
    g_noalloc_sms[dev] = n;
  }
  *ptr = g_noalloc_ptr[dev];
  *sms = g_noalloc_sms[dev];
  return BBX_OK;
}

}  // namespace bbx

using namespace bbx;

extern "C" int bbx_quantize_e4m3_batched_noalloc(int src_dtype, const void* const* in, void* const* out,
                                                 int count, int rows, int cols, int transpose,
                                                 float* scales_out, void* stream) {
  if (count == 0) return BBX_OK;  // an empty batch touches nothing, null arrays included
  if (!in || !out || !scales_out || rows <= 0 || cols <= 0 || count < 0)
    return set_error(BBX_ERR_INVALID, "bad no-alloc quantize arguments");
  if (count > kNoAllocMaxBlocks)
    return set_error(BBX_ERR_INVALID,
                     "bbx_quantize_e4m3_batched_noalloc: %d blocks requested, the fixed scratch holds at most %d "
                     "per call; split the batch",
                     count, kNoAllocMaxBlocks);
  if (src_dtype != BBX_F32 && src_dtype != BBX_BF16) return set_error(BBX_ERR_UNSUPPORTED, "quantize source dtype");
  for (int i = 0; i < count; ++i)
    if (!in[i] || !out[i]) return set_error(BBX_ERR_INVALID, "null block pointer %d", i);
  unsigned int* scratch = nullptr;
  int sms = 0;
  int rc = noalloc_scratch(&scratch, &sms);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // the array keeps the previous call's words: clear the ones this call uses
  cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned int) * count, st);
  if (e != cudaSuccess) return set_error(BBX_ERR_CUDA, "cudaMemsetAsync(no-alloc scratch): %s", cudaGetErrorString(e));
  e = src_dtype == BBX_F32
          ? launch_quantize_batch((const float* const*)in, (uint8_t* const*)out, count, rows, cols, transpose, scratch,
                                  scales_out, sms, st)
          : launch_quantize_batch((const __nv_bfloat16* const*)in, (uint8_t* const*)out, count, rows, cols, transpose,
                                  scratch, scales_out, sms, st);
  if (e != cudaSuccess) return set_error(BBX_ERR_CUDA, "no-alloc quantize launch: %s", cudaGetErrorString(e));
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(BBX_ERR_CUDA, "no-alloc quantize launch: %s", cudaGetErrorString(e));
  return BBX_OK;
}
