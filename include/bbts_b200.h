/*
 * bbts_b200 C ABI: B200 (sm_100a) kernels behind BarbaTOS's block-op ud functions.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t passed
 * as `void*` (NULL = legacy default stream), returns 0 on success and a negative
 * BBX_ERR_* code on failure (message via bbx_last_error), and never throws.
 * Work is stream-ordered: a call returns after enqueueing its kernels.
 * Matrices are row-major with an explicit leading dimension (pitch, elements),
 * the layout of the reference's "dense" format (src/tensor/builtin_formats.cc:23-42).
 *
 * Reference interfaces replaced (paths inside dcbdan/bbts):
 *   ud_impl_t::fn of the dense block uds      src/ud_functions/ud_function.h:168-170
 *   dense_matrix_mult_t::mult                 src/ud_functions/impls/dense_matrix_mult.cc:50-86
 *   dense_matrix_gpu_mult_t::mult (cuBLAS)    src/ud_functions/impls/dense_matrix_gpu_mult.cu:51-85
 *   dense_matrix_add_t::add / dense_add_kernel src/ud_functions/impls/dense_matrix_add.cc:46-77,
 *                                             src/ud_functions/impls/dense_matrix_gpu_add.cu:47-85
 *   local_reduce_op_t::apply (n-ary reduce)   src/operations/local_reduce_op.cc:23-91
 *   relu / relu_dif / sigmoid / hadamard /
 *   weighted_sum impls                        src/ud_functions/impls/dense_matrix_*.cc:46-81
 *   FNN ops                                   applications/fnn/ffnn_*.cc
 *   contraction (einsum) cpu_op / gpu_op      libraries/cutensor/contraction.h:204-631
 *   gpu_scheduler_impl_t (per-op UVM path)    src/ud_functions/gpu_scheduler_impl.cc:34-112
 */
#ifndef BBTS_B200_H
#define BBTS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BBX_OK 0
#define BBX_ERR_INVALID (-1)     /* bad argument (shape, alignment, null pointer) */
#define BBX_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define BBX_ERR_UNSUPPORTED (-3) /* valid request this build does not implement */
#define BBX_ERR_DEVICE (-4)      /* a kernel reported a bounded-wait timeout */
#define BBX_ERR_NOT_FOUND (-5)   /* unknown ud / tensor / handle */

/* element types of block payloads */
#define BBX_F32 0
#define BBX_BF16 1
#define BBX_E4M3 2

/* unary ops (bbx_unary_f32) */
#define BBX_U_RELU 0        /* dense_matrix_relu.cc:63-69 */
#define BBX_U_RELU_DIF 1    /* dense_matrix_relu_dif.cc:63-69 */
#define BBX_U_SIGMOID_REF 2 /* dense_matrix_sigmoid.cc:64-70, 1/(1+exp(v)) exactly as the reference */
#define BBX_U_SIGMOID 3     /* 1/(1+exp(-v)), libraries/cutensor/ew.h:158-161 */
#define BBX_U_EXP 4
#define BBX_U_SQUARE 5
#define BBX_U_SQRT 6
#define BBX_U_ADD_SCALAR 7
#define BBX_U_SCALE 8
/* relu(v) - bf16(relu(v)), exact in f32: with an f32 -> bf16 output it is the
 * low part lo of bbx_relu_split, so a grouped launch can write hi (BBX_U_RELU
 * to bf16) and lo as two element-wise ops */
#define BBX_U_RELU_LO 9

/* binary ops (bbx_binary_f32) */
#define BBX_B_ADD 0         /* dense_matrix_add.cc:67-73 */
#define BBX_B_WEIGHTED 1    /* dense_matrix_weighted_sum.cc:70-76, ca*a + cb*b */
#define BBX_B_HADAMARD 2    /* dense_matrix_hadamard.cc:67-73 */
#define BBX_B_MAX 3
#define BBX_B_MIN 4
#define BBX_B_SUB 5
#define BBX_B_DIV 6

/* tensor-core epilogue flags (bbx_tc_problem_t.flags) */
#define BBX_EPI_RELU 1
#define BBX_EPI_OUT_BF16 2
#define BBX_EPI_BIAS 4
#define BBX_EPI_BETA 8
/* tensor-core problems only: C is column-major, element (i, j) at
 * c[i + j * ldc] (ldc >= m); not with BBX_EPI_BETA (BBX_ERR_UNSUPPORTED) */
#define BBX_EPI_C_COLMAJOR 32

/* ------------------------------------------------------------------ misc */
const char* bbx_version(void);
/* Copies the calling thread's last error message into buf; returns its length. */
int bbx_last_error(char* buf, size_t len);
/* Number of SMs of the current device (grids are sized to multiples of it).
 * The library sets up per-device state (a status word, kernel attributes) on
 * the first call that needs it on a device; that set-up allocates, so the
 * first call should not come inside a stream capture: calling this function
 * once per device first does it. */
int bbx_num_sms(void);
/* Synchronises `stream`, then reads and clears the device status word written
 * by kernels whose bounded waits ran out. Returns 0 or BBX_ERR_DEVICE. */
int bbx_check_device_status(void* stream, uint32_t* code_out);

/* ------------------------------------------------------------------ block matmul */
/* FP32 SIMT matmul: C = alpha*op(A)*op(B) + beta*C (+bias[col]) (relu), batched
 * over `batch` with element strides. Replaces dense_matrix_mult_t::mult
 * (dense_matrix_mult.cc:78-82: cblas_sgemm RowMajor with trans flags b0/b1) and
 * the batched cblas_sgemm_batch_strided of contraction.h:439-461. */
int bbx_matmul_f32(const float* a, const float* b, float* c, int m, int n, int k, long long lda,
                   long long ldb, long long ldc, int trans_a, int trans_b, float alpha, float beta,
                   const float* bias, int relu, int batch, long long stride_a, long long stride_b,
                   long long stride_c, void* stream);

/* One tensor-core block product. a/b are bf16 or e4m3 (row-major, pitches in
 * elements, pitch*elem_size and base pointers 16-byte aligned), c is f32 or
 * bf16 (BBX_EPI_OUT_BF16). op(A) is m x k, op(B) is k x n. */
typedef struct bbx_tc_problem {
  const void* a;
  const void* b;
  void* c;
  const float* bias; /* length n, used with BBX_EPI_BIAS */
  int m, n, k;
  int trans_a, trans_b;
  int flags;
  long long lda, ldb, ldc;
  float alpha, beta;
} bbx_tc_problem_t;

/* Grouped tensor-core matmul over `count` independent problems in ONE
 * persistent tcgen05 kernel (TMA-fed smem ring, TMEM accumulators).
 * in_dtype = BBX_BF16 or BBX_E4M3; tile_n = 128, 256 or 0 (auto). Replaces the
 * per-op cuBLAS SGEMM of dense_matrix_gpu_mult.cu:81 for a whole batch of
 * matrix_mult APPLY commands. */
int bbx_matmul_tc(int in_dtype, const bbx_tc_problem_t* problems, int count, int tile_n,
                  void* stream);

/* A prepared grouped matmul (tensor maps built and uploaded once) for repeated
 * launches, e.g. inside a captured CUDA graph. */
typedef struct bbx_tc_plan bbx_tc_plan_t;
int bbx_tc_plan_create(int in_dtype, const bbx_tc_problem_t* problems, int count, int tile_n,
                       bbx_tc_plan_t** out);
int bbx_tc_plan_launch(bbx_tc_plan_t* plan, void* stream);
int bbx_tc_plan_destroy(bbx_tc_plan_t* plan);
/* The tile the plan runs (128, 256, or 512 = the 2-SM 256 x 256 pair); the
 * choice made for tile_n = 0. Returns 0 for a null plan. */
int bbx_tc_plan_tile_n(const bbx_tc_plan_t* plan);

/* ------------------------------------------------------------------ streaming ops */
/* c = a + b (dense_matrix_add.cc:67-73, dense_matrix_gpu_add.cu:47-55); c may alias a or b. */
int bbx_add_f32(const float* a, const float* b, float* c, long long n, void* stream);

/* out = in[0] + in[1] + ... + in[n_in-1], summed left to right as the reference's
 * local reduce folds matrix_add (local_reduce_op.cc:23-91), reading each input
 * once. kahan=1 adds Kahan compensation; kahan=0 is bit-identical to the
 * reference's fold. `inputs` is a HOST array of device pointers; out may alias
 * inputs[0]. Any n_in >= 1. */
int bbx_reduce_f32(const float* const* inputs, int n_in, float* out, long long n, int kahan,
                   void* stream);

int bbx_unary_f32(int op, const float* in, float* out, long long n, float param, void* stream);
int bbx_binary_f32(int op, const float* a, const float* b, float* c, long long n, float ca,
                   float cb, void* stream);

/* out[r][c] = in[r][c] + bias[c] (+relu): the bias step of ffnn_activation_mult.cc:88-94. */
int bbx_bias_add_f32(const float* in, const float* bias, float* out, int rows, int cols, int relu,
                     void* stream);
/* out[c] (+)= sum over rows of in[r][c], rows in order: the bias gradient of
 * ffnn_back_mult.cc:86-90 (with the output zero-initialised when accumulate=0). */
int bbx_colsum_f32(const float* in, float* out, int rows, int cols, long long ld, int accumulate,
                   void* stream);

/* Element-type conversion f32 <-> bf16. */
int bbx_cast(int src_dtype, const void* in, int dst_dtype, void* out, long long n, void* stream);
/* New (no reference counterpart): relu of an f32 block split into two bf16
 * blocks, hi = bf16(relu(z)) and lo = bf16(relu(z) - hi). A layer whose
 * activation feeds another ReLU layer multiplies both by the next weights, so
 * its tensor-core operand carries ~16 significant bits instead of 8 (ud
 * matrix_relu_split). */
int bbx_relu_split(const float* z, void* hi, void* lo, long long n, void* stream);

/* Per-block absmax FP8-E4M3 quantisation: out = e4m3(in * 448/absmax(in)),
 * *scale_out (device f32) = absmax/448. transpose=1 writes cols x rows. Uses a
 * library-owned device scratch word for the absmax. */
int bbx_quantize_e4m3(int src_dtype, const void* in, void* out, int rows, int cols, int transpose,
                      float* scale_out, void* stream);

/* bbx_quantize_e4m3 over `count` blocks of rows x cols (in / out HOST arrays
 * of device pointers, scales_out a device array of `count` floats): the same
 * bytes per block, with each pass one launch per 64 blocks. Takes a
 * stream-ordered scratch of one word per block. */
int bbx_quantize_e4m3_batched(int src_dtype, const void* const* in, void* const* out, int count, int rows, int cols,
                              int transpose, float* scales_out, void* stream);

/* Allocation-free batched variant of bbx_quantize_e4m3 (no counterpart in the
 * reference). For callers that must not allocate device memory while they
 * run -- code under a memory manager that owns all of the GPU, latency paths
 * where cudaMalloc would synchronise, fixed-footprint deployments. It
 * quantises `count` blocks (each rows x cols; in / out are HOST arrays of
 * device pointers, scales_out a device array of `count` floats) and calls no
 * cudaMalloc / cudaFree: its absmax scratch is a fixed 4 KiB __device__ array
 * of the library, so count is at most 1024 per call (larger counts fail with
 * BBX_ERR_INVALID; count 0 is a no-op). The first call on a device looks the
 * array up (cudaGetSymbolAddress) and caches its address for the process, so
 * make it before any stream capture, and do not call the function after
 * cudaDeviceReset on that device (the cached address belongs to the old
 * context). All calls on a device share that array: calls that overlap on the
 * GPU race. */
int bbx_quantize_e4m3_batched_noalloc(int src_dtype, const void* const* in, void* const* out, int count,
                                      int rows, int cols, int transpose, float* scales_out, void* stream);

/* Seeded counter-based fill (Philox4x32-10): dist 0 = U(a,b), 1 = N(a, b^2). */
int bbx_fill_philox(int dtype, void* out, long long n, unsigned long long seed, int dist, float a,
                    float b, void* stream);

/* Softmax cross-entropy per row against integer labels (new ud, no reference
 * counterpart): loss[r] = logsumexp(z_r) - z_r[y_r]; if grad != NULL,
 * grad = (softmax(z) - onehot(y)) * grad_scale. */
int bbx_softmax_ce_f32(const float* logits, const int* labels, float* loss, float* grad, int rows,
                       int cols, long long ld, float grad_scale, void* stream);
/* Same with the gradient written as BBX_F32 or BBX_BF16 (grad_dtype). */
int bbx_softmax_ce(const float* logits, const int* labels, float* loss, void* grad, int grad_dtype, int rows,
                   int cols, long long ld, float grad_scale, void* stream);

/* Rank<=4 permutation with optional cast: out[...] = in[...] where output dim d
 * is input dim perm[d]. Dims are listed outermost-first (row-major). dst_dtype
 * f32 or bf16. */
int bbx_permute(const float* in, int rank, const long long* in_dims, const int* perm,
                int dst_dtype, void* out, void* stream);

/* Grouped streaming ops: ONE launch runs a whole batch of independent
 * add / n-ary reduce / elementwise / cast block ops over f32 or bf16 payloads
 * (inputs read once, math in f32). Used per DAG level by the executor, in
 * place of one dense_add_kernel launch per op (dense_matrix_gpu_add.cu:74-81). */
#define BBX_S_SUM 0    /* out = in[0] + ... + in[n_in-1], left to right (kahan optional) */
#define BBX_S_UNARY 1  /* out = unary(op, in[0], p0) */
#define BBX_S_BINARY 2 /* out = binary(op, in[0], in[1], p0, p1) */
#define BBX_S_CAST 3   /* out = in[0] converted */
#define BBX_STREAM_MAX_IN 16
typedef struct bbx_stream_op {
  int kind, op, in_dtype, out_dtype, n_in, kahan;
  long long n;
  const void* in[BBX_STREAM_MAX_IN];
  void* out;
  float p0, p1;
} bbx_stream_op_t;
int bbx_stream_group(const bbx_stream_op_t* ops, int count, void* stream);
typedef struct bbx_stream_plan bbx_stream_plan_t;
int bbx_stream_plan_create(const bbx_stream_op_t* ops, int count, bbx_stream_plan_t** out);
int bbx_stream_plan_launch(bbx_stream_plan_t* plan, void* stream);
int bbx_stream_plan_destroy(bbx_stream_plan_t* plan);
/* Kernel choice of a plan: AUTO runs the bulk-staged kernel when every
 * pointer is 16-byte aligned (fastest alone, but its 196 KB of shared memory
 * leaves no room on an SM for a tensor-core CTA), REGISTER always runs the
 * register kernel (no shared memory: it shares SMs with a concurrent
 * tensor-core launch). */
#define BBX_STREAM_KERNEL_AUTO 0
#define BBX_STREAM_KERNEL_REGISTER 1
/* DAG builds only (bbx_rt_set_dag_stream_kernel): per wave, the register
 * kernel when the wave's predicted tensor-core time is at least its predicted
 * bulk streaming time (the streaming work then hides under the tensor work),
 * else AUTO. Tensor time comes from the runtime's tile model when one is
 * installed (bbx_rt_set_tile_predictor), else from the group's FLOPs. */
#define BBX_STREAM_KERNEL_PER_WAVE 2
int bbx_stream_plan_create_kernel(const bbx_stream_op_t* ops, int count, int kernel, bbx_stream_plan_t** out);
/* 1 when the plan runs the bulk-staged kernel (every pointer of every op
 * 16-byte aligned: inputs staged in shared memory by cp.async.bulk), 0 for
 * the register kernel, negative on error. */
int bbx_stream_plan_bulk(const bbx_stream_plan_t* plan);

/* einsum contraction of the reference's "cutensor" plugin
 * (libraries/cutensor/contraction.h:25-63 params, :131-202 semantics):
 * out = alpha * sum lhs * rhs over modes absent from the output. Tensors are
 * COLUMN-major with int64 dims (cu.h:65-169). precision = BBX_F32 (SIMT) or
 * BBX_BF16 (tensor cores, f32 accumulate). */
int bbx_contraction(const float* lhs, int rank_l, const long long* dims_l, const int* modes_l,
                    const float* rhs, int rank_r, const long long* dims_r, const int* modes_r,
                    float* out, int rank_o, const int* modes_o, float alpha, int precision,
                    void* stream);

/* The other block ops of the cutensor plugin, on column-major FP32 tensors of
 * rank <= 4 (dims listed mode 0 first):
 * reduction.h:13-21,42-111: out = alpha * fold(op: 0 add, 1 max, 2 min, 3 mul)
 *   over the modes not in `ordering`; output mode r = input mode ordering[r]. */
int bbx_cu_reduction(const float* in, int rank, const long long* dims, int op, float alpha, const int* ordering,
                     int rank_out, float* out, void* stream);
/* ew.h:13-21,131-190: out = permute(alpha * uop(in)), uop 0 e^v/(1+e^v), 1 exp,
 *   2 square, 3 max(v,0), 4 (v<0 ? 0 : 1), 5 sqrt, 6 v + scalar; output mode r =
 *   input mode ordering[r]. */
int bbx_cu_ew(const float* in, int rank, const long long* dims, int uop, float scalar, float alpha,
              const int* ordering, float* out, void* stream);
/* ewb.h:13-46,122-204: out[i] = op(alpha * lhs[i|lhs], beta * rhs[i|rhs]) with
 *   op 0 add, 1 max, 2 min, 3 mul, 4 sub, 5 div; lhs mode r is output mode
 *   ord_l[r] (likewise rhs), output modes absent from an input broadcast it.
 *   ewb_castable (ewb_castable.h:24-91) is the same-shape case with
 *   alpha = beta = 1. The output rank / dims are returned. */
int bbx_cu_ewb(const float* lhs, int rank_l, const long long* dims_l, const int* ord_l, const float* rhs,
               int rank_r, const long long* dims_r, const int* ord_r, int op, float alpha, float beta, float* out,
               int* rank_out, long long* dims_out, void* stream);
/* expand.h:1-110: params5 = per mode (sz_in, sz_out, num, start_in, start_out);
 *   out (sz_out...) = 0, then out[start_out + i] = in[start_in + i] for i < num. */
int bbx_cu_expand(const float* in, const int* params5, int rank, float* out, void* stream);

/* ------------------------------------------------------------------ runtime
 * A single-GPU runtime: the tensor factory + ud registry (with this library's
 * B200 impls registered through the reference's register_tensors /
 * register_udfs entry points), device-resident block storage, a command list,
 * the reservation station and the executors.
 * Tensor metas are the reference's 260-byte tensor_meta_t (4-byte format id +
 * 256-byte blob, src/tensor/tensor.h:20-34); the last 8 blob bytes carry the
 * payload's device address. */
typedef struct bbx_rt bbx_rt_t;
int bbx_rt_create(bbx_rt_t** out);
int bbx_rt_destroy(bbx_rt_t* rt);
/* stream every launch of this runtime is ordered on */
int bbx_rt_stream(bbx_rt_t* rt, void** stream_out);
/* tensor_factory_t::get_tensor_ftm (src/tensor/tensor_factory.cc:60-68); -1 if unknown */
int bbx_rt_fmt_id(bbx_rt_t* rt, const char* fmt_name);
/* udf_manager_t::get_matcher_for + udf_matcher::findMatch
 * (src/ud_functions/udf_manager.cc:10-37,114-125) with REAL type matching;
 * type lists are comma separated, e.g. "dense,dense". */
int bbx_rt_find_impl(bbx_rt_t* rt, const char* ud_name, const char* in_types, const char* out_types,
                     int require_gpu, int* ud_id, int* impl_id);
int bbx_rt_impl_name(bbx_rt_t* rt, int ud_id, int impl_id, char* buf, size_t len);
/* complexity hint of an impl on the given input metas (get_complexity_hint) */
int bbx_rt_complexity(bbx_rt_t* rt, int ud_id, int impl_id, const uint32_t* params, int n_params,
                      const void* in_metas, int n_in, unsigned long long* hint);
/* Creates / replaces tensor `tid` from a 260-byte meta and `bytes` of payload
 * (src on the host, or on the device when src_on_device). */
int bbx_rt_tensor_put(bbx_rt_t* rt, int tid, const void* meta, const void* src, size_t bytes,
                      int src_on_device);
/* Copies tensor `tid`'s meta (260 bytes) and up to `cap` payload bytes out. */
int bbx_rt_tensor_get(bbx_rt_t* rt, int tid, void* meta_out, void* dst, size_t cap, int dst_on_device);
/* Device address of tensor `tid`'s payload (copied back first if it was
 * spilled). The caller may read or write it with work queued on the runtime
 * stream; with a storage budget set the address stays valid until the next
 * call that creates, reloads or runs commands. */
int bbx_rt_tensor_payload(bbx_rt_t* rt, int tid, void** ptr, size_t* bytes);
/* Storage budget with spill (nvme_storage_t(com, max_allocated, file),
 * src/storage/nvme_storage.h:121-135; set_max_storage, nvme_storage.cc:270-280).
 * Resident block payloads stay within device_bytes: the least recently used
 * blocks no command holds are copied to pinned host memory (up to host_bytes)
 * and past that to `spill_file` (truncated here, removed when the runtime is
 * destroyed; NULL = no file tier), and copied back when a command reads them.
 * A single command needing more than device_bytes fails, as the reference's
 * "Can not process this." does. device_bytes 0 = no budget (every block is
 * brought back). The per-op path (bbx_rt_run) spills; a compiled DAG holds
 * every block resident while it lives. */
int bbx_rt_set_storage_budget(bbx_rt_t* rt, unsigned long long device_bytes, unsigned long long host_bytes,
                              const char* spill_file);
/* Spill counters since the budget was set, in this order: evictions, reloads,
 * D2H bytes, H2D bytes, file bytes written, file bytes read, evictions that
 * needed no copy (a valid copy existed), resident bytes, peak resident bytes,
 * pinned host bytes held by spilled copies. Writes min(n, 10) values. */
int bbx_rt_spill_stats(bbx_rt_t* rt, unsigned long long* out, int n);
int bbx_rt_tensor_count(bbx_rt_t* rt);
int bbx_rt_tensor_remove(bbx_rt_t* rt, int tid);
/* command_t::create_apply / create_reduce / create_delete (src/commands/command.h:228-457);
 * params are the raw 4-byte command_param_t words. Commands are appended to the
 * runtime's command list in increasing id order. */
int bbx_rt_queue_apply(bbx_rt_t* rt, int cmd_id, int ud_id, int impl_id, const uint32_t* params,
                       int n_params, const int* in_tids, int n_in, const int* out_tids, int n_out);
int bbx_rt_queue_reduce(bbx_rt_t* rt, int cmd_id, int ud_id, int impl_id, const uint32_t* params,
                        int n_params, const int* in_tids, int n_in, int out_tid);
int bbx_rt_queue_delete(bbx_rt_t* rt, int cmd_id, const int* tids, int n);
int bbx_rt_clear_commands(bbx_rt_t* rt);
int bbx_rt_num_commands(bbx_rt_t* rt);
/* Appends the commands of a program file, compiled for this single node:
 * .sbbts text compile sources (compile_source_file_t,
 * src/commands/command_compiler.h:977-1027, compiled as command_compiler_t
 * does with all placement on node 0) and .bbts binary parsed command lists
 * (parsed_command_list_t, src/commands/parsed_command.h:194-383, compiled as
 * command_loader_t does, command_loader.h:10-182). *n_added = commands added. */
int bbx_rt_load_sbbts(bbx_rt_t* rt, const char* path, int* n_added);
int bbx_rt_load_bbts(bbx_rt_t* rt, const char* path, int* n_added);
/* Writes the runtime's command list back out as a .bbts parsed command list. */
int bbx_rt_save_bbts(bbx_rt_t* rt, const char* path);
/* The per-op path: the command list runs through the reservation station
 * (LIFO, or learned priority with policy 1) with one stream-ordered launch per
 * command, like command_runner_t::local_command_runner
 * (src/commands/command_runner.cc:18-259). Synchronous. */
int bbx_rt_run(bbx_rt_t* rt, int policy);
/* Worker streams of the per-op path (1..16; default 1 = the plain path, one
 * stream). The reference runs ready commands on num_threads worker threads
 * (src/server/node.cc:67-69); here each worker is a stream and a command waits
 * only on the completion events of its inputs' producers. */
int bbx_rt_set_workers(bbx_rt_t* rt, int workers);
/* Same as bbx_rt_run on one stream, recording each command's (12 features,
 * latency in us, the ud's get_complexity_hint) as training data for the cost
 * model; any output pointer may be null; returns the record count in *n_out. */
int bbx_rt_record(bbx_rt_t* rt, int policy, float* features, float* latency_us, double* hints, int cap,
                  int* n_out);

#define BBX_SCHED_HEURISTIC 0
#define BBX_SCHED_LEARNED 1
/* The grouped path: lower the command list into waves of grouped launches with
 * a static arena, captured in one CUDA graph. No reference counterpart (the
 * reference issues one call per command). */
typedef struct bbx_dag bbx_dag_t;
/* tile_n: 128 or 256 forces the tcgen05 tile width, 0 picks it from the
 * shapes, -1 runs the autotuner (times both widths on each grouped launch's own
 * problems once per shape bucket; cached in the file named by $BBX_TUNE_CACHE). */
int bbx_dag_build(bbx_rt_t* rt, int policy, int tile_n, bbx_dag_t** out);
int bbx_dag_launch(bbx_dag_t* dag, void* stream);
int bbx_dag_destroy(bbx_dag_t* dag);
int bbx_dag_stats(bbx_dag_t* dag, double* flops, double* bytes, int* waves, int* tc_launches,
                  int* stream_launches, int* other_launches, size_t* arena_bytes);
/* Replays each launch group of the DAG on its own, one after another on
 * `stream`, and reports per group (up to cap): kind (0 contraction input
 * gathers, 1 grouped streaming ops, 2 ops called through their impls, 3
 * grouped tcgen05 GEMM, 4 contraction output gathers), wave, duration in ms and
 * the algorithmic FLOPs / bytes of the launch; *n_out = the group count.
 * Synchronous; results equal a graph replay's. cap <= 0 only counts the
 * groups and runs nothing. */
int bbx_dag_profile(bbx_dag_t* dag, void* stream, int cap, int* kinds, int* waves, float* ms, double* flops,
                    double* bytes, int* n_out);
/* device address and meta of a tensor the DAG reads or produces */
int bbx_dag_tensor(bbx_dag_t* dag, int tid, void** ptr, void* meta_out);
/* copies up to `cap` payload bytes of a DAG tensor to host memory (synchronous) */
int bbx_dag_read(bbx_dag_t* dag, int tid, void* host_dst, size_t cap);
/* Kernel of the grouped streaming launches of DAGs built afterwards on this
 * runtime (BBX_STREAM_KERNEL_AUTO, the default: the bulk-staged kernel where
 * aligned; BBX_STREAM_KERNEL_REGISTER: the register kernel, which can share
 * SMs with the wave's tensor-core launch on the other stream;
 * BBX_STREAM_KERNEL_PER_WAVE: chosen per wave from predicted times). */
int bbx_rt_set_dag_stream_kernel(bbx_rt_t* rt, int kernel);
/* Waves of the DAG whose streaming launches run the register kernel. */
int bbx_dag_register_waves(bbx_dag_t* dag);
/* Stream-ordered host <-> block copies around bbx_dag_launch, the DAG's
 * counterpart of the reference's per-command storage transactions
 * (src/commands/command_runner.cc:86-172 reads inputs / writes outputs through
 * the storage). bbx_dag_write overwrites `bytes` of an input block that the
 * DAG reads in place (a registered tensor no command of the DAG writes;
 * anything else is BBX_ERR_INVALID); bbx_dag_fetch copies up to `cap` bytes
 * of any DAG tensor out. Both only enqueue a cudaMemcpyAsync on `stream`:
 * with pinned host memory they overlap other work; the caller synchronises
 * before reading `dst` or reusing `src`. */
int bbx_dag_write(bbx_dag_t* dag, int tid, const void* src, size_t bytes, int src_on_device, void* stream);
int bbx_dag_fetch(bbx_dag_t* dag, int tid, void* dst, size_t cap, int dst_on_device, void* stream);
/* Tile of each launch group in profile order: 128 / 256 (1-SM tcgen05 width),
 * 512 (the 2-SM 256 x 256 pair) for tensor-core groups, 0 for the others.
 * Writes min(cap, groups) values; *n_out = the group count. */
int bbx_dag_group_tiles(bbx_dag_t* dag, int cap, int* tiles, int* n_out);

/* ------------------------------------------------------------------ learned cost model
 * MLP 12 -> 128 -> 128 -> 128 -> 1 (ReLU, FP32) predicting log latency from op
 * features; trained and evaluated on the GPU by this library's kernels. */
typedef struct bbx_mlp bbx_mlp_t;
#define BBX_MLP_IN 12
#define BBX_MLP_HIDDEN 128
int bbx_mlp_create(unsigned long long seed, bbx_mlp_t** out);
int bbx_mlp_destroy(bbx_mlp_t* mlp);
/* standardisation of the inputs (per-feature mean / std), applied inside */
int bbx_mlp_set_norm(bbx_mlp_t* mlp, const float* mean, const float* std);
/* Adam on MSE; x host (n x 12), y host (n) = log latency. Returns final loss. */
int bbx_mlp_train(bbx_mlp_t* mlp, const float* x, const float* y, int n, int epochs, int batch,
                  float lr, float* loss_out);
int bbx_mlp_predict(bbx_mlp_t* mlp, const float* x, int n, float* y_out);
/* loss and all gradients for one batch (for gradient checks); grads laid out
 * as W1,b1,W2,b2,W3,b3,W4,b4 (Wi row-major in x out) */
int bbx_mlp_loss_grad(bbx_mlp_t* mlp, const float* x, const float* y, int n, float* loss,
                      float* grads);
int bbx_mlp_num_params(void);
int bbx_mlp_get_params(bbx_mlp_t* mlp, float* out);
int bbx_mlp_set_params(bbx_mlp_t* mlp, const float* in);
/* install the MLP as the runtime's latency predictor (policy BBX_SCHED_LEARNED) */
int bbx_rt_set_predictor(bbx_rt_t* rt, bbx_mlp_t* mlp);
/* New (no reference counterpart): learned tile choice. While recording is on,
 * the DAG autotuner (bbx_dag_build with tile_n = -1) logs one sample per group
 * and candidate tile: 12 features of the grouped launch run with that tile
 * (tile one-hot 128/256/512, log2 problem count, FLOPs, largest m, largest n,
 * tiles, mean k, dtype, operand layouts) and its time in us. Turning it on
 * clears the samples; recording bypasses the tune cache. An MLP trained on
 * them and installed with bbx_rt_set_tile_predictor makes bbx_dag_build with
 * tile_n = -2 pick each group's tile of least predicted time, with no timing
 * launches (without a tile model, -2 is the size heuristic of tile_n = 0). */
int bbx_tile_record(int on);
int bbx_tile_samples(float* features, float* latency_us, int cap, int* n_out);
int bbx_rt_set_tile_predictor(bbx_rt_t* rt, bbx_mlp_t* mlp);
/* install the calibrated complexity-hint model exp(a * ln(max(hint, 1)) + b) us
 * as the predictor instead: the reference's get_complexity_hint, fit to
 * recorded latencies, driving the same list scheduling as the MLP. */
int bbx_rt_set_hint_predictor(bbx_rt_t* rt, double a, double b);

#ifdef __cplusplus
}
#endif
#endif /* BBTS_B200_H */
