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

/* ------------------------------------------------------------------ misc */
const char* bbx_version(void);
/* Copies the calling thread's last error message into buf; returns its length. */
int bbx_last_error(char* buf, size_t len);
/* Number of SMs of the current device (grids are sized to multiples of it). */
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

/* Per-block absmax FP8-E4M3 quantisation: out = e4m3(in * 448/absmax(in)),
 * *scale_out (device f32) = absmax/448. transpose=1 writes cols x rows. Uses a
 * library-owned device scratch word for the absmax. */
int bbx_quantize_e4m3(int src_dtype, const void* in, void* out, int rows, int cols, int transpose,
                      float* scale_out, void* stream);

/* Seeded counter-based fill (Philox4x32-10): dist 0 = U(a,b), 1 = N(a, b^2). */
int bbx_fill_philox(int dtype, void* out, long long n, unsigned long long seed, int dist, float a,
                    float b, void* stream);

/* Softmax cross-entropy per row against integer labels (new ud, no reference
 * counterpart): loss[r] = logsumexp(z_r) - z_r[y_r]; if grad != NULL,
 * grad = (softmax(z) - onehot(y)) * grad_scale. */
int bbx_softmax_ce_f32(const float* logits, const int* labels, float* loss, float* grad, int rows,
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

/* einsum contraction of the reference's "cutensor" plugin
 * (libraries/cutensor/contraction.h:25-63 params, :131-202 semantics):
 * out = alpha * sum lhs * rhs over modes absent from the output. Tensors are
 * COLUMN-major with int64 dims (cu.h:65-169). precision = BBX_F32 (SIMT) or
 * BBX_BF16 (tensor cores, f32 accumulate). */
int bbx_contraction(const float* lhs, int rank_l, const long long* dims_l, const int* modes_l,
                    const float* rhs, int rank_r, const long long* dims_r, const int* modes_r,
                    float* out, int rank_o, const int* modes_o, float alpha, int precision,
                    void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BBTS_B200_H */
