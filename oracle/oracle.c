/*
 * CPU oracle for the bbts_b200 block kernels -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library, and only as the checker / the timed CPU reference. The product
 * library never links or calls it.
 *
 * Each function restates the semantics of one reference CPU ud kernel of
 * dcbdan/bbts (file:line given per function) in plain C. The reference itself
 * cannot be compiled here: every ud includes <cutensor.h> via
 * src/ud_functions/ud_function.h:8 and the matmuls need Intel MKL
 * (dense_matrix_mult.cc:3-4), neither of which is available, so this is a
 * restatement, pinned against the reference's own known-answer add test
 * (tests/test_builtin_ud.cc:32-71) and self-evident known-answer cases.
 *
 * FP32 functions evaluate in IEEE single precision with no contraction of
 * multiply-adds (compiled with -ffp-contract=off) in the order the reference
 * loops use; *_f64 functions are the FP64 oracles.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------ elementwise */

/* dense_matrix_add.cc:67-73 */
void oracle_add(const float* a, const float* b, float* c, int64_t n) {
  for (int64_t i = 0; i < n; ++i) c[i] = a[i] + b[i];
}

/* local_reduce_op.cc:23-91: lhs = ud(lhs, in[i]) for i = 1..n-1 (left fold of
 * matrix_add), each step a fresh fp32 result. */
void oracle_reduce_fold(const float* const* in, int n_in, float* out, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    float s = in[0][i];
    for (int j = 1; j < n_in; ++j) s = s + in[j][i];
    out[i] = s;
  }
}

/* FP64 sum of the inputs (the reduce's FP64 oracle). */
void oracle_reduce_f64(const float* const* in, int n_in, double* out, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    double s = 0.0;
    for (int j = 0; j < n_in; ++j) s += (double)in[j][i];
    out[i] = s;
  }
}

/* op codes follow include/bbts_b200.h BBX_U_* */
void oracle_unary(int op, const float* in, float* out, int64_t n, float p) {
  for (int64_t i = 0; i < n; ++i) {
    float v = in[i], r = v;
    switch (op) {
      case 0: r = v > 0 ? v : 0; break;                       /* dense_matrix_relu.cc:63-69 */
      case 1: r = v > 0 ? 1.0f : 0; break;                    /* dense_matrix_relu_dif.cc:63-69 */
      case 2: r = 1 / (1.0f + expf(v)); break;                /* dense_matrix_sigmoid.cc:64-70 */
      case 3: r = 1 / (1.0f + expf(-v)); break;               /* cutensor ew.h:158-161 */
      case 4: r = expf(v); break;
      case 5: r = v * v; break;
      case 6: r = sqrtf(v); break;
      case 7: r = v + p; break;
      case 8: r = v * p; break;
    }
    out[i] = r;
  }
}

/* op codes follow BBX_B_*; weighted sum = dense_matrix_weighted_sum.cc:70-76,
 * hadamard = dense_matrix_hadamard.cc:67-73 */
void oracle_binary(int op, const float* a, const float* b, float* c, int64_t n, float ca,
                   float cb) {
  for (int64_t i = 0; i < n; ++i) {
    float x = a[i], y = b[i], r = x;
    switch (op) {
      case 0: r = x + y; break;
      case 1: { float t1 = ca * x; float t2 = cb * y; r = t1 + t2; } break;
      case 2: r = x * y; break;
      case 3: r = x > y ? x : y; break;
      case 4: r = x < y ? x : y; break;
      case 5: r = x - y; break;
      case 6: r = x / y; break;
    }
    c[i] = r;
  }
}

/* ffnn_activation_mult.cc:88-94: out[r][c] = in[r][c] + bias[c] */
void oracle_bias_add(const float* in, const float* bias, float* out, int rows, int cols, int relu) {
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c) {
      float v = in[(int64_t)r * cols + c] + bias[c];
      out[(int64_t)r * cols + c] = (relu && v < 0) ? 0 : v;
    }
}

/* ffnn_back_mult.cc:86-90: bias[c] += b[r][c] over rows in order (the
 * reference starts from uninitialised memory; the oracle starts from zero or
 * from the given values when accumulate != 0). */
void oracle_colsum(const float* in, float* out, int rows, int cols, int64_t ld, int accumulate) {
  for (int c = 0; c < cols; ++c) {
    float s = accumulate ? out[c] : 0.0f;
    for (int r = 0; r < rows; ++r) s = s + in[(int64_t)r * ld + c];
    out[c] = s;
  }
}

/* Softmax cross-entropy (new ud; no reference counterpart), FP64. */
void oracle_softmax_ce_f64(const float* z, const int* y, double* loss, double* grad, int rows,
                           int cols, int64_t ld, double grad_scale) {
  for (int r = 0; r < rows; ++r) {
    const float* zr = z + (int64_t)r * ld;
    double mx = -INFINITY;
    for (int c = 0; c < cols; ++c) mx = zr[c] > mx ? zr[c] : mx;
    double se = 0;
    for (int c = 0; c < cols; ++c) se += exp((double)zr[c] - mx);
    loss[r] = mx + log(se) - zr[y[r]];
    if (grad)
      for (int c = 0; c < cols; ++c)
        grad[(int64_t)r * ld + c] = (exp((double)zr[c] - mx) / se - (c == y[r] ? 1.0 : 0.0)) * grad_scale;
  }
}

/* ------------------------------------------------------------ matmul */

/* dense_matrix_mult.cc:78-82: cblas_sgemm(RowMajor, tA, tB, I, J, K, 1, A, lda,
 * B, ldb, 0, C, ldc) -- C = op(A) op(B), FP64 accumulation of FP32 inputs. */
void oracle_matmul_f64(const float* A, const float* B, double* C, int M, int N, int K,
                       int64_t lda, int64_t ldb, int64_t ldc, int ta, int tb) {
  double* row = (double*)malloc(sizeof(double) * (size_t)N);
  for (int i = 0; i < M; ++i) {
    for (int j = 0; j < N; ++j) row[j] = 0.0;
    for (int k = 0; k < K; ++k) {
      double a = ta ? A[(int64_t)k * lda + i] : A[(int64_t)i * lda + k];
      if (!tb) {
        const float* br = B + (int64_t)k * ldb;
        for (int j = 0; j < N; ++j) row[j] += a * (double)br[j];
      } else {
        for (int j = 0; j < N; ++j) row[j] += a * (double)B[(int64_t)j * ldb + k];
      }
    }
    for (int j = 0; j < N; ++j) C[(int64_t)i * ldc + j] = row[j];
  }
  free(row);
}

/* FP32 blocked, multithreaded restatement of the same SGEMM: the timed CPU
 * path of the reference's dense_matrix_mult (MKL is not available here, so
 * this is the project's own blocked loop; results agree with any FP32 SGEMM to
 * FP32 rounding, not bitwise). Row panels of C are split over `threads`. */
typedef struct {
  const float *A, *B;
  float* C;
  int M, N, K, ta, tb, r0, r1;
  int64_t lda, ldb, ldc;
} sgemm_job_t;

/* Register-blocked worker: a 6 x 32 tile of C stays in registers over a
 * k-block (packed A rows, packed and zero-padded B panel). Every element
 * accumulates its products one k after another. The tile uses fused
 * multiply-adds (the file is otherwise built without contraction), as an
 * optimised SGEMM such as the reference's MKL call does; results agree with
 * any FP32 SGEMM to FP32 rounding, and exactly on integer-valued inputs. */
enum { SG_MR = 6, SG_NR = 32, SG_KB = 256, SG_NB = 512 };

__attribute__((optimize("fp-contract=fast")))
static void sgemm_tile(int kb, const float* ap, const float* bp, float* c, int64_t ldc, int mr, int nr) {
  float acc[SG_MR][SG_NR];
  if (mr == SG_MR && nr == SG_NR) {
    for (int r = 0; r < SG_MR; ++r)
      for (int x = 0; x < SG_NR; ++x) acc[r][x] = c[r * ldc + x];
  } else {
    for (int r = 0; r < SG_MR; ++r)
      for (int x = 0; x < SG_NR; ++x) acc[r][x] = (r < mr && x < nr) ? c[r * ldc + x] : 0.0f;
  }
  for (int k = 0; k < kb; ++k) {
    const float* b = bp + (int64_t)k * SG_NB;
    const float* a = ap + k * SG_MR;
    for (int r = 0; r < SG_MR; ++r)
      for (int x = 0; x < SG_NR; ++x) acc[r][x] += a[r] * b[x];
  }
  for (int r = 0; r < mr; ++r)
    for (int x = 0; x < nr; ++x) c[r * ldc + x] = acc[r][x];
}

static void* sgemm_worker(void* arg) {
  sgemm_job_t* j = (sgemm_job_t*)arg;
  float* bpanel = (float*)aligned_alloc(64, sizeof(float) * (size_t)SG_KB * SG_NB);
  float* apanel = (float*)aligned_alloc(64, sizeof(float) * (size_t)SG_KB * SG_MR);
  for (int i = j->r0; i < j->r1; ++i)
    for (int c = 0; c < j->N; ++c) j->C[(int64_t)i * j->ldc + c] = 0.0f;
  for (int k0 = 0; k0 < j->K; k0 += SG_KB) {
    const int kb = j->K - k0 < SG_KB ? j->K - k0 : SG_KB;
    for (int n0 = 0; n0 < j->N; n0 += SG_NB) {
      const int nb = j->N - n0 < SG_NB ? j->N - n0 : SG_NB;
      const int nbp = (nb + SG_NR - 1) / SG_NR * SG_NR;  // padded to whole tiles with zeros
      for (int k = 0; k < kb; ++k)
        for (int c = 0; c < nbp; ++c)
          bpanel[k * SG_NB + c] = c >= nb ? 0.0f
                                  : j->tb ? j->B[(int64_t)(n0 + c) * j->ldb + k0 + k]
                                          : j->B[(int64_t)(k0 + k) * j->ldb + n0 + c];
      for (int i0 = j->r0; i0 < j->r1; i0 += SG_MR) {
        const int mr = j->r1 - i0 < SG_MR ? j->r1 - i0 : SG_MR;
        for (int k = 0; k < kb; ++k)
          for (int r = 0; r < SG_MR; ++r) {
            const int i = i0 + r;
            apanel[k * SG_MR + r] = r >= mr ? 0.0f
                                    : j->ta ? j->A[(int64_t)(k0 + k) * j->lda + i]
                                            : j->A[(int64_t)i * j->lda + k0 + k];
          }
        for (int x0 = 0; x0 < nb; x0 += SG_NR) {
          const int nr = nb - x0 < SG_NR ? nb - x0 : SG_NR;
          sgemm_tile(kb, apanel, bpanel + x0, j->C + (int64_t)i0 * j->ldc + n0 + x0, j->ldc, mr, nr);
        }
      }
    }
  }
  free(apanel);
  free(bpanel);
  return 0;
}

void oracle_sgemm_mt(const float* A, const float* B, float* C, int M, int N, int K, int64_t lda,
                     int64_t ldb, int64_t ldc, int ta, int tb, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  pthread_t th[256];
  sgemm_job_t jobs[256];
  int per = (M + threads - 1) / threads;
  int used = 0;
  for (int t = 0; t < threads; ++t) {
    int r0 = t * per, r1 = r0 + per > M ? M : r0 + per;
    if (r0 >= r1) break;
    jobs[t] = (sgemm_job_t){A, B, C, M, N, K, ta, tb, r0, r1, lda, ldb, ldc};
    pthread_create(&th[t], 0, sgemm_worker, &jobs[t]);
    ++used;
  }
  for (int t = 0; t < used; ++t) pthread_join(th[t], 0);
}

/* ------------------------------------------------------------ contraction */

/* libraries/cutensor/contraction.h:131-202 (`reference`): for every index over
 * all incident modes, out[o] += lhs[l] * rhs[r]; then out *= alpha. Tensors are
 * column-major (libraries/cutensor/utils.h get_offset: stride 1 on dim 0).
 * FP64 accumulation. Mode ids index the incident dims (contraction.h:25-55). */
void oracle_contraction_f64(const float* lhs, int rank_l, const int64_t* dims_l, const int* modes_l,
                            const float* rhs, int rank_r, const int64_t* dims_r, const int* modes_r,
                            double* out, int rank_o, const int* modes_o, double alpha) {
  int64_t ext[16];
  int nm = 0;
  for (int i = 0; i < 16; ++i) ext[i] = 1;
  for (int d = 0; d < rank_l; ++d) { ext[modes_l[d]] = dims_l[d]; if (modes_l[d] + 1 > nm) nm = modes_l[d] + 1; }
  for (int d = 0; d < rank_r; ++d) { ext[modes_r[d]] = dims_r[d]; if (modes_r[d] + 1 > nm) nm = modes_r[d] + 1; }
  int64_t total = 1, nout = 1;
  for (int m = 0; m < nm; ++m) total *= ext[m];
  for (int d = 0; d < rank_o; ++d) nout *= ext[modes_o[d]];
  for (int64_t i = 0; i < nout; ++i) out[i] = 0.0;
  int64_t idx[16];
  for (int64_t e = 0; e < total; ++e) {
    int64_t r = e;
    for (int m = 0; m < nm; ++m) { idx[m] = r % ext[m]; r /= ext[m]; }
    int64_t ol = 0, orr = 0, oo = 0, s;
    s = 1; for (int d = 0; d < rank_l; ++d) { ol += idx[modes_l[d]] * s; s *= dims_l[d]; }
    s = 1; for (int d = 0; d < rank_r; ++d) { orr += idx[modes_r[d]] * s; s *= dims_r[d]; }
    s = 1; for (int d = 0; d < rank_o; ++d) { oo += idx[modes_o[d]] * s; s *= ext[modes_o[d]]; }
    out[oo] += (double)lhs[ol] * (double)rhs[orr];
  }
  for (int64_t i = 0; i < nout; ++i) out[i] *= alpha;
}

/* ------------------------------------------------------------ generator */

/* Philox4x32-10 (Salmon et al., SC 2011), the same counter/key convention as
 * the device fill: counter (g_lo, g_hi, 0, 0), key (seed_lo, seed_hi). Writes
 * 4 words per group for groups [0, ngroups). */
void oracle_philox(uint64_t seed, int64_t ngroups, uint32_t* out) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int64_t g = 0; g < ngroups; ++g) {
    uint32_t c0 = (uint32_t)g, c1 = (uint32_t)((uint64_t)g >> 32), c2 = 0, c3 = 0;
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (int r = 0; r < 10; ++r) {
      uint64_t p0 = (uint64_t)M0 * c0, p1 = (uint64_t)M1 * c2;
      uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n1 = (uint32_t)p1;
      uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1, n3 = (uint32_t)p0;
      c0 = n0; c1 = n1; c2 = n2; c3 = n3;
      k0 += W0; k1 += W1;
    }
    out[4 * g + 0] = c0; out[4 * g + 1] = c1; out[4 * g + 2] = c2; out[4 * g + 3] = c3;
  }
}

/* U(lo,hi) from the top 24 bits of each Philox word: the device fill's
 * uniform mapping, which is exact in FP32 (no transcendental involved). */
void oracle_uniform(uint64_t seed, int64_t n, float lo, float hi, float* out) {
  int64_t groups = (n + 3) / 4;
  uint32_t* w = (uint32_t*)malloc(sizeof(uint32_t) * 4 * (size_t)groups);
  oracle_philox(seed, groups, w);
  for (int64_t i = 0; i < n; ++i) out[i] = fmaf(hi - lo, (float)(w[i] >> 8) * (1.0f / 16777216.0f), lo);
  free(w);
}
