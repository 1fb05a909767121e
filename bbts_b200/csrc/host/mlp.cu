// Learned cost model: MLP 12 -> 128 -> 128 -> 128 -> 1 with ReLU, FP32,
// predicting log(latency in us) of a block op from its 12 features.
// Forward and backward run on the GPU through this library's own kernels
// (SIMT FP32 GEMM with fused bias/ReLU epilogue, column sums) plus the small
// kernels below (input standardisation, MSE, ReLU backward, Adam).
#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <stdexcept>
#include <vector>
#include "bbts_b200.h"
#include "common.h"
#include "runtime.h"

namespace {

constexpr int IN = BBX_MLP_IN, H = BBX_MLP_HIDDEN;
// parameter layout: W1 (IN x H), b1 (H), W2 (H x H), b2, W3 (H x H), b3, W4 (H x 1), b4 (1)
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + IN * H, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
              OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + H * H, OFF_W4 = OFF_B3 + H, OFF_B4 = OFF_W4 + H,
              NPARAM = OFF_B4 + 1;

__global__ void k_standardize(const float* __restrict__ x, const float* __restrict__ mean,
                              const float* __restrict__ inv_std, float* out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n * IN) {
    int f = i % IN;
    out[i] = (x[i] - mean[f]) * inv_std[f];
  }
}

// dy = 2 (pred - y) / n ; loss_acc += sum (pred - y)^2 / n  (loss_acc is zeroed by the caller)
__global__ void k_mse(const float* __restrict__ pred, const float* __restrict__ y, float* dy,
                      float* loss_acc, int n) {
  float local = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float d = pred[i] - y[i];
    dy[i] = 2.f * d / n;
    local += d * d / n;
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss_acc, local);
}

// dh *= (h > 0): backward of ReLU given the post-activation h
__global__ void k_relu_bwd(float* dh, const float* __restrict__ h, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (!(h[i] > 0.f)) dh[i] = 0.f;
}

__global__ void k_adam(float* p, const float* __restrict__ g, float* m, float* v, int n, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    float gi = g[i];
    float mi = b1 * m[i] + (1.f - b1) * gi;
    float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

void ck(cudaError_t e, const char* w) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(w) + ": " + cudaGetErrorString(e));
}
void bk(int rc) {
  if (rc != 0) {
    char buf[1024];
    bbx_last_error(buf, sizeof(buf));
    throw std::runtime_error(buf);
  }
}

}  // namespace

struct bbx_mlp {
  cudaStream_t st = nullptr;
  float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
  float *mean = nullptr, *inv_std = nullptr, *loss = nullptr;
  int cap = 0;  // activation capacity (rows)
  float *x = nullptr, *xn = nullptr, *y = nullptr, *h1 = nullptr, *h2 = nullptr, *h3 = nullptr,
        *out = nullptr, *dout = nullptr, *d3 = nullptr, *d2 = nullptr, *d1 = nullptr;
  long long step = 0;

  void reserve(int n) {
    if (n <= cap) return;
    for (float* p : {x, xn, y, h1, h2, h3, out, dout, d3, d2, d1})
      if (p) cudaFree(p);
    cap = n;
    ck(cudaMalloc(&x, sizeof(float) * n * IN), "mlp alloc");
    ck(cudaMalloc(&xn, sizeof(float) * n * IN), "mlp alloc");
    ck(cudaMalloc(&y, sizeof(float) * n), "mlp alloc");
    ck(cudaMalloc(&h1, sizeof(float) * n * H), "mlp alloc");
    ck(cudaMalloc(&h2, sizeof(float) * n * H), "mlp alloc");
    ck(cudaMalloc(&h3, sizeof(float) * n * H), "mlp alloc");
    ck(cudaMalloc(&out, sizeof(float) * n), "mlp alloc");
    ck(cudaMalloc(&dout, sizeof(float) * n), "mlp alloc");
    ck(cudaMalloc(&d3, sizeof(float) * n * H), "mlp alloc");
    ck(cudaMalloc(&d2, sizeof(float) * n * H), "mlp alloc");
    ck(cudaMalloc(&d1, sizeof(float) * n * H), "mlp alloc");
  }

  // x (device, n x IN) -> out (device, n)
  void forward(const float* xdev, int n) {
    k_standardize<<<(n * IN + 255) / 256, 256, 0, st>>>(xdev, mean, inv_std, xn, n);
    bk(bbx_matmul_f32(xn, params + OFF_W1, h1, n, H, IN, IN, H, H, 0, 0, 1.f, 0.f, params + OFF_B1, 1, 1, 0, 0, 0, st));
    bk(bbx_matmul_f32(h1, params + OFF_W2, h2, n, H, H, H, H, H, 0, 0, 1.f, 0.f, params + OFF_B2, 1, 1, 0, 0, 0, st));
    bk(bbx_matmul_f32(h2, params + OFF_W3, h3, n, H, H, H, H, H, 0, 0, 1.f, 0.f, params + OFF_B3, 1, 1, 0, 0, 0, st));
    bk(bbx_matmul_f32(h3, params + OFF_W4, out, n, 1, H, H, 1, 1, 0, 0, 1.f, 0.f, params + OFF_B4, 0, 1, 0, 0, 0, st));
  }

  // after forward: loss (device scalar) and grads
  void backward(int n) {
    ck(cudaMemsetAsync(loss, 0, sizeof(float), st), "memset");
    k_mse<<<std::min((n + 255) / 256, 148), 256, 0, st>>>(out, y, dout, loss, n);
    // layer 4: dW4 = h3^T dout, db4 = sum dout, d3 = dout W4^T
    bk(bbx_matmul_f32(h3, dout, grads + OFF_W4, H, 1, n, H, 1, 1, 1, 0, 1.f, 0.f, nullptr, 0, 1, 0, 0, 0, st));
    bk(bbx_colsum_f32(dout, grads + OFF_B4, n, 1, 1, 0, st));
    bk(bbx_matmul_f32(dout, params + OFF_W4, d3, n, H, 1, 1, 1, H, 0, 1, 1.f, 0.f, nullptr, 0, 1, 0, 0, 0, st));
    k_relu_bwd<<<std::min((n * H + 255) / 256, 148 * 8), 256, 0, st>>>(d3, h3, (long long)n * H);
    // layer 3
    bk(bbx_matmul_f32(h2, d3, grads + OFF_W3, H, H, n, H, H, H, 1, 0, 1.f, 0.f, nullptr, 0, 1, 0, 0, 0, st));
    bk(bbx_colsum_f32(d3, grads + OFF_B3, n, H, H, 0, st));
    bk(bbx_matmul_f32(d3, params + OFF_W3, d2, n, H, H, H, H, H, 0, 1, 1.f, 0.f, nullptr, 0, 1, 0, 0, 0, st));
    k_relu_bwd<<<std::min((n * H + 255) / 256, 148 * 8), 256, 0, st>>>(d2, h2, (long long)n * H);
    // layer 2
    bk(bbx_matmul_f32(h1, d2, grads + OFF_W2, H, H, n, H, H, H, 1, 0, 1.f, 0.f, nullptr, 0, 1, 0, 0, 0, st));
    bk(bbx_colsum_f32(d2, grads + OFF_B2, n, H, H, 0, st));
    bk(bbx_matmul_f32(d2, params + OFF_W2, d1, n, H, H, H, H, H, 0, 1, 1.f, 0.f, nullptr, 0, 1, 0, 0, 0, st));
    k_relu_bwd<<<std::min((n * H + 255) / 256, 148 * 8), 256, 0, st>>>(d1, h1, (long long)n * H);
    // layer 1
    bk(bbx_matmul_f32(xn, d1, grads + OFF_W1, IN, H, n, IN, H, H, 1, 0, 1.f, 0.f, nullptr, 0, 1, 0, 0, 0, st));
    bk(bbx_colsum_f32(d1, grads + OFF_B1, n, H, H, 0, st));
  }

  void adam(float lr) {
    ++step;
    const float b1 = 0.9f, b2 = 0.999f;
    k_adam<<<(NPARAM + 255) / 256, 256, 0, st>>>(params, grads, m, v, NPARAM, lr, b1, b2, 1e-8f,
                                                  1.f - std::pow(b1, (float)step), 1.f - std::pow(b2, (float)step));
  }
};

extern "C" {

int bbx_mlp_num_params(void) { return NPARAM; }

int bbx_mlp_create(unsigned long long seed, bbx_mlp_t** out) {
  if (!out) return bbx::set_error(BBX_ERR_INVALID, "null out");
  try {
    auto* m = new bbx_mlp();
    ck(cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking), "mlp stream");
    ck(cudaMalloc(&m->params, sizeof(float) * NPARAM), "mlp alloc");
    ck(cudaMalloc(&m->grads, sizeof(float) * NPARAM), "mlp alloc");
    ck(cudaMalloc(&m->m, sizeof(float) * NPARAM), "mlp alloc");
    ck(cudaMalloc(&m->v, sizeof(float) * NPARAM), "mlp alloc");
    ck(cudaMalloc(&m->mean, sizeof(float) * IN), "mlp alloc");
    ck(cudaMalloc(&m->inv_std, sizeof(float) * IN), "mlp alloc");
    ck(cudaMalloc(&m->loss, sizeof(float)), "mlp alloc");
    ck(cudaMemset(m->m, 0, sizeof(float) * NPARAM), "memset");
    ck(cudaMemset(m->v, 0, sizeof(float) * NPARAM), "memset");
    // He-uniform weights, zero biases
    std::vector<float> p(NPARAM, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int fan_in, int count) {
      float lim = std::sqrt(6.f / fan_in);
      std::uniform_real_distribution<float> u(-lim, lim);
      for (int i = 0; i < count; ++i) p[off + i] = u(rng);
    };
    fill(OFF_W1, IN, IN * H);
    fill(OFF_W2, H, H * H);
    fill(OFF_W3, H, H * H);
    fill(OFF_W4, H, H);
    ck(cudaMemcpy(m->params, p.data(), sizeof(float) * NPARAM, cudaMemcpyHostToDevice), "upload");
    std::vector<float> zero(IN, 0.f), one(IN, 1.f);
    ck(cudaMemcpy(m->mean, zero.data(), sizeof(float) * IN, cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(m->inv_std, one.data(), sizeof(float) * IN, cudaMemcpyHostToDevice), "upload");
    *out = m;
    return BBX_OK;
  } catch (const std::exception& e) {
    return bbx::set_error(BBX_ERR_CUDA, "%s", e.what());
  }
}

int bbx_mlp_destroy(bbx_mlp_t* m) {
  if (!m) return BBX_OK;
  cudaStreamSynchronize(m->st);
  for (float* p : {m->params, m->grads, m->m, m->v, m->mean, m->inv_std, m->loss, m->x, m->xn, m->y, m->h1,
                   m->h2, m->h3, m->out, m->dout, m->d3, m->d2, m->d1})
    if (p) cudaFree(p);
  cudaStreamDestroy(m->st);
  delete m;
  return BBX_OK;
}

int bbx_mlp_set_norm(bbx_mlp_t* m, const float* mean, const float* stdv) {
  if (!m || !mean || !stdv) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  float inv[IN];
  for (int i = 0; i < IN; ++i) inv[i] = stdv[i] > 1e-12f ? 1.f / stdv[i] : 1.f;
  if (cudaMemcpy(m->mean, mean, sizeof(float) * IN, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(m->inv_std, inv, sizeof(float) * IN, cudaMemcpyHostToDevice) != cudaSuccess)
    return bbx::set_error(BBX_ERR_CUDA, "mlp norm upload");
  return BBX_OK;
}

int bbx_mlp_train(bbx_mlp_t* m, const float* x, const float* y, int n, int epochs, int batch, float lr,
                  float* loss_out) {
  if (!m || !x || !y || n <= 0 || epochs <= 0 || batch <= 0) return bbx::set_error(BBX_ERR_INVALID, "bad train arguments");
  try {
    batch = std::min(batch, n);
    m->reserve(n);
    float *dx = nullptr, *dy = nullptr;
    ck(cudaMalloc(&dx, sizeof(float) * n * IN), "train alloc");
    ck(cudaMalloc(&dy, sizeof(float) * n), "train alloc");
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::mt19937 rng(1234);
    std::vector<float> px((size_t)n * IN), py(n);
    float last = 0.f;
    for (int e = 0; e < epochs; ++e) {
      std::shuffle(perm.begin(), perm.end(), rng);
      for (int i = 0; i < n; ++i) {
        std::memcpy(&px[(size_t)i * IN], x + (size_t)perm[i] * IN, sizeof(float) * IN);
        py[i] = y[perm[i]];
      }
      ck(cudaMemcpyAsync(dx, px.data(), sizeof(float) * n * IN, cudaMemcpyHostToDevice, m->st), "upload");
      ck(cudaMemcpyAsync(dy, py.data(), sizeof(float) * n, cudaMemcpyHostToDevice, m->st), "upload");
      double tot = 0;
      int nb = 0;
      for (int s = 0; s + batch <= n; s += batch) {
        ck(cudaMemcpyAsync(m->y, dy + s, sizeof(float) * batch, cudaMemcpyDeviceToDevice, m->st), "copy");
        m->forward(dx + (size_t)s * IN, batch);
        m->backward(batch);
        m->adam(lr);
        if (s + 2 * batch > n) {  // last batch of the epoch: read the loss
          float l;
          ck(cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->st), "loss");
          ck(cudaStreamSynchronize(m->st), "sync");
          tot += l;
          ++nb;
        }
      }
      last = nb ? (float)(tot / nb) : 0.f;
    }
    ck(cudaStreamSynchronize(m->st), "sync");
    cudaFree(dx);
    cudaFree(dy);
    if (loss_out) *loss_out = last;
    return BBX_OK;
  } catch (const std::exception& e) {
    return bbx::set_error(BBX_ERR_CUDA, "%s", e.what());
  }
}

int bbx_mlp_predict(bbx_mlp_t* m, const float* x, int n, float* y_out) {
  if (!m || !x || !y_out || n < 0) return bbx::set_error(BBX_ERR_INVALID, "bad predict arguments");
  if (n == 0) return BBX_OK;
  try {
    m->reserve(n);
    ck(cudaMemcpyAsync(m->x, x, sizeof(float) * n * IN, cudaMemcpyHostToDevice, m->st), "upload");
    m->forward(m->x, n);
    ck(cudaMemcpyAsync(y_out, m->out, sizeof(float) * n, cudaMemcpyDeviceToHost, m->st), "download");
    ck(cudaStreamSynchronize(m->st), "sync");
    return BBX_OK;
  } catch (const std::exception& e) {
    return bbx::set_error(BBX_ERR_CUDA, "%s", e.what());
  }
}

int bbx_mlp_loss_grad(bbx_mlp_t* m, const float* x, const float* y, int n, float* loss, float* grads) {
  if (!m || !x || !y || n <= 0) return bbx::set_error(BBX_ERR_INVALID, "bad loss_grad arguments");
  try {
    m->reserve(n);
    ck(cudaMemcpyAsync(m->x, x, sizeof(float) * n * IN, cudaMemcpyHostToDevice, m->st), "upload");
    ck(cudaMemcpyAsync(m->y, y, sizeof(float) * n, cudaMemcpyHostToDevice, m->st), "upload");
    m->forward(m->x, n);
    m->backward(n);
    if (loss) ck(cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->st), "download");
    if (grads) ck(cudaMemcpyAsync(grads, m->grads, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, m->st), "download");
    ck(cudaStreamSynchronize(m->st), "sync");
    return BBX_OK;
  } catch (const std::exception& e) {
    return bbx::set_error(BBX_ERR_CUDA, "%s", e.what());
  }
}

int bbx_mlp_get_params(bbx_mlp_t* m, float* out) {
  if (!m || !out) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  if (cudaMemcpy(out, m->params, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost) != cudaSuccess)
    return bbx::set_error(BBX_ERR_CUDA, "params download");
  return BBX_OK;
}

int bbx_mlp_set_params(bbx_mlp_t* m, const float* in) {
  if (!m || !in) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  if (cudaMemcpy(m->params, in, sizeof(float) * NPARAM, cudaMemcpyHostToDevice) != cudaSuccess)
    return bbx::set_error(BBX_ERR_CUDA, "params upload");
  return BBX_OK;
}

}  // extern "C"

// Installs the MLP as the runtime's latency predictor: exp(predicted log latency).
struct bbx_rt;
namespace bbts {
runtime_t* rt_of(bbx_rt* rt);
}

extern "C" int bbx_rt_set_predictor(bbx_rt_t* rt, bbx_mlp_t* mlp) {
  if (!rt) return bbx::set_error(BBX_ERR_INVALID, "null runtime");
  bbts::runtime_t* r = bbts::rt_of(rt);
  if (!mlp) {
    r->predictor = nullptr;
    r->batch_predictor = nullptr;
    return BBX_OK;
  }
  r->batch_predictor = [mlp](const std::vector<bbts::op_features_t>& fs) {
    std::vector<float> x(fs.size() * IN), y(fs.size());
    for (size_t i = 0; i < fs.size(); ++i) std::memcpy(&x[i * IN], fs[i].f, sizeof(float) * IN);
    bk(bbx_mlp_predict(mlp, x.data(), (int)fs.size(), y.data()));
    std::vector<double> out(fs.size());
    for (size_t i = 0; i < fs.size(); ++i) out[i] = std::exp((double)y[i]);
    return out;
  };
  r->predictor = [r](const bbts::op_features_t& f) { return r->batch_predictor({f})[0]; };
  return BBX_OK;
}

// Installs an MLP trained on tile_features rows as the runtime's tile model
// (dag_build with tile_n = -2 picks the tile of least predicted time).
extern "C" int bbx_rt_set_tile_predictor(bbx_rt_t* rt, bbx_mlp_t* mlp) {
  if (!rt) return bbx::set_error(BBX_ERR_INVALID, "null runtime");
  bbts::runtime_t* r = bbts::rt_of(rt);
  if (!mlp) {
    r->tile_predictor = nullptr;
    return BBX_OK;
  }
  r->tile_predictor = [mlp](const std::vector<bbts::op_features_t>& fs) {
    std::vector<float> x(fs.size() * IN), y(fs.size());
    for (size_t i = 0; i < fs.size(); ++i) std::memcpy(&x[i * IN], fs[i].f, sizeof(float) * IN);
    bk(bbx_mlp_predict(mlp, x.data(), (int)fs.size(), y.data()));
    std::vector<double> out(fs.size());
    for (size_t i = 0; i < fs.size(); ++i) out[i] = std::exp((double)y[i]);
    return out;
  };
  return BBX_OK;
}

// The heuristic cost, calibrated: the ud's get_complexity_hint mapped to
// microseconds by a fit of log latency on log hint.
extern "C" int bbx_rt_set_hint_predictor(bbx_rt_t* rt, double a, double b) {
  if (!rt) return bbx::set_error(BBX_ERR_INVALID, "null runtime");
  if (!std::isfinite(a) || !std::isfinite(b)) return bbx::set_error(BBX_ERR_INVALID, "non-finite hint model");
  bbts::runtime_t* r = bbts::rt_of(rt);
  r->batch_predictor = [a, b](const std::vector<bbts::op_features_t>& fs) {
    std::vector<double> out(fs.size());
    for (size_t i = 0; i < fs.size(); ++i) out[i] = std::exp(a * std::log(std::max(1.0, fs[i].hint)) + b);
    return out;
  };
  r->predictor = [a, b](const bbts::op_features_t& f) { return std::exp(a * std::log(std::max(1.0, f.hint)) + b); };
  return BBX_OK;
}
