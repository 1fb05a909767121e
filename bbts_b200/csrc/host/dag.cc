// Grouped DAG executor.
//
// A compiled command list (APPLY / REDUCE / DELETE) is lowered once into
// waves. Every wave issues at most: the grouped streaming launches of its
// add / reduce / elementwise nodes, one grouped tcgen05 launch per operand
// layout class of its block matmuls, and direct calls of the remaining impls
// (FP32 SIMT matmul, contraction, FNN ops). Intermediate blocks live in one
// arena whose offsets come from a lifetime-based first-fit plan, and the whole
// launch sequence is captured into one CUDA graph that dag_launch replays.
//
// Scheduling policies (what the learned cost model changes):
//   heuristic  waves = ASAP levels; matmul tiles in reservation-station LIFO
//              order; costs = the ud's complexity hint.
//   learned    nodes get the MLP's predicted latency; a node with slack is
//              placed in the wave (within [ASAP, ALAP]) with the least
//              predicted load, and each grouped launch orders its problems by
//              predicted cost, longest first.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include "runtime.h"

namespace bbts {

namespace {

void dag_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
void dag_bbx(int rc) {
  if (rc != 0) {
    char buf[1024];
    bbx_last_error(buf, sizeof(buf));
    throw std::runtime_error(std::string("bbts_b200 DAG: ") + buf);
  }
}

struct node_t {
  const command_t* cmd;
  ud_impl_t* impl;
  node_kind_t kind;
  std::vector<tid_t> ins, outs;
  int asap = 0, height = 0, wave = 0;
  double cost = 1.0, flops = 0.0, bytes = 0.0;
  std::vector<int> preds, succs;
};

struct tplan_t {
  tensor_meta_t meta;
  size_t bytes = 0;
  int def = -1, last = -1;
  bool external = false, deleted = false;
  void* payload = nullptr;
};

struct opaque_t {
  ud_impl_t* impl;
  std::vector<command_param_t> params;
  std::vector<tid_t> ins, outs;
  bool reduce = false;
};

struct wave_t {
  std::vector<bbx_stream_plan_t*> phases;  // in order
  std::vector<bbx_tc_plan_t*> tc;
  std::vector<opaque_t> opaque;
};

}  // namespace

struct dag_t {
  runtime_t* rt = nullptr;
  std::vector<wave_t> waves;
  std::unordered_map<tid_t, tplan_t> tensors;
  std::unordered_map<tid_t, std::unique_ptr<char[]>> headers;
  void* arena = nullptr;
  size_t arena_bytes = 0;
  std::vector<void*> persistent;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  dag_stats_t stats{};
};

namespace {

tensor_t* header(dag_t* d, tid_t tid) {
  auto it = d->headers.find(tid);
  if (it != d->headers.end()) return (tensor_t*)it->second.get();
  auto& tp = d->tensors.at(tid);
  std::unique_ptr<char[]> h(new char[sizeof(tensor_meta_t)]);
  std::memcpy(h.get(), &tp.meta, sizeof(tensor_meta_t));
  ((tensor_t*)h.get())->_meta.set_payload(tp.payload);
  tensor_t* t = (tensor_t*)h.get();
  d->headers[tid] = std::move(h);
  return t;
}

void run_opaque(dag_t* d, opaque_t& o, cudaStream_t st) {
  ud_impl_t::tensor_params_t params;
  params._params = command_param_list_t{o.params.data(), o.params.size()};
  params.stream = st;
  std::vector<tensor_t*> ins, outs;
  for (tid_t t : o.ins) ins.push_back(header(d, t));
  for (tid_t t : o.outs) outs.push_back(header(d, t));
  ud_impl_t::tensor_args_t ia(ins), oa(outs);
  o.impl->call_ud(params, ia, oa);
}

// ---------------------------------------------------------------- tile autotuner
// Picks the tcgen05 tile width (BN = 128 or 256) of a grouped launch by timing
// both on the group's own problems, once per shape bucket. Buckets: input
// dtype, operand layouts, problem count and log2 of the group's FLOPs, of its
// largest n and of its largest m. Results persist in a text file when the
// BBX_TUNE_CACHE environment variable names one ("key tile_n" lines).
std::mutex g_tune_mu;
std::map<std::string, int> g_tune;
bool g_tune_loaded = false;

std::string tune_key(int dtype, bool ta, bool tb, const std::vector<bbx_tc_problem_t>& ps) {
  double fl = 0;
  int maxn = 0, maxm = 0;
  for (auto& q : ps) {
    fl += 2.0 * q.m * q.n * (double)q.k;
    maxn = std::max(maxn, q.n);
    maxm = std::max(maxm, q.m);
  }
  char buf[128];
  std::snprintf(buf, sizeof(buf), "d%d_a%d_b%d_p%d_f%d_n%d_m%d", dtype, (int)ta, (int)tb,
                (int)std::ceil(std::log2((double)ps.size() + 1)), (int)std::log2(fl + 1), (int)std::log2(maxn + 1),
                (int)std::log2(maxm + 1));
  return buf;
}

int autotune_tile_n(int dtype, bool ta, bool tb, const std::vector<bbx_tc_problem_t>& ps) {
  const std::string key = tune_key(dtype, ta, tb, ps);
  const char* path = std::getenv("BBX_TUNE_CACHE");
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (!g_tune_loaded && path) {
      FILE* f = std::fopen(path, "r");
      if (f) {
        char k[128];
        int v;
        while (std::fscanf(f, "%127s %d", k, &v) == 2) g_tune[k] = v;
        std::fclose(f);
      }
      g_tune_loaded = true;
    }
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second;
  }
  cudaStream_t st;
  dag_cuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "tune stream");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best = 256;
  float best_ms = 1e30f;
  for (int tn : {256, 128}) {
    bbx_tc_plan_t* p = nullptr;
    if (bbx_tc_plan_create(dtype == ELEM_E4M3 ? BBX_E4M3 : BBX_BF16, ps.data(), (int)ps.size(), tn, &p) != 0) continue;
    dag_bbx(bbx_tc_plan_launch(p, st));  // warm-up
    cudaEventRecord(e0, st);
    for (int r = 0; r < 3; ++r) dag_bbx(bbx_tc_plan_launch(p, st));
    cudaEventRecord(e1, st);
    dag_cuda(cudaEventSynchronize(e1), "tune sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    bbx_tc_plan_destroy(p);
    if (ms < best_ms) { best_ms = ms; best = tn; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best;
  if (path) {
    FILE* f = std::fopen(path, "a");
    if (f) {
      std::fprintf(f, "%s %d\n", key.c_str(), best);
      std::fclose(f);
    }
  }
  return best;
}

void issue(dag_t* d, cudaStream_t st) {
  for (auto& w : d->waves) {
    for (auto* p : w.phases) dag_bbx(bbx_stream_plan_launch(p, st));
    for (auto* p : w.tc) dag_bbx(bbx_tc_plan_launch(p, st));
    for (auto& o : w.opaque) run_opaque(d, o, st);
  }
}

}  // namespace

dag_t* dag_build(runtime_t* rt, int policy, int tile_n) {
  auto d = std::make_unique<dag_t>();
  d->rt = rt;
  const tensor_factory_t& tf = *rt->tf;

  // ---- tensors that already exist (registered inputs)
  for (tid_t t : rt->storage->tids()) {
    tplan_t tp;
    tp.meta = rt->storage->get(t)->_meta;
    tp.external = true;
    tp.payload = tp.meta.payload();
    tp.bytes = tf.get_payload_size(tp.meta);
    d->tensors[t] = tp;
  }

  // ---- nodes, output metas, dependencies
  std::vector<node_t> nodes;
  std::vector<op_features_t> feats;
  std::unordered_map<tid_t, int> producer;
  for (const auto& cp : rt->commands) {
    const command_t& c = *cp;
    if (c.is_delete()) {
      for (size_t i = 0; i < c.get_num_inputs(); ++i) {
        auto it = d->tensors.find(c.get_input(i).tid);
        if (it != d->tensors.end() && !it->second.external) it->second.deleted = true;
      }
      continue;
    }
    if (!c.is_apply() && !c.is_reduce()) throw std::runtime_error("DAG: only APPLY / REDUCE / DELETE on one node");
    node_t n;
    n.cmd = &c;
    n.impl = rt->udm->get_fn_impl(c.fun_id);
    if (!n.impl) throw std::runtime_error("DAG: command " + std::to_string(c.id) + " names an unknown ud impl");
    n.kind = classify(n.impl, c.is_reduce());
    if (c.is_reduce() && n.kind != NK_SUM)
      throw std::runtime_error("DAG: REDUCE is supported for matrix_add over dense / dense_bf16 blocks");
    std::vector<tensor_meta_t> in_metas;
    for (size_t i = 0; i < c.get_num_inputs(); ++i) {
      tid_t t = c.get_input(i).tid;
      auto it = d->tensors.find(t);
      if (it == d->tensors.end()) throw std::runtime_error("DAG: command " + std::to_string(c.id) + " reads tensor " + std::to_string(t) + " that nothing creates");
      in_metas.push_back(it->second.meta);
      n.ins.push_back(t);
      auto pit = producer.find(t);
      if (pit != producer.end()) n.preds.push_back(pit->second);
    }
    std::vector<tensor_meta_t> out_metas(c.get_num_outputs());
    for (auto& m : out_metas) std::memset(&m, 0, sizeof(m));
    ud_impl_t::tensor_params_t params;
    params._params = c.get_parameters();
    if (c.is_apply()) {
      ud_impl_t::meta_args_t im(in_metas), om(out_metas);
      n.impl->get_out_meta(params, im, om);
      for (size_t i = 0; i < out_metas.size(); ++i) out_metas[i].fmt_id = tf.get_tensor_ftm(n.impl->outputTypes[i]);
    } else {
      out_metas[0] = in_metas[0];
    }
    size_t hint = 0;
    feats.push_back(features_of(tf, c, n.impl, in_metas, &hint));
    n.cost = (double)std::max<size_t>(1, hint);
    const int idx = (int)nodes.size();
    for (size_t i = 0; i < c.get_num_outputs(); ++i) {
      tid_t t = c.get_output(i).tid;
      tplan_t tp;
      tp.meta = out_metas[i];
      tp.bytes = tf.get_payload_size(out_metas[i]);
      d->tensors[t] = tp;
      producer[t] = idx;
      n.outs.push_back(t);
    }
    // algorithmic work
    if (n.kind == NK_TC || n.kind == NK_SIMT) {
      const auto& ma = in_metas[0].as<dense_tensor_meta_t>().m();
      const auto& mb = in_metas[1].as<dense_tensor_meta_t>().m();
      bool ta = params.get_bool_or_default<0>(false), tb = params.get_bool_or_default<1>(false);
      double M = ta ? ma.num_cols : ma.num_rows, K = ta ? ma.num_rows : ma.num_cols, N = tb ? mb.num_rows : mb.num_cols;
      n.flops = 2.0 * M * N * K;
      n.bytes = (double)tf.get_payload_size(in_metas[0]) + tf.get_payload_size(in_metas[1]) + tf.get_payload_size(out_metas[0]);
    } else if (n.kind == NK_CONTRACT) {
      n.flops = 2.0 * (double)hint;
    } else {
      double b = 0;
      for (auto& m : in_metas) b += (double)tf.get_payload_size(m);
      for (auto& m : out_metas) b += (double)tf.get_payload_size(m);
      n.bytes = b;
    }
    nodes.push_back(std::move(n));
  }
  const int N = (int)nodes.size();
  if (policy == SCHED_LEARNED && rt->batch_predictor && N > 0) {
    std::vector<double> pred = rt->batch_predictor(feats);  // one batched GPU inference
    for (int i = 0; i < N; ++i) nodes[i].cost = pred[i];
  }
  for (int i = 0; i < N; ++i)
    for (int p : nodes[i].preds) nodes[p].succs.push_back(i);
  int max_level = 0;
  for (int i = 0; i < N; ++i) {
    int a = 0;
    for (int p : nodes[i].preds) a = std::max(a, nodes[p].asap + 1);
    nodes[i].asap = a;
    max_level = std::max(max_level, a);
  }
  for (int i = N - 1; i >= 0; --i) {
    int h = 0;
    for (int s : nodes[i].succs) h = std::max(h, nodes[s].height + 1);
    nodes[i].height = h;
  }

  // ---- waves
  const int W = max_level + 1;
  if (policy == SCHED_LEARNED) {
    std::vector<double> load(W, 0.0);
    for (int i = 0; i < N; ++i) {  // command order is topological
      int lo = nodes[i].asap;
      for (int p : nodes[i].preds) lo = std::max(lo, nodes[p].wave + 1);
      int hi = std::max(lo, max_level - nodes[i].height);
      int best = lo;
      for (int w = lo; w <= hi; ++w)
        if (load[w] < load[best] - 1e-9) best = w;
      nodes[i].wave = best;
      load[best] += nodes[i].cost;
    }
  } else {
    for (auto& n : nodes) n.wave = n.asap;
  }
  int nw = 0;
  for (auto& n : nodes) nw = std::max(nw, n.wave + 1);

  // ---- tensor lifetimes
  for (int i = 0; i < N; ++i) {
    for (tid_t t : nodes[i].outs) {
      auto& tp = d->tensors[t];
      tp.def = nodes[i].wave;
      tp.last = std::max(tp.last, nodes[i].wave);
    }
    for (tid_t t : nodes[i].ins) {
      auto& tp = d->tensors[t];
      tp.last = std::max(tp.last, nodes[i].wave);
    }
  }

  // ---- memory: deleted intermediates share one arena (first fit on disjoint
  // lifetimes); results nobody deletes get their own allocations.
  struct placed_t { size_t off, bytes; int def, last; };
  std::vector<placed_t> placed;
  std::vector<std::pair<tid_t, tplan_t*>> order;
  for (auto& kv : d->tensors)
    if (!kv.second.external && kv.second.deleted) order.push_back({kv.first, &kv.second});
  std::sort(order.begin(), order.end(), [](const auto& a, const auto& b) {
    if (a.second->bytes != b.second->bytes) return a.second->bytes > b.second->bytes;
    return a.first < b.first;
  });
  std::unordered_map<tid_t, size_t> offsets;
  size_t arena = 0;
  for (auto& [tid, tp] : order) {
    const size_t bytes = (tp->bytes + 255) & ~(size_t)255;
    std::vector<std::pair<size_t, size_t>> busy;
    for (auto& p : placed)
      if (!(p.last < tp->def || tp->last < p.def)) busy.push_back({p.off, p.off + p.bytes});
    std::sort(busy.begin(), busy.end());
    size_t off = 0;
    for (auto& b : busy) {
      if (off + bytes <= b.first) break;
      off = std::max(off, b.second);
    }
    placed.push_back({off, bytes, tp->def, tp->last});
    offsets[tid] = off;
    arena = std::max(arena, off + bytes);
  }
  if (arena) dag_cuda(cudaMalloc(&d->arena, arena), "cudaMalloc(DAG arena)");
  d->arena_bytes = arena;
  for (auto& kv : offsets) d->tensors[kv.first].payload = (char*)d->arena + kv.second;
  for (auto& kv : d->tensors) {
    auto& tp = kv.second;
    if (tp.external || tp.deleted) continue;
    void* p = nullptr;
    if (tp.bytes) dag_cuda(cudaMalloc(&p, tp.bytes), "cudaMalloc(DAG result)");
    tp.payload = p;
    d->persistent.push_back(p);
  }
  for (auto& kv : d->tensors) kv.second.meta.set_payload(kv.second.payload);

  // ---- per-wave launch plans
  std::vector<std::vector<int>> by_wave(nw);
  for (int i = 0; i < N; ++i) by_wave[nodes[i].wave].push_back(i);
  d->waves.resize(nw);
  for (int w = 0; w < nw; ++w) {
    auto& ids = by_wave[w];
    if (policy == SCHED_LEARNED)
      std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) { return nodes[a].cost > nodes[b].cost; });
    else
      std::reverse(ids.begin(), ids.end());  // LIFO: the last queued ready command first
    std::map<int, std::vector<bbx_tc_problem_t>> tc_groups;  // key: dtype | amn | bmn
    std::vector<std::vector<bbx_stream_op_t>> phases(1);
    for (int i : ids) {
      node_t& n = nodes[i];
      const command_t& c = *n.cmd;
      ud_impl_t::tensor_params_t params;
      params._params = c.get_parameters();
      if (n.kind == NK_TC) {
        auto& ta_ = d->tensors.at(n.ins[0]);
        auto& tb_ = d->tensors.at(n.ins[1]);
        auto& tc_ = d->tensors.at(n.outs[0]);
        const auto& ma = ta_.meta.as<dense_tensor_meta_t>().m();
        const auto& mb = tb_.meta.as<dense_tensor_meta_t>().m();
        bbx_tc_problem_t q{};
        bool ta = params.get_bool_or_default<0>(false), tb = params.get_bool_or_default<1>(false);
        q.a = ta_.payload; q.b = tb_.payload; q.c = tc_.payload;
        q.m = ta ? ma.num_cols : ma.num_rows;
        q.k = ta ? ma.num_rows : ma.num_cols;
        q.n = tb ? mb.num_rows : mb.num_cols;
        q.trans_a = ta; q.trans_b = tb;
        q.lda = ma.num_cols; q.ldb = mb.num_cols; q.ldc = q.n;
        const int in_dt = elem_of(tf, ta_.meta.fmt_id);
        q.alpha = in_dt == ELEM_E4M3 ? ma.scale * mb.scale : 1.0f;
        q.flags = elem_of(tf, tc_.meta.fmt_id) == ELEM_BF16 ? BBX_EPI_OUT_BF16 : 0;
        tc_groups[in_dt * 4 + (ta ? 2 : 0) + (tb ? 1 : 0)].push_back(q);
      } else if (n.kind == NK_SUM || n.kind == NK_UNARY || n.kind == NK_BINARY) {
        auto& to = d->tensors.at(n.outs[0]);
        const auto& m0 = d->tensors.at(n.ins[0]).meta.as<dense_tensor_meta_t>().m();
        const long long elems = (long long)m0.num_rows * m0.num_cols;
        const int dt = elem_of(tf, d->tensors.at(n.ins[0]).meta.fmt_id) == ELEM_BF16 ? BBX_BF16 : BBX_F32;
        if (n.kind == NK_SUM) {
          size_t done = 0;
          int ph = 0;
          while (done < n.ins.size()) {
            bbx_stream_op_t s{};
            s.kind = BBX_S_SUM; s.in_dtype = dt; s.out_dtype = dt; s.kahan = 1; s.n = elems; s.out = to.payload;
            int cnt = 0;
            if (done > 0) s.in[cnt++] = to.payload;  // keep folding into the output
            while (cnt < BBX_STREAM_MAX_IN && done < n.ins.size()) s.in[cnt++] = d->tensors.at(n.ins[done++]).payload;
            s.n_in = cnt;
            if ((int)phases.size() <= ph) phases.resize(ph + 1);
            phases[ph++].push_back(s);
          }
        } else {
          bbx_stream_op_t s{};
          s.kind = n.kind == NK_UNARY ? BBX_S_UNARY : BBX_S_BINARY;
          const std::string& nm = n.impl->impl_name;
          if (n.kind == NK_UNARY)
            s.op = nm.find("relu_dif") != std::string::npos ? BBX_U_RELU_DIF
                 : nm.find("relu") != std::string::npos     ? BBX_U_RELU
                                                            : BBX_U_SIGMOID_REF;
          else
            s.op = nm.find("hadamard") != std::string::npos ? BBX_B_HADAMARD : BBX_B_WEIGHTED;
          if (s.op == BBX_B_WEIGHTED) {
            s.p0 = params.get_float_or_default<0>(1.f);
            s.p1 = params.get_float_or_default<1>(1.f);
          }
          s.in_dtype = dt; s.out_dtype = dt; s.n = elems; s.out = to.payload;
          s.n_in = n.kind == NK_UNARY ? 1 : 2;
          for (int j = 0; j < s.n_in; ++j) s.in[j] = d->tensors.at(n.ins[j]).payload;
          phases[0].push_back(s);
        }
      } else {
        opaque_t o;
        o.impl = n.impl;
        auto pl = c.get_parameters();
        o.params.assign(pl.begin(), pl.end());
        o.ins = n.ins;
        o.outs = n.outs;
        d->waves[w].opaque.push_back(std::move(o));
      }
      d->stats.flops += n.flops;
      d->stats.bytes += n.bytes;
    }
    for (auto& ph : phases) {
      if (ph.empty()) continue;
      bbx_stream_plan_t* p = nullptr;
      dag_bbx(bbx_stream_plan_create(ph.data(), (int)ph.size(), &p));
      d->waves[w].phases.push_back(p);
      d->stats.stream_launches++;
    }
    for (auto& kv : tc_groups) {
      bbx_tc_plan_t* p = nullptr;
      const int dt = kv.first / 4;
      // tile_n < 0: autotune per group; 0: size heuristic; 128 / 256: forced
      const int tn = tile_n < 0 ? autotune_tile_n(dt, (kv.first & 2) != 0, (kv.first & 1) != 0, kv.second) : tile_n;
      dag_bbx(bbx_tc_plan_create(dt == ELEM_E4M3 ? BBX_E4M3 : BBX_BF16, kv.second.data(),
                                 (int)kv.second.size(), tn, &p));
      d->waves[w].tc.push_back(p);
      d->stats.tc_launches++;
    }
    d->stats.opaque_launches += (int)d->waves[w].opaque.size();
  }
  d->stats.waves = nw;
  d->stats.nodes = N;
  d->stats.arena_bytes = arena;

  // ---- capture the whole launch sequence in one CUDA graph
  cudaStream_t cs;
  dag_cuda(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "cudaStreamCreate(capture)");
  dag_cuda(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  try {
    issue(d.get(), cs);
  } catch (...) {
    cudaGraph_t g;
    cudaStreamEndCapture(cs, &g);
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    dag_destroy(d.release());
    throw;
  }
  dag_cuda(cudaStreamEndCapture(cs, &d->graph), "cudaStreamEndCapture");
  dag_cuda(cudaGraphInstantiate(&d->exec, d->graph, 0), "cudaGraphInstantiate");
  cudaStreamDestroy(cs);
  return d.release();
}

void dag_launch(dag_t* d, cudaStream_t st) {
  dag_cuda(cudaGraphLaunch(d->exec, st), "cudaGraphLaunch");
}

void dag_destroy(dag_t* d) {
  if (!d) return;
  cudaDeviceSynchronize();
  if (d->exec) cudaGraphExecDestroy(d->exec);
  if (d->graph) cudaGraphDestroy(d->graph);
  for (auto& w : d->waves) {
    for (auto* p : w.phases) bbx_stream_plan_destroy(p);
    for (auto* p : w.tc) bbx_tc_plan_destroy(p);
  }
  if (d->arena) cudaFree(d->arena);
  for (void* p : d->persistent) cudaFree(p);
  delete d;
}

dag_stats_t dag_stats(const dag_t* d) { return d->stats; }

// Device address of a tensor a DAG produced or read (nullptr if unknown).
void* dag_tensor(const dag_t* d, tid_t tid, tensor_meta_t* meta) {
  auto it = d->tensors.find(tid);
  if (it == d->tensors.end()) return nullptr;
  if (meta) *meta = it->second.meta;
  return it->second.payload;
}

size_t dag_payload_bytes(const dag_t* d, tid_t tid) {
  auto it = d->tensors.find(tid);
  return it == d->tensors.end() ? 0 : it->second.bytes;
}

}  // namespace bbts
