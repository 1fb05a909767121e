// Grouped DAG executor.
//
// A compiled command list (APPLY / REDUCE / DELETE) is lowered once into
// waves of launch groups:
//   PRE     one grouped gather launch: the operand gathers of the wave's
//           tensor-core contractions (Lc / Rc staging blocks)
//   STREAM  grouped streaming launches: every add / n-ary reduce / elementwise
//           node of the wave, and the split first activation as two
//           element-wise ops (more than 16 reduce inputs chain extra phases)
//   OTHER   direct calls of the remaining impls (FP32 SIMT matmul, FP32
//           contraction, FNN ops, softmax, uniform)
//   TC      one grouped tcgen05 launch per operand-layout class: the wave's
//           block matmuls and contraction matmuls
//   POST    one grouped gather launch: contraction outputs whose mode order
//           needs a final permutation
// TC groups run on a tensor stream, everything else on a memory stream, and
// the launches are captured into ONE CUDA graph whose edges are the true
// tensor dependencies between groups plus a wave barrier two waves back, so a
// wave's HBM-bound streaming work overlaps its tensor-core work and the next
// wave's. Intermediate blocks share one arena: a slot is reused only by a block
// defined at least two waves after the slot's last reader (the barrier makes
// that reader finished).
//
// Scheduling policies (what the learned cost model changes):
//   heuristic  waves = ASAP levels; problems of a grouped launch in
//              reservation-station LIFO order; costs = complexity hints.
//   learned    nodes carry the MLP's predicted latency and a resource (tensor
//              or memory); a node with slack goes to the wave within
//              [ASAP, ALAP] that least increases max(tensor time, memory time)
//              of that wave, and grouped launches order problems longest first.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include "contraction.h"
#include "runtime.h"

namespace bbx {
int pick_tile_n(const bbx_tc_problem_t* probs, int count, int in_dtype);  // abi_kernels.cu
}

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
  bool tc_contract = false;  // bf16 contraction lowered into PRE / TC / POST groups
  std::vector<tid_t> ins, outs;
  int asap = 0, height = 0, wave = 0;
  int resource = 1;          // 0 tensor stream, 1 memory stream
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
};

enum group_kind_t { G_PRE = 0, G_STREAM = 1, G_OTHER = 2, G_TC = 3, G_POST = 4 };

struct group_t {
  group_kind_t kind;
  int wave;
  std::vector<tid_t> reads, writes;
  bbx_stream_plan_t* stream_plan = nullptr;
  bbx_tc_plan_t* tc_plan = nullptr;
  bbx::GatherPlan* gather_plan = nullptr;
  std::vector<opaque_t> opaque;
  std::vector<int> deps;  // indices of earlier groups this one waits for
  double flops = 0.0;     // algorithmic work of the launch: 2mnk for tensor groups,
  double bytes = 0.0;     // bytes read + written once for streaming / gather groups
};

double tc_group_flops(const std::vector<bbx_tc_problem_t>& ps) {
  double f = 0;
  for (auto& q : ps) f += 2.0 * q.m * (double)q.n * q.k;
  return f;
}

double tc_group_bytes(const std::vector<bbx_tc_problem_t>& ps, int in_esz) {
  double b = 0;
  for (auto& q : ps)
    b += ((double)q.m * q.k + (double)q.k * q.n) * in_esz + (double)q.m * q.n * ((q.flags & BBX_EPI_OUT_BF16) ? 2 : 4);
  return b;
}

double stream_group_bytes(const std::vector<bbx_stream_op_t>& ops) {
  double b = 0;
  for (auto& s : ops)
    b += (double)s.n * (s.n_in * (s.in_dtype == BBX_BF16 ? 2 : 4) + (s.out_dtype == BBX_BF16 ? 2 : 4));
  return b;
}

double gather_group_bytes(const std::vector<bbx::GatherRec>& rs) {
  double b = 0;
  for (auto& r : rs) b += (double)r.n * (4 + (r.dst_bf16 ? 2 : 4));
  return b;
}

}  // namespace

struct dag_t {
  runtime_t* rt = nullptr;
  std::vector<group_t> groups;
  std::unordered_map<tid_t, tplan_t> tensors;
  std::unordered_map<tid_t, std::unique_ptr<char[]>> headers;
  void* arena = nullptr;
  size_t arena_bytes = 0;
  std::vector<void*> persistent;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  dag_stats_t stats{};
  // blocks the graph reads in place: held resident (never spilled) while it lives
  std::vector<tid_t> held;
  ~dag_t() {
    if (rt && !held.empty()) rt->storage->release(held);
  }
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

void launch_group(dag_t* d, group_t& g, cudaStream_t st) {
  switch (g.kind) {
    case G_PRE:
    case G_POST: dag_bbx(bbx::gather_plan_launch(g.gather_plan, st)); break;
    case G_STREAM: dag_bbx(bbx_stream_plan_launch(g.stream_plan, st)); break;
    case G_TC: dag_bbx(bbx_tc_plan_launch(g.tc_plan, st)); break;
    case G_OTHER:
      for (auto& o : g.opaque) run_opaque(d, o, st);
      break;
  }
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
  int maxn = 0, maxm = 0, ccol = 0;
  for (auto& q : ps) {
    fl += 2.0 * q.m * q.n * (double)q.k;
    maxn = std::max(maxn, q.n);
    maxm = std::max(maxm, q.m);
    ccol |= (q.flags & BBX_EPI_C_COLMAJOR) ? 1 : 0;
  }
  char buf[128];
  std::snprintf(buf, sizeof(buf), "d%d_a%d_b%d_c%d_p%d_f%d_n%d_m%d", dtype, (int)ta, (int)tb, ccol,
                (int)std::ceil(std::log2((double)ps.size() + 1)), (int)std::log2(fl + 1), (int)std::log2(maxn + 1),
                (int)std::log2(maxm + 1));
  return buf;
}

// Features of a grouped tensor-core launch run with tile `tn` (the input of the
// learned tile choice, same 12-wide layout as the per-op features): tile
// one-hot (128, 256, 512), log2 of the problem count, of the FLOPs, of the
// largest m and n, of the tiles the launch runs, of the mean k, dtype (0 bf16,
// 1 e4m3), operand layouts.
op_features_t tile_features(int dtype, bool ta, bool tb, const std::vector<bbx_tc_problem_t>& ps, int tn) {
  op_features_t f{};
  double fl = 0, ksum = 0, tiles = 0;
  int maxm = 0, maxn = 0;
  for (auto& q : ps) {
    fl += 2.0 * q.m * q.n * (double)q.k;
    ksum += q.k;
    maxm = std::max(maxm, q.m);
    maxn = std::max(maxn, q.n);
    const int bm = tn == 512 ? 256 : 128, bn = tn == 512 ? 256 : tn;
    tiles += (double)((q.m + bm - 1) / bm) * ((q.n + bn - 1) / bn);
  }
  f.f[0] = tn == 128 ? 1.f : 0.f;
  f.f[1] = tn == 256 ? 1.f : 0.f;
  f.f[2] = tn == 512 ? 1.f : 0.f;
  f.f[3] = (float)std::log2((double)ps.size());
  f.f[4] = (float)std::log2(std::max(1.0, fl));
  f.f[5] = (float)std::log2(std::max(1, maxm));
  f.f[6] = (float)std::log2(std::max(1, maxn));
  f.f[7] = (float)std::log2(std::max(1.0, tiles));
  f.f[8] = (float)std::log2(std::max(1.0, ksum / std::max<size_t>(1, ps.size())));
  f.f[9] = dtype == ELEM_E4M3 ? 1.f : 0.f;
  f.f[10] = ta ? 1.f : 0.f;
  f.f[11] = tb ? 1.f : 0.f;
  return f;
}

// Samples of the autotuner's own timings, (group features for a tile, us per
// launch), recorded while tile_record(true) is on: the training set of the
// learned tile choice.
std::mutex g_tile_mu;
bool g_tile_rec = false;
std::vector<std::pair<op_features_t, float>> g_tile_samples;

int autotune_tile_n(int dtype, bool ta, bool tb, const std::vector<bbx_tc_problem_t>& ps) {
  const std::string key = tune_key(dtype, ta, tb, ps);
  const char* path = std::getenv("BBX_TUNE_CACHE");
  bool recording;
  {
    std::lock_guard<std::mutex> lk(g_tile_mu);
    recording = g_tile_rec;
  }
  if (!recording) {
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
  // every candidate's plan is built before any runs and freed after all ran,
  // so no plan's table lands where another candidate's tensor maps were used
  std::vector<std::pair<int, bbx_tc_plan_t*>> cand;
  for (int tn : {512, 256, 128}) {
    if (tn == 512 && dtype == ELEM_E4M3) continue;  // the 2-SM pair tile is bf16 only
    bbx_tc_plan_t* p = nullptr;
    if (bbx_tc_plan_create(dtype == ELEM_E4M3 ? BBX_E4M3 : BBX_BF16, ps.data(), (int)ps.size(), tn, &p) == 0)
      cand.push_back({tn, p});
  }
  auto release = [&]() {
    cudaStreamSynchronize(st);
    for (auto& c : cand) bbx_tc_plan_destroy(c.second);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
  };
  try {
    for (auto& c : cand) {
      dag_bbx(bbx_tc_plan_launch(c.second, st));  // warm-up
      cudaEventRecord(e0, st);
      for (int r = 0; r < 3; ++r) dag_bbx(bbx_tc_plan_launch(c.second, st));
      cudaEventRecord(e1, st);
      dag_cuda(cudaEventSynchronize(e1), "tune sync");
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best_ms) { best_ms = ms; best = c.first; }
      if (recording) {
        std::lock_guard<std::mutex> lk(g_tile_mu);
        g_tile_samples.push_back({tile_features(dtype, ta, tb, ps, c.first), ms * 1000.f / 3.f});
      }
    }
  } catch (...) {
    release();
    throw;
  }
  release();
  if (recording) return best;  // samples are being taken: the cache is neither read nor written
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

// The tile whose launch the runtime's tile model predicts fastest.
int learned_tile_n(const runtime_t& rt, int dtype, bool ta, bool tb, const std::vector<bbx_tc_problem_t>& ps) {
  std::vector<int> cand;
  for (int tn : {512, 256, 128})
    if (!(tn == 512 && dtype == ELEM_E4M3)) cand.push_back(tn);
  std::vector<op_features_t> fs;
  for (int tn : cand) fs.push_back(tile_features(dtype, ta, tb, ps, tn));
  const std::vector<double> t = rt.tile_predictor(fs);
  size_t best = 0;
  for (size_t i = 1; i < cand.size() && i < t.size(); ++i)
    if (t[i] < t[best]) best = i;
  return cand[best];
}

// Bytes per microsecond of the bulk streaming kernel alone on DAG levels
// (5.0-5.3 TB/s measured on the 2000-op DAG's levels).
constexpr double kBulkStreamBytesPerUs = 5.2e6;

// Predicted duration (us) of a grouped tensor-core launch with tile `tn`: the
// tile model's prediction when one is installed, else its FLOPs at 1 PFLOP/s
// (about the grouped kernel's rate on the DAG's matmul groups).
double predicted_tc_us(const runtime_t& rt, int dtype, bool ta, bool tb, const std::vector<bbx_tc_problem_t>& ps,
                       int tn) {
  if (rt.tile_predictor) {
    if (tn == 0) {
      std::vector<bbx_tc_problem_t> v(ps);
      tn = bbx::pick_tile_n(v.data(), (int)v.size(), dtype == ELEM_E4M3 ? BBX_E4M3 : BBX_BF16);
    }
    return rt.tile_predictor({tile_features(dtype, ta, tb, ps, tn)})[0];
  }
  return tc_group_flops(ps) / 1e15 * 1e6;
}

// Contraction params: rank_l, rank_r, rank_o, modes_l..., modes_r..., modes_o..., alpha.
struct cparams_t {
  std::vector<int> ml, mr, mo;
  float alpha;
};
cparams_t parse_contraction(const command_t& c) {
  auto p = c.get_parameters();
  cparams_t r;
  int rl = p[0].i, rr = p[1].i, ro = p[2].i;
  size_t i = 3;
  for (int d = 0; d < rl; ++d) r.ml.push_back(p[i++].i);
  for (int d = 0; d < rr; ++d) r.mr.push_back(p[i++].i);
  for (int d = 0; d < ro; ++d) r.mo.push_back(p[i++].i);
  r.alpha = p[i].f;
  return r;
}

}  // namespace

dag_t* dag_build(runtime_t* rt, int policy, int tile_n) {
  auto d = std::make_unique<dag_t>();
  d->rt = rt;
  const tensor_factory_t& tf = *rt->tf;

  // ---- tensors that already exist (registered inputs), resident for the graph's lifetime
  d->held = rt->storage->hold_all();
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
    n.tc_contract = n.kind == NK_CONTRACT && n.impl->impl_name == "b200_contraction_bf16";
    n.resource = (n.kind == NK_TC || n.tc_contract) ? 0 : 1;
    std::vector<tensor_meta_t> in_metas;
    for (size_t i = 0; i < c.get_num_inputs(); ++i) {
      tid_t t = c.get_input(i).tid;
      auto it = d->tensors.find(t);
      if (it == d->tensors.end())
        throw std::runtime_error("DAG: command " + std::to_string(c.id) + " reads tensor " + std::to_string(t) +
                                 " that nothing creates");
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
    // tensor and memory streams overlap inside a wave: minimise sum_w max(tc_w, mem_w)
    std::vector<double> load[2] = {std::vector<double>(W, 0.0), std::vector<double>(W, 0.0)};
    for (int i = 0; i < N; ++i) {  // command order is topological
      int lo = nodes[i].asap;
      for (int p : nodes[i].preds) lo = std::max(lo, nodes[p].wave + 1);
      int hi = std::max(lo, max_level - nodes[i].height);
      const int r = nodes[i].resource;
      int best = lo;
      double best_inc = 1e300;
      for (int w = lo; w <= hi; ++w) {
        double before = std::max(load[0][w], load[1][w]);
        double after = std::max(load[r][w] + nodes[i].cost, load[1 - r][w]);
        double inc = after - before;
        if (inc < best_inc - 1e-12) { best_inc = inc; best = w; }
      }
      nodes[i].wave = best;
      load[r][best] += nodes[i].cost;
    }
  } else {
    for (auto& n : nodes) n.wave = n.asap;
  }
  int nw = 0;
  for (auto& n : nodes) nw = std::max(nw, n.wave + 1);

  // ---- contraction staging blocks (arena slots living for one wave)
  struct cstage_t { tid_t lc, rc, ct; bbx::ContractionLowering L; cparams_t p; };
  std::unordered_map<int, cstage_t> cstage;
  tid_t next_stage = -1000000;
  for (int i = 0; i < N; ++i) {
    node_t& n = nodes[i];
    if (!n.tc_contract) continue;
    cstage_t cs;
    cs.p = parse_contraction(*n.cmd);
    const auto& sl = d->tensors.at(n.ins[0]).meta.as<cu_meta_t>().m();
    const auto& sr = d->tensors.at(n.ins[1]).meta.as<cu_meta_t>().m();
    std::vector<long long> dl(sl.dims, sl.dims + sl.rank), dr(sr.dims, sr.dims + sr.rank);
    dag_bbx(bbx::lower_contraction((int)dl.size(), dl.data(), cs.p.ml.data(), (int)dr.size(), dr.data(),
                                   cs.p.mr.data(), (int)cs.p.mo.size(), cs.p.mo.data(), true, &cs.L));
    auto stage = [&](size_t bytes) {
      tid_t t = next_stage--;
      tplan_t tp;
      std::memset(&tp.meta, 0, sizeof(tp.meta));
      tp.bytes = bytes;
      tp.def = tp.last = n.wave;
      tp.deleted = true;
      d->tensors[t] = tp;
      return t;
    };
    cs.lc = stage((size_t)(cs.L.lc_elems * 2 + 16));
    cs.rc = stage((size_t)(cs.L.rc_elems * 2 + 16));
    cs.ct = cs.L.direct ? TID_NONE : stage((size_t)(cs.L.nb * cs.L.nn * cs.L.nm * 4));
    cstage[i] = cs;
  }

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

  // ---- memory: deleted intermediates and staging blocks share one arena; a
  // slot is reused only by a block defined two or more waves after its last use
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
      if (!(p.last + 1 < tp->def || tp->last + 1 < p.def)) busy.push_back({p.off, p.off + p.bytes});
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

  // ---- launch groups per wave
  std::vector<std::vector<int>> by_wave(nw);
  for (int i = 0; i < N; ++i) by_wave[nodes[i].wave].push_back(i);
  // waves with block matmuls on the tensor stream: a wave's gathers may run
  // beside its own and the previous wave's matmul launches, which the
  // bulk-staged gather (its shared memory) would keep off those SMs
  std::vector<char> wave_mm(nw, 0);
  for (int i = 0; i < N; ++i)
    if (nodes[i].kind == NK_TC) wave_mm[nodes[i].wave] = 1;
  for (int w = 0; w < nw; ++w) {
    auto& ids = by_wave[w];
    const bool bulk_gather = !wave_mm[w] && !(w > 0 && wave_mm[w - 1]);
    if (policy == SCHED_LEARNED)
      std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) { return nodes[a].cost > nodes[b].cost; });
    else
      std::reverse(ids.begin(), ids.end());  // LIFO: the last queued ready command first
    std::map<int, std::vector<bbx_tc_problem_t>> tc_groups;  // key: dtype*4 + ta*2 + tb
    std::map<int, std::pair<std::vector<tid_t>, std::vector<tid_t>>> tc_rw;
    std::vector<std::vector<bbx_stream_op_t>> phases(1);
    std::vector<std::pair<std::vector<tid_t>, std::vector<tid_t>>> phase_rw(1);
    std::vector<bbx::GatherRec> pre, post;
    group_t gpre{G_PRE, w}, gpost{G_POST, w}, gother{G_OTHER, w};
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
        const int key = in_dt * 4 + (ta ? 2 : 0) + (tb ? 1 : 0);
        tc_groups[key].push_back(q);
        tc_rw[key].first.insert(tc_rw[key].first.end(), n.ins.begin(), n.ins.end());
        tc_rw[key].second.push_back(n.outs[0]);
      } else if (n.tc_contract) {
        cstage_t& cs = cstage.at(i);
        auto& L = cs.L;
        if (!L.empty) {
          auto& tl = d->tensors.at(cs.lc);
          auto& tr = d->tensors.at(cs.rc);
          bbx::GatherRec ra{}, rb{};
          ra.a = L.ga; ra.src = (const float*)d->tensors.at(n.ins[0]).payload; ra.dst = tl.payload; ra.dst_bf16 = 1; ra.n = L.nl;
          rb.a = L.gb; rb.src = (const float*)d->tensors.at(n.ins[1]).payload; rb.dst = tr.payload; rb.dst_bf16 = 1; rb.n = L.nr;
          pre.push_back(ra);
          pre.push_back(rb);
          gpre.reads.insert(gpre.reads.end(), n.ins.begin(), n.ins.end());
          gpre.writes.push_back(cs.lc);
          gpre.writes.push_back(cs.rc);
          void* C = L.direct ? d->tensors.at(n.outs[0]).payload : d->tensors.at(cs.ct).payload;
          // A = Rc, B = Lc in their staging layouts. Contraction problems get
          // groups of their own (key bit 8): they wait for the wave's gathers,
          // while the matmul groups can start as soon as their inputs exist
          // operand layouts (hence the kernel variant) depend on the GEMM's orientation
          const bbx::ContractionGemm g0 = bbx::contraction_gemm(L, tl.payload, tr.payload, C, 0);
          const int key = 256 + ELEM_BF16 * 4 + (g0.trans_a ? 2 : 0) + (g0.trans_b ? 1 : 0);
          for (long long b = 0; b < L.nb; ++b) {
            const bbx::ContractionGemm g = bbx::contraction_gemm(L, tl.payload, tr.payload, C, b);
            bbx_tc_problem_t q{};
            q.a = g.a; q.b = g.b; q.c = g.c;
            q.m = g.m; q.n = g.n; q.k = g.k;
            q.trans_a = g.trans_a; q.trans_b = g.trans_b;
            q.lda = g.lda; q.ldb = g.ldb; q.ldc = g.ldc;
            q.flags = g.flags;
            q.alpha = cs.p.alpha;
            tc_groups[key].push_back(q);
          }
          tc_rw[key].first.push_back(cs.lc);
          tc_rw[key].first.push_back(cs.rc);
          tc_rw[key].second.push_back(L.direct ? n.outs[0] : cs.ct);
          if (!L.direct) {
            bbx::GatherRec ro{};
            ro.a = L.go; ro.src = (const float*)d->tensors.at(cs.ct).payload; ro.dst = d->tensors.at(n.outs[0]).payload;
            ro.dst_bf16 = 0; ro.n = L.no;
            post.push_back(ro);
            gpost.reads.push_back(cs.ct);
            gpost.writes.push_back(n.outs[0]);
          }
        }
      } else if (n.kind == NK_SUM || n.kind == NK_UNARY || n.kind == NK_BINARY) {
        auto& to = d->tensors.at(n.outs[0]);
        const auto& m0 = d->tensors.at(n.ins[0]).meta.as<dense_tensor_meta_t>().m();
        const long long elems = (long long)m0.num_rows * m0.num_cols;
        const int dt = elem_of(tf, d->tensors.at(n.ins[0]).meta.fmt_id) == ELEM_BF16 ? BBX_BF16 : BBX_F32;
        const int odt = elem_of(tf, to.meta.fmt_id) == ELEM_BF16 ? BBX_BF16 : BBX_F32;
        if (n.kind == NK_SUM) {
          size_t done = 0;
          int ph = 0;
          while (done < n.ins.size()) {
            bbx_stream_op_t s{};
            s.kind = BBX_S_SUM; s.in_dtype = dt; s.out_dtype = dt; s.kahan = 1; s.n = elems; s.out = to.payload;
            int cnt = 0;
            if (done > 0) s.in[cnt++] = to.payload;  // keep folding into the output
            const size_t first = done;
            while (cnt < BBX_STREAM_MAX_IN && done < n.ins.size()) s.in[cnt++] = d->tensors.at(n.ins[done++]).payload;
            s.n_in = cnt;
            if ((int)phases.size() <= ph) { phases.resize(ph + 1); phase_rw.resize(ph + 1); }
            phases[ph].push_back(s);
            phase_rw[ph].first.insert(phase_rw[ph].first.end(), n.ins.begin() + first, n.ins.begin() + done);
            phase_rw[ph].second.push_back(n.outs[0]);
            ++ph;
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
          s.in_dtype = dt; s.out_dtype = odt; s.n = elems; s.out = to.payload;
          s.n_in = n.kind == NK_UNARY ? 1 : 2;
          for (int j = 0; j < s.n_in; ++j) s.in[j] = d->tensors.at(n.ins[j]).payload;
          phases[0].push_back(s);
          phase_rw[0].first.insert(phase_rw[0].first.end(), n.ins.begin(), n.ins.end());
          phase_rw[0].second.push_back(n.outs[0]);
        }
      } else if (n.kind == NK_OPAQUE && !c.is_reduce() && n.impl->impl_name == "b200_dense_split_relu") {
        // the split first activation as two element-wise ops of the wave's
        // streaming launch: hi = bf16(relu(z)), lo = bf16(relu(z) - hi), the
        // bytes of its impl (bbx_relu_split)
        const auto& mz = d->tensors.at(n.ins[0]).meta.as<dense_tensor_meta_t>().m();
        for (int j = 0; j < 2; ++j) {
          bbx_stream_op_t s{};
          s.kind = BBX_S_UNARY;
          s.op = j == 0 ? BBX_U_RELU : BBX_U_RELU_LO;
          s.in_dtype = BBX_F32; s.out_dtype = BBX_BF16; s.n_in = 1; s.kahan = 0;
          s.n = (long long)mz.num_rows * mz.num_cols;
          s.in[0] = d->tensors.at(n.ins[0]).payload;
          s.out = d->tensors.at(n.outs[j]).payload;
          phases[0].push_back(s);
          phase_rw[0].second.push_back(n.outs[j]);
        }
        phase_rw[0].first.push_back(n.ins[0]);
      } else {
        opaque_t o;
        o.impl = n.impl;
        auto pl = c.get_parameters();
        o.params.assign(pl.begin(), pl.end());
        o.ins = n.ins;
        o.outs = n.outs;
        gother.reads.insert(gother.reads.end(), n.ins.begin(), n.ins.end());
        gother.writes.insert(gother.writes.end(), n.outs.begin(), n.outs.end());
        gother.opaque.push_back(std::move(o));
      }
      d->stats.flops += n.flops;
      d->stats.bytes += n.bytes;
    }
    // group order inside a wave: PRE, STREAM phases, OTHER (memory stream); TC (tensor stream); POST
    if (!pre.empty()) {
      dag_bbx(bbx::gather_plan_create(pre.data(), (int)pre.size(), &gpre.gather_plan, bulk_gather));
      gpre.bytes = gather_group_bytes(pre);
      d->groups.push_back(std::move(gpre));
      d->stats.stream_launches++;
    }
    // tiles of the wave's tensor groups first: the per-wave streaming kernel
    // choice weighs the wave's predicted tensor time
    std::map<int, int> tc_tile;
    double tc_us = 0.0;
    for (auto& kv : tc_groups) {
      const int dt = (kv.first & 0xff) / 4;
      // tile_n -1: autotune per group; -2: the learned tile model (the size
      // heuristic without one); 0: size heuristic; 128 / 256 / 512: forced
      const bool ta = (kv.first & 2) != 0, tb = (kv.first & 1) != 0;
      int tn = tile_n;
      if (tile_n == -2) tn = rt->tile_predictor ? learned_tile_n(*rt, dt, ta, tb, kv.second) : 0;
      else if (tile_n < 0) tn = autotune_tile_n(dt, ta, tb, kv.second);
      tc_tile[kv.first] = tn;
      if (rt->dag_stream_kernel == BBX_STREAM_KERNEL_PER_WAVE)
        tc_us += predicted_tc_us(*rt, dt, ta, tb, kv.second, tn);
    }
    int stream_kernel = rt->dag_stream_kernel;
    if (stream_kernel == BBX_STREAM_KERNEL_PER_WAVE) {
      double st_bytes = 0.0;
      for (auto& ph : phases) st_bytes += stream_group_bytes(ph);
      // the register kernel shares SMs with the tensor launch but streams
      // slower than the bulk kernel alone: worth it when the wave's tensor work
      // is long enough to hide the streaming work under it
      const double st_us = st_bytes / kBulkStreamBytesPerUs;
      stream_kernel = (st_bytes > 0 && tc_us >= st_us) ? BBX_STREAM_KERNEL_REGISTER : BBX_STREAM_KERNEL_AUTO;
      if (stream_kernel == BBX_STREAM_KERNEL_REGISTER && st_bytes > 0) d->stats.register_waves++;
    }
    for (size_t ph = 0; ph < phases.size(); ++ph) {
      if (phases[ph].empty()) continue;
      group_t g{G_STREAM, w};
      dag_bbx(bbx_stream_plan_create_kernel(phases[ph].data(), (int)phases[ph].size(), stream_kernel,
                                            &g.stream_plan));
      g.bytes = stream_group_bytes(phases[ph]);
      g.reads = phase_rw[ph].first;
      g.writes = phase_rw[ph].second;
      d->groups.push_back(std::move(g));
      d->stats.stream_launches++;
    }
    if (!gother.opaque.empty()) {
      d->stats.opaque_launches += (int)gother.opaque.size();
      d->groups.push_back(std::move(gother));
    }
    for (auto& kv : tc_groups) {
      group_t g{G_TC, w};
      const int dt = (kv.first & 0xff) / 4;
      const int tn = tc_tile.at(kv.first);
      dag_bbx(bbx_tc_plan_create(dt == ELEM_E4M3 ? BBX_E4M3 : BBX_BF16, kv.second.data(), (int)kv.second.size(), tn,
                                 &g.tc_plan));
      g.flops = tc_group_flops(kv.second);
      g.bytes = tc_group_bytes(kv.second, dt == ELEM_E4M3 ? 1 : 2);
      g.reads = tc_rw[kv.first].first;
      g.writes = tc_rw[kv.first].second;
      d->groups.push_back(std::move(g));
      d->stats.tc_launches++;
    }
    if (!post.empty()) {
      dag_bbx(bbx::gather_plan_create(post.data(), (int)post.size(), &gpost.gather_plan, bulk_gather));
      gpost.bytes = gather_group_bytes(post);
      d->groups.push_back(std::move(gpost));
      d->stats.stream_launches++;
    }
  }
  d->stats.waves = nw;
  d->stats.nodes = N;
  d->stats.arena_bytes = arena;

  // ---- dependencies between groups: producers of every read, and every group
  // two or more waves back (the wave barrier the arena reuse rule relies on)
  {
    std::unordered_map<tid_t, int> writer;
    for (int gi = 0; gi < (int)d->groups.size(); ++gi) {
      group_t& g = d->groups[gi];
      std::set<int> deps;
      for (tid_t t : g.reads) {
        auto it = writer.find(t);
        if (it != writer.end()) deps.insert(it->second);
      }
      for (int gj = 0; gj < gi; ++gj)
        if (d->groups[gj].wave <= g.wave - 2) deps.insert(gj);
      g.deps.assign(deps.begin(), deps.end());
      for (tid_t t : g.writes) writer[t] = gi;
    }
  }

  // ---- capture: tensor groups on one stream, the rest on another, joined by events
  cudaStream_t origin, s_mem, s_tc;
  dag_cuda(cudaStreamCreateWithFlags(&origin, cudaStreamNonBlocking), "cudaStreamCreate");
  dag_cuda(cudaStreamCreateWithFlags(&s_mem, cudaStreamNonBlocking), "cudaStreamCreate");
  dag_cuda(cudaStreamCreateWithFlags(&s_tc, cudaStreamNonBlocking), "cudaStreamCreate");
  std::vector<cudaEvent_t> ev(d->groups.size() + 1);
  for (auto& e : ev) dag_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
  // the library's per-device state (status word, kernel attributes) is set up
  // on its first use and allocates: never inside the capture below
  if (bbx_num_sms() < 0) {
    char msg[512];
    bbx_last_error(msg, sizeof msg);
    throw std::runtime_error(std::string("DAG build: device set-up failed: ") + msg);
  }
  dag_cuda(cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  bool ok = false;
  try {
    cudaEvent_t fork = ev.back();
    dag_cuda(cudaEventRecord(fork, origin), "fork");
    dag_cuda(cudaStreamWaitEvent(s_mem, fork, 0), "fork mem");
    dag_cuda(cudaStreamWaitEvent(s_tc, fork, 0), "fork tc");
    std::vector<bool> on_tc(d->groups.size());
    for (size_t gi = 0; gi < d->groups.size(); ++gi) {
      group_t& g = d->groups[gi];
      on_tc[gi] = g.kind == G_TC;
      cudaStream_t st = on_tc[gi] ? s_tc : s_mem;
      for (int dep : g.deps)
        if (on_tc[dep] != on_tc[gi]) dag_cuda(cudaStreamWaitEvent(st, ev[dep], 0), "dependency");
      launch_group(d.get(), g, st);
      dag_cuda(cudaEventRecord(ev[gi], st), "group event");
    }
    // join both streams back into the origin stream
    cudaEvent_t jm, jt;
    dag_cuda(cudaEventCreateWithFlags(&jm, cudaEventDisableTiming), "join event");
    dag_cuda(cudaEventCreateWithFlags(&jt, cudaEventDisableTiming), "join event");
    dag_cuda(cudaEventRecord(jm, s_mem), "join mem");
    dag_cuda(cudaEventRecord(jt, s_tc), "join tc");
    dag_cuda(cudaStreamWaitEvent(origin, jm, 0), "join");
    dag_cuda(cudaStreamWaitEvent(origin, jt, 0), "join");
    ok = true;
    dag_cuda(cudaStreamEndCapture(origin, &d->graph), "cudaStreamEndCapture");
    cudaEventDestroy(jm);
    cudaEventDestroy(jt);
  } catch (...) {
    if (!ok) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(origin, &g);
      if (g) cudaGraphDestroy(g);
    }
    for (auto& e : ev) cudaEventDestroy(e);
    cudaStreamDestroy(origin);
    cudaStreamDestroy(s_mem);
    cudaStreamDestroy(s_tc);
    dag_destroy(d.release());
    throw;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  cudaStreamDestroy(origin);
  cudaStreamDestroy(s_mem);
  cudaStreamDestroy(s_tc);
  dag_cuda(cudaGraphInstantiate(&d->exec, d->graph, 0), "cudaGraphInstantiate");
  return d.release();
}

void dag_launch(dag_t* d, cudaStream_t st) { dag_cuda(cudaGraphLaunch(d->exec, st), "cudaGraphLaunch"); }

// Replays every group on its own, one after another on `st`, bracketed by
// timing events: each launch's duration without the graph's overlap, for
// per-group roofline fractions. Group order is topological, so one stream
// honours every dependency; the results equal a graph replay's.
std::vector<dag_group_profile_t> dag_profile(dag_t* d, cudaStream_t st) {
  const size_t G = d->groups.size();
  std::vector<cudaEvent_t> ev(G + 1);
  for (auto& e : ev) dag_cuda(cudaEventCreate(&e), "cudaEventCreate");
  dag_cuda(cudaEventRecord(ev[0], st), "profile event");
  for (size_t gi = 0; gi < G; ++gi) {
    launch_group(d, d->groups[gi], st);
    dag_cuda(cudaEventRecord(ev[gi + 1], st), "profile event");
  }
  dag_cuda(cudaEventSynchronize(ev[G]), "profile sync");
  std::vector<dag_group_profile_t> out(G);
  for (size_t gi = 0; gi < G; ++gi) {
    const group_t& g = d->groups[gi];
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[gi], ev[gi + 1]);
    out[gi] = {(int)g.kind, g.wave, ms, g.flops, g.bytes};
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return out;
}

int dag_num_groups(const dag_t* d) { return (int)d->groups.size(); }

void dag_destroy(dag_t* d) {
  if (!d) return;
  cudaDeviceSynchronize();
  if (d->exec) cudaGraphExecDestroy(d->exec);
  if (d->graph) cudaGraphDestroy(d->graph);
  for (auto& g : d->groups) {
    if (g.stream_plan) bbx_stream_plan_destroy(g.stream_plan);
    if (g.tc_plan) bbx_tc_plan_destroy(g.tc_plan);
    if (g.gather_plan) bbx::gather_plan_destroy(g.gather_plan);
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

// 1 when `tid` is a block the DAG reads in place from storage (an input that
// no command of the DAG writes), 0 otherwise.
int dag_is_input(const dag_t* d, tid_t tid) {
  auto it = d->tensors.find(tid);
  return it != d->tensors.end() && it->second.external && it->second.def < 0 ? 1 : 0;
}

// Tile of each launch group (128, 256, 512 = 2-SM pair) for tensor-core
// groups, 0 for the others.
std::vector<int> dag_group_tiles(const dag_t* d) {
  std::vector<int> out;
  for (auto& g : d->groups) out.push_back(g.kind == G_TC && g.tc_plan ? bbx_tc_plan_tile_n(g.tc_plan) : 0);
  return out;
}

void tile_record(bool on) {
  std::lock_guard<std::mutex> lk(g_tile_mu);
  g_tile_rec = on;
  if (on) g_tile_samples.clear();
}

std::vector<std::pair<op_features_t, float>> tile_samples() {
  std::lock_guard<std::mutex> lk(g_tile_mu);
  return g_tile_samples;
}

}  // namespace bbts
