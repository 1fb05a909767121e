// C ABI of the runtime (declared in include/bbts_b200.h). Exceptions never
// cross the ABI: they become BBX_ERR_* codes with the message in bbx_last_error.
#include <cstring>
#include <sstream>
#include <stdexcept>
#include "bbts_b200.h"
#include "common.h"
#include "runtime.h"
#include "compiler.h"
#include <fstream>

using namespace bbts;

struct bbx_rt {
  runtime_t rt;
};
struct bbx_dag {
  dag_t* d = nullptr;
};

namespace bbts {
void* dag_tensor(const dag_t* d, tid_t tid, tensor_meta_t* meta);
size_t dag_payload_bytes(const dag_t* d, tid_t tid);
int dag_is_input(const dag_t* d, tid_t tid);
std::vector<int> dag_group_tiles(const dag_t* d);
runtime_t* rt_of(bbx_rt* rt) { return &rt->rt; }
}

#define RT_TRY(...)                                                      \
  try {                                                                  \
    __VA_ARGS__;                                                         \
    return BBX_OK;                                                       \
  } catch (const std::exception& e) {                                    \
    return bbx::set_error(BBX_ERR_INVALID, "%s", e.what());              \
  } catch (...) {                                                        \
    return bbx::set_error(BBX_ERR_INVALID, "unknown exception");         \
  }

static std::vector<std::string> split_types(const char* s) {
  std::vector<std::string> out;
  if (!s) return out;
  std::stringstream ss(s);
  std::string item;
  while (std::getline(ss, item, ','))
    if (!item.empty()) out.push_back(item);
  return out;
}

static std::vector<command_param_t> to_params(const uint32_t* p, int n) {
  std::vector<command_param_t> out(n);
  for (int i = 0; i < n; ++i) out[i].u = p[i];
  return out;
}

extern "C" {

int bbx_rt_create(bbx_rt_t** out) {
  if (!out) return bbx::set_error(BBX_ERR_INVALID, "null out");
  RT_TRY(*out = new bbx_rt());
}

int bbx_rt_destroy(bbx_rt_t* rt) {
  RT_TRY(delete rt);
}

int bbx_rt_stream(bbx_rt_t* rt, void** s) {
  if (!rt || !s) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  *s = (void*)rt->rt.stream;
  return BBX_OK;
}

int bbx_rt_fmt_id(bbx_rt_t* rt, const char* name) {
  if (!rt || !name) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  return rt->rt.tf->get_tensor_ftm(name);
}

int bbx_rt_find_impl(bbx_rt_t* rt, const char* ud_name, const char* in_types, const char* out_types,
                     int require_gpu, int* ud_id, int* impl_id) {
  if (!rt || !ud_name || !ud_id || !impl_id) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  auto m = rt->rt.udm->get_matcher_for(ud_name);
  if (!m) return bbx::set_error(BBX_ERR_NOT_FOUND, "no ud function named %s", ud_name);
  ud_impl_t* impl = m->findMatch(split_types(in_types), split_types(out_types), require_gpu != 0);
  if (!impl) return bbx::set_error(BBX_ERR_NOT_FOUND, "no impl of %s for (%s) -> (%s)", ud_name, in_types, out_types);
  *ud_id = impl->impl_id.ud_id;
  *impl_id = impl->impl_id.impl_id;
  return BBX_OK;
}

int bbx_rt_impl_name(bbx_rt_t* rt, int ud_id, int impl_id, char* buf, size_t len) {
  if (!rt) return bbx::set_error(BBX_ERR_INVALID, "null runtime");
  ud_impl_t* impl = rt->rt.udm->get_fn_impl({ud_id, impl_id});
  if (!impl) return bbx::set_error(BBX_ERR_NOT_FOUND, "unknown impl (%d,%d)", ud_id, impl_id);
  if (buf && len) {
    size_t n = std::min(len - 1, impl->impl_name.size());
    memcpy(buf, impl->impl_name.data(), n);
    buf[n] = 0;
  }
  return BBX_OK;
}

int bbx_rt_complexity(bbx_rt_t* rt, int ud_id, int impl_id, const uint32_t* params, int n_params,
                      const void* in_metas, int n_in, unsigned long long* hint) {
  if (!rt || !hint) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  ud_impl_t* impl = rt->rt.udm->get_fn_impl({ud_id, impl_id});
  if (!impl) return bbx::set_error(BBX_ERR_NOT_FOUND, "unknown impl (%d,%d)", ud_id, impl_id);
  RT_TRY({
    std::vector<tensor_meta_t> metas(n_in);
    for (int i = 0; i < n_in; ++i) memcpy(&metas[i], (const char*)in_metas + i * sizeof(tensor_meta_t), sizeof(tensor_meta_t));
    auto p = to_params(params, n_params);
    ud_impl_t::tensor_params_t tp;
    tp._params = command_param_list_t{p.data(), p.size()};
    ud_impl_t::meta_args_t ma(metas);
    *hint = impl->get_complexity_hint(tp, ma);
  });
}

int bbx_rt_tensor_put(bbx_rt_t* rt, int tid, const void* meta, const void* src, size_t bytes,
                      int src_on_device) {
  if (!rt || !meta) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  RT_TRY({
    tensor_meta_t m;
    memcpy(&m, meta, sizeof(m));
    tensor_t* t = rt->rt.storage->create(tid, m);
    size_t need = rt->rt.tf->get_payload_size(m);
    if (src && bytes) {
      if (bytes > need) throw std::runtime_error("tensor_put: more bytes than the meta describes");
      cudaError_t e = cudaMemcpyAsync(t->_meta.payload(), src, bytes,
                                      src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                      rt->rt.stream);
      if (e != cudaSuccess) throw std::runtime_error(std::string("tensor_put copy: ") + cudaGetErrorString(e));
      e = cudaStreamSynchronize(rt->rt.stream);
      if (e != cudaSuccess) throw std::runtime_error(std::string("tensor_put sync: ") + cudaGetErrorString(e));
    }
  });
}

int bbx_rt_tensor_get(bbx_rt_t* rt, int tid, void* meta_out, void* dst, size_t cap, int dst_on_device) {
  if (!rt) return bbx::set_error(BBX_ERR_INVALID, "null runtime");
  tensor_t* t = rt->rt.storage->get(tid);
  if (!t) return bbx::set_error(BBX_ERR_NOT_FOUND, "no tensor %d", tid);
  RT_TRY({
    if (meta_out) memcpy(meta_out, &t->_meta, sizeof(tensor_meta_t));
    size_t have = rt->rt.tf->get_payload_size(t->_meta);
    size_t n = std::min(have, cap);
    if (dst && n) {
      void* src = rt->rt.storage->caller_payload(tid, nullptr, false);  // reloaded if spilled
      cudaError_t e = cudaMemcpyAsync(dst, src, n,
                                      dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                      rt->rt.stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(rt->rt.stream);
      if (e != cudaSuccess) throw std::runtime_error(std::string("tensor_get copy: ") + cudaGetErrorString(e));
    }
  });
}

int bbx_rt_tensor_payload(bbx_rt_t* rt, int tid, void** ptr, size_t* bytes) {
  if (!rt) return bbx::set_error(BBX_ERR_INVALID, "null runtime");
  if (!rt->rt.storage->get(tid)) return bbx::set_error(BBX_ERR_NOT_FOUND, "no tensor %d", tid);
  RT_TRY({
    size_t n = 0;
    void* p = rt->rt.storage->caller_payload(tid, &n, true);  // reloaded if spilled; the caller may write
    if (ptr) *ptr = p;
    if (bytes) *bytes = n;
  });
}

int bbx_rt_set_storage_budget(bbx_rt_t* rt, unsigned long long device_bytes, unsigned long long host_bytes,
                              const char* spill_file) {
  if (!rt) return bbx::set_error(BBX_ERR_INVALID, "null runtime");
  RT_TRY(rt->rt.storage->set_budget((size_t)device_bytes, (size_t)host_bytes, spill_file ? spill_file : ""));
}

int bbx_rt_spill_stats(bbx_rt_t* rt, unsigned long long* out, int n) {
  if (!rt || !out) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  spill_stats_t s = rt->rt.storage->stats();
  const unsigned long long v[10] = {s.evictions,        s.reloads,         s.d2h_bytes,      s.h2d_bytes,
                                    s.file_write_bytes, s.file_read_bytes, s.clean_evictions, s.resident_bytes,
                                    s.peak_resident_bytes, s.host_bytes};
  for (int i = 0; i < n && i < 10; ++i) out[i] = v[i];
  return BBX_OK;
}

int bbx_rt_tensor_count(bbx_rt_t* rt) { return rt ? (int)rt->rt.storage->size() : -1; }

int bbx_rt_tensor_remove(bbx_rt_t* rt, int tid) {
  if (!rt) return bbx::set_error(BBX_ERR_INVALID, "null runtime");
  return rt->rt.storage->remove(tid) ? BBX_OK : bbx::set_error(BBX_ERR_NOT_FOUND, "no tensor %d", tid);
}

static int check_order(bbx_rt_t* rt, int cmd_id) {
  if (!rt->rt.commands.empty() && rt->rt.commands.back()->id >= cmd_id)
    return bbx::set_error(BBX_ERR_INVALID, "command ids must increase (got %d after %d)", cmd_id,
                          rt->rt.commands.back()->id);
  return BBX_OK;
}

int bbx_rt_queue_apply(bbx_rt_t* rt, int cmd_id, int ud_id, int impl_id, const uint32_t* params,
                       int n_params, const int* in_tids, int n_in, const int* out_tids, int n_out) {
  if (!rt || n_in < 0 || n_out < 1) return bbx::set_error(BBX_ERR_INVALID, "bad apply");
  if (int rc = check_order(rt, cmd_id)) return rc;
  if (!rt->rt.udm->get_fn_impl({ud_id, impl_id})) return bbx::set_error(BBX_ERR_NOT_FOUND, "unknown impl (%d,%d)", ud_id, impl_id);
  RT_TRY({
    std::vector<command_t::tid_node_id_t> in, out;
    for (int i = 0; i < n_in; ++i) in.push_back({in_tids[i], 0});
    for (int i = 0; i < n_out; ++i) out.push_back({out_tids[i], 0});
    rt->rt.commands.push_back(command_t::create_apply(cmd_id, {ud_id, impl_id}, true, to_params(params, n_params), in, out));
  });
}

int bbx_rt_queue_reduce(bbx_rt_t* rt, int cmd_id, int ud_id, int impl_id, const uint32_t* params,
                        int n_params, const int* in_tids, int n_in, int out_tid) {
  if (!rt || n_in < 1) return bbx::set_error(BBX_ERR_INVALID, "bad reduce");
  if (int rc = check_order(rt, cmd_id)) return rc;
  ud_func_t* f = rt->rt.udm->get_udf(ud_id);
  if (!f || !rt->rt.udm->get_fn_impl({ud_id, impl_id})) return bbx::set_error(BBX_ERR_NOT_FOUND, "unknown impl (%d,%d)", ud_id, impl_id);
  // REDUCE needs an associative and commutative ud (src/commands/command_loader.h:146)
  if (!f->is_ass || !f->is_com) return bbx::set_error(BBX_ERR_INVALID, "REDUCE needs an associative, commutative ud (%s is not)", f->ud_name.c_str());
  RT_TRY({
    std::vector<command_t::tid_node_id_t> in;
    for (int i = 0; i < n_in; ++i) in.push_back({in_tids[i], 0});
    rt->rt.commands.push_back(command_t::create_reduce(cmd_id, {ud_id, impl_id}, true, to_params(params, n_params), in, {out_tid, 0}));
  });
}

int bbx_rt_queue_delete(bbx_rt_t* rt, int cmd_id, const int* tids, int n) {
  if (!rt || n < 1) return bbx::set_error(BBX_ERR_INVALID, "bad delete");
  if (int rc = check_order(rt, cmd_id)) return rc;
  RT_TRY({
    std::vector<command_t::tid_node_id_t> in;
    for (int i = 0; i < n; ++i) in.push_back({tids[i], 0});
    rt->rt.commands.push_back(command_t::create_delete(cmd_id, in));
  });
}

int bbx_rt_clear_commands(bbx_rt_t* rt) {
  if (!rt) return bbx::set_error(BBX_ERR_INVALID, "null runtime");
  rt->rt.commands.clear();
  return BBX_OK;
}

int bbx_rt_num_commands(bbx_rt_t* rt) { return rt ? (int)rt->rt.commands.size() : -1; }

static command_id_t next_id(bbx_rt_t* rt) {
  return rt->rt.commands.empty() ? 0 : rt->rt.commands.back()->id + 1;
}

int bbx_rt_load_sbbts(bbx_rt_t* rt, const char* path, int* n_added) {
  if (!rt || !path) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  RT_TRY({
    std::ifstream f(path);
    if (!f.is_open()) throw std::runtime_error(std::string("cannot open ") + path);
    compile_source_file_t src;
    src.read(f);
    auto cmds = compile_single_node(src, *rt->rt.udm, next_id(rt));
    if (n_added) *n_added = (int)cmds.size();
    for (auto& c : cmds) rt->rt.commands.push_back(std::move(c));
  });
}

int bbx_rt_load_bbts(bbx_rt_t* rt, const char* path, int* n_added) {
  if (!rt || !path) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  RT_TRY({
    parsed_command_list_t list;
    if (!list.deserialize(path)) throw std::runtime_error(std::string("cannot open ") + path);
    auto cmds = load_parsed(list, *rt->rt.udm, next_id(rt));
    if (n_added) *n_added = (int)cmds.size();
    for (auto& c : cmds) rt->rt.commands.push_back(std::move(c));
  });
}

int bbx_rt_save_bbts(bbx_rt_t* rt, const char* path) {
  if (!rt || !path) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  RT_TRY({
    parsed_command_list_t list;
    for (auto& cp : rt->rt.commands) {
      const command_t& c = *cp;
      parsed_command_t p;
      if (c.is_delete()) p.type = parsed_command_t::op_type_t::DELETE;
      else if (c.is_reduce()) p.type = parsed_command_t::op_type_t::REDUCE;
      else if (c.is_apply()) p.type = parsed_command_t::op_type_t::APPLY;
      else p.type = parsed_command_t::op_type_t::MOVE;
      if (!c.is_delete()) {
        ud_impl_t* impl = rt->rt.udm->get_fn_impl(c.fun_id);
        if (impl) {
          p.def.ud_name = impl->ud_name;
          p.def.input_types = impl->inputTypes;
          p.def.output_types = impl->outputTypes;
          p.def.is_gpu = impl->is_gpu;
        }
      }
      for (size_t i = 0; i < c.get_num_inputs(); ++i) p.inputs.push_back({c.get_input(i).tid, c.get_input(i).node});
      for (size_t i = 0; i < c.get_num_outputs(); ++i) p.outputs.push_back({c.get_output(i).tid, c.get_output(i).node});
      auto prm = c.get_parameters();
      p.parameters.assign(prm.begin(), prm.end());
      list.commands.push_back(std::move(p));
    }
    if (!list.serialize(path)) throw std::runtime_error(std::string("cannot write ") + path);
  });
}

int bbx_rt_run(bbx_rt_t* rt, int policy) {
  if (!rt) return bbx::set_error(BBX_ERR_INVALID, "null runtime");
  RT_TRY({
    rt->rt.run_per_op(policy, nullptr);
    cudaError_t e = cudaStreamSynchronize(rt->rt.stream);
    if (e != cudaSuccess) throw std::runtime_error(std::string("run: ") + cudaGetErrorString(e));
  });
}

int bbx_rt_set_workers(bbx_rt_t* rt, int workers) {
  if (!rt) return bbx::set_error(BBX_ERR_INVALID, "null runtime");
  if (workers < 1 || workers > 16) return bbx::set_error(BBX_ERR_INVALID, "workers must be in [1, 16]");
  rt->rt.workers = workers;
  return BBX_OK;
}

int bbx_rt_record(bbx_rt_t* rt, int policy, float* features, float* latency_us, double* hints, int cap,
                  int* n_out) {
  if (!rt) return bbx::set_error(BBX_ERR_INVALID, "null runtime");
  RT_TRY({
    std::vector<std::pair<op_features_t, float>> rec;
    rt->rt.run_per_op(policy, &rec);
    int n = std::min<int>(cap, (int)rec.size());
    for (int i = 0; i < n; ++i) {
      if (features) memcpy(features + 12 * i, rec[i].first.f, 12 * sizeof(float));
      if (latency_us) latency_us[i] = rec[i].second;
      if (hints) hints[i] = rec[i].first.hint;
    }
    if (n_out) *n_out = (int)rec.size();
  });
}

int bbx_dag_build(bbx_rt_t* rt, int policy, int tile_n, bbx_dag_t** out) {
  if (!rt || !out) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  RT_TRY({
    cudaError_t e = cudaStreamSynchronize(rt->rt.stream);
    if (e != cudaSuccess) throw std::runtime_error(std::string("dag_build: ") + cudaGetErrorString(e));
    auto* d = new bbx_dag();
    try {
      d->d = dag_build(&rt->rt, policy, tile_n);
    } catch (...) {
      delete d;
      throw;
    }
    *out = d;
  });
}

int bbx_tile_record(int on) {
  bbts::tile_record(on != 0);
  return BBX_OK;
}

int bbx_tile_samples(float* features, float* latency_us, int cap, int* n_out) {
  auto v = bbts::tile_samples();
  const int n = (int)v.size();
  for (int i = 0; i < n && i < cap; ++i) {
    if (features) std::memcpy(features + 12 * (size_t)i, v[i].first.f, sizeof(float) * 12);
    if (latency_us) latency_us[i] = v[i].second;
  }
  if (n_out) *n_out = n;
  return BBX_OK;
}

int bbx_dag_launch(bbx_dag_t* dag, void* stream) {
  if (!dag) return bbx::set_error(BBX_ERR_INVALID, "null dag");
  RT_TRY(dag_launch(dag->d, (cudaStream_t)stream));
}

int bbx_dag_destroy(bbx_dag_t* dag) {
  if (!dag) return BBX_OK;
  RT_TRY({
    dag_destroy(dag->d);
    delete dag;
  });
}

int bbx_dag_stats(bbx_dag_t* dag, double* flops, double* bytes, int* waves, int* tc_launches,
                  int* stream_launches, int* other_launches, size_t* arena_bytes) {
  if (!dag) return bbx::set_error(BBX_ERR_INVALID, "null dag");
  dag_stats_t s = dag_stats(dag->d);
  if (flops) *flops = s.flops;
  if (bytes) *bytes = s.bytes;
  if (waves) *waves = s.waves;
  if (tc_launches) *tc_launches = s.tc_launches;
  if (stream_launches) *stream_launches = s.stream_launches;
  if (other_launches) *other_launches = s.opaque_launches;
  if (arena_bytes) *arena_bytes = s.arena_bytes;
  return BBX_OK;
}

int bbx_dag_profile(bbx_dag_t* dag, void* stream, int cap, int* kinds, int* waves, float* ms, double* flops,
                    double* bytes, int* n_out) {
  if (!dag) return bbx::set_error(BBX_ERR_INVALID, "null dag");
  if (cap <= 0) {  // count only, nothing runs
    if (n_out) *n_out = dag_num_groups(dag->d);
    return BBX_OK;
  }
  RT_TRY({
    auto prof = dag_profile(dag->d, (cudaStream_t)stream);
    const int n = std::min<int>(cap, (int)prof.size());
    for (int i = 0; i < n; ++i) {
      if (kinds) kinds[i] = prof[i].kind;
      if (waves) waves[i] = prof[i].wave;
      if (ms) ms[i] = prof[i].ms;
      if (flops) flops[i] = prof[i].flops;
      if (bytes) bytes[i] = prof[i].bytes;
    }
    if (n_out) *n_out = (int)prof.size();
  });
}

int bbx_dag_tensor(bbx_dag_t* dag, int tid, void** ptr, void* meta_out) {
  if (!dag) return bbx::set_error(BBX_ERR_INVALID, "null dag");
  tensor_meta_t m;
  void* p = dag_tensor(dag->d, tid, &m);
  if (!p && !meta_out) return bbx::set_error(BBX_ERR_NOT_FOUND, "DAG has no tensor %d", tid);
  if (ptr) *ptr = p;
  if (meta_out) memcpy(meta_out, &m, sizeof(m));
  return p ? BBX_OK : bbx::set_error(BBX_ERR_NOT_FOUND, "DAG has no tensor %d", tid);
}

int bbx_dag_read(bbx_dag_t* dag, int tid, void* host_dst, size_t cap) {
  if (!dag || !host_dst) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  tensor_meta_t m;
  void* p = dag_tensor(dag->d, tid, &m);
  if (!p) return bbx::set_error(BBX_ERR_NOT_FOUND, "DAG has no tensor %d", tid);
  RT_TRY({
    size_t n = std::min(cap, dag->d ? dag_payload_bytes(dag->d, tid) : 0);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(host_dst, p, n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) throw std::runtime_error(std::string("dag_read: ") + cudaGetErrorString(e));
  });
}

int bbx_rt_set_dag_stream_kernel(bbx_rt_t* rt, int kernel) {
  if (!rt) return bbx::set_error(BBX_ERR_INVALID, "null runtime");
  if (kernel != BBX_STREAM_KERNEL_AUTO && kernel != BBX_STREAM_KERNEL_REGISTER && kernel != BBX_STREAM_KERNEL_PER_WAVE)
    return bbx::set_error(BBX_ERR_INVALID, "dag stream kernel %d", kernel);
  rt->rt.dag_stream_kernel = kernel;
  return BBX_OK;
}

int bbx_dag_register_waves(bbx_dag_t* dag) {
  if (!dag) return bbx::set_error(BBX_ERR_INVALID, "null dag");
  return dag_stats(dag->d).register_waves;
}

int bbx_dag_write(bbx_dag_t* dag, int tid, const void* src, size_t bytes, int src_on_device, void* stream) {
  if (!dag || (!src && bytes)) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  void* p = dag_tensor(dag->d, tid, nullptr);
  if (!p) return bbx::set_error(BBX_ERR_NOT_FOUND, "DAG has no tensor %d", tid);
  if (!dag_is_input(dag->d, tid))
    return bbx::set_error(BBX_ERR_INVALID, "tensor %d is not an input the DAG reads in place", tid);
  if (bytes > dag_payload_bytes(dag->d, tid))
    return bbx::set_error(BBX_ERR_INVALID, "dag_write: %zu bytes into a %zu-byte block", bytes,
                          dag_payload_bytes(dag->d, tid));
  if (!bytes) return BBX_OK;
  cudaError_t e = cudaMemcpyAsync(p, src, bytes, src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                  (cudaStream_t)stream);
  return e == cudaSuccess ? BBX_OK : bbx::set_error(BBX_ERR_CUDA, "dag_write: %s", cudaGetErrorString(e));
}

int bbx_dag_fetch(bbx_dag_t* dag, int tid, void* dst, size_t cap, int dst_on_device, void* stream) {
  if (!dag || (!dst && cap)) return bbx::set_error(BBX_ERR_INVALID, "null argument");
  void* p = dag_tensor(dag->d, tid, nullptr);
  if (!p) return bbx::set_error(BBX_ERR_NOT_FOUND, "DAG has no tensor %d", tid);
  const size_t n = std::min(cap, dag_payload_bytes(dag->d, tid));
  if (!n) return BBX_OK;
  cudaError_t e = cudaMemcpyAsync(dst, p, n, dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                  (cudaStream_t)stream);
  return e == cudaSuccess ? BBX_OK : bbx::set_error(BBX_ERR_CUDA, "dag_fetch: %s", cudaGetErrorString(e));
}

int bbx_dag_group_tiles(bbx_dag_t* dag, int cap, int* tiles, int* n_out) {
  if (!dag) return bbx::set_error(BBX_ERR_INVALID, "null dag");
  auto t = dag_group_tiles(dag->d);
  for (int i = 0; i < cap && i < (int)t.size(); ++i) tiles[i] = t[i];
  if (n_out) *n_out = (int)t.size();
  return BBX_OK;
}

}  // extern "C"
