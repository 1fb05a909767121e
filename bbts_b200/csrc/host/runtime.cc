// Runtime: block storage, per-op runner and the grouped DAG executor.
#include "runtime.h"

#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstring>
#include <cmath>
#include <numeric>
#include <set>
#include <stdexcept>

namespace bbts {

namespace {
void cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
void bbx_ok(int rc) {
  if (rc != 0) {
    char buf[1024];
    bbx_last_error(buf, sizeof(buf));
    throw std::runtime_error(std::string("bbts_b200: ") + buf);
  }
}
bool starts_with(const std::string& s, const char* p) { return s.rfind(p, 0) == 0; }
}  // namespace

// ------------------------------------------------------------------ storage
namespace {
constexpr size_t kStageBytes = 64ull << 20;  // file-tier staging buffer
constexpr size_t kFileAlign = 4096;
void wait_on(cudaStream_t st, const event_ptr& e) {
  if (e) cuda_ok(cudaStreamWaitEvent(st, e.get(), 0), "cudaStreamWaitEvent(storage)");
}
}  // namespace

block_storage_t::block_storage_t(tensor_factory_ptr_t tf, cudaStream_t st) : _tf(std::move(tf)), _st(st) {
  int dev = 0;
  cuda_ok(cudaGetDevice(&dev), "cudaGetDevice");
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cuda_ok(cudaMemPoolCreate(&_pool, &props), "cudaMemPoolCreate(blocks)");
  unsigned long long keep = ~0ULL;  // never trim at synchronisation points
  cuda_ok(cudaMemPoolSetAttribute(_pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool release threshold");
}

block_storage_t::~block_storage_t() {
  for (auto& kv : _blocks)
    if (kv.second.owned && kv.second.resident && kv.second.payload) cudaFreeAsync(kv.second.payload, _st);
  cudaStreamSynchronize(_st);
  if (_out_st) {
    cudaStreamSynchronize(_out_st);
    cudaStreamDestroy(_out_st);
  }
  _blocks.clear();
  _host_cache.clear();
  _freed.reset();
  for (void* h : _host_all) cudaFreeHost(h);
  if (_stage) cudaFreeHost(_stage);
  if (_fd >= 0) {
    close(_fd);
    unlink(_file.c_str());  // the spill file is scratch
  }
  if (_pool) cudaMemPoolDestroy(_pool);
}

event_ptr block_storage_t::_record(cudaStream_t st) {
  cudaEvent_t e;
  cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate(storage)");
  cudaError_t r = cudaEventRecord(e, st);
  if (r != cudaSuccess) {
    cudaEventDestroy(e);
    cuda_ok(r, "cudaEventRecord(storage)");
  }
  return event_ptr(e, [](cudaEvent_t x) { cudaEventDestroy(x); });
}

void block_storage_t::_lru_remove(block_t& b) {
  if (b.in_lru) {
    _lru[b.lru_list].erase(b.lru_it);
    b.in_lru = false;
  }
}

// Most recently used position of the list the block belongs in.
void block_storage_t::_lru_touch(tid_t tid, block_t& b) {
  _lru_remove(b);
  if (!_budget || b.pins || !b.resident || !b.owned) return;
  b.lru_list = b.readers_left == 0 ? 1 : 0;
  _lru[b.lru_list].push_front(tid);
  b.lru_it = _lru[b.lru_list].begin();
  b.in_lru = true;
}

void block_storage_t::_pin(tid_t, block_t& b) {
  _lru_remove(b);
  ++b.pins;
}

void block_storage_t::_unpin(tid_t tid, block_t& b) {
  if (b.pins > 0) --b.pins;
  if (b.pins == 0) _lru_touch(tid, b);
}

void block_storage_t::set_readers_left(tid_t tid, int n) {
  std::lock_guard<std::recursive_mutex> lk(_m);
  auto it = _blocks.find(tid);
  if (it == _blocks.end()) return;
  block_t& b = it->second;
  const bool moved = b.in_lru && (b.lru_list == 1) != (n == 0);
  b.readers_left = n;
  if (moved) _lru_touch(tid, b);
}

// The host copy goes back to the pinned cache; the D2H that reuses it waits
// for the last H2D that read it.
void block_storage_t::_drop_copies(block_t& b) {
  if (b.host) {
    _host_cache.insert({b.bytes, {b.host, b.host_read}});
    _stats.host_bytes -= b.bytes;
    b.host = nullptr;
  }
  b.host_valid = false;
  b.file_valid = false;
  b.copied.reset();
  b.host_read.reset();
}

void block_storage_t::_free_payload(block_t& b, cudaStream_t st) {
  _lru_remove(b);
  if (b.owned && b.resident && b.payload) {
    cudaFreeAsync(b.payload, st);  // stream-ordered
    _stats.resident_bytes -= b.bytes;
  }
  b.payload = nullptr;
  _drop_copies(b);
}

void* block_storage_t::_host_alloc(size_t bytes, event_ptr* last_read) {
  auto it = _host_cache.find(bytes);
  if (it != _host_cache.end()) {
    void* p = it->second.first;
    *last_read = it->second.second;
    _host_cache.erase(it);
    return p;
  }
  void* p = nullptr;
  cuda_ok(cudaHostAlloc(&p, bytes, cudaHostAllocDefault), "cudaHostAlloc(spill)");
  _host_all.push_back(p);
  last_read->reset();
  return p;
}

// File tier: chunks through a pinned staging buffer, synchronous like the
// reference's pwrite / pread (nvme_storage.cc:167,577).
void block_storage_t::_file_io(block_t& b, bool write, cudaStream_t st) {
  if (!_stage) cuda_ok(cudaHostAlloc(&_stage, kStageBytes, cudaHostAllocDefault), "cudaHostAlloc(stage)");
  if (write && b.file_off < 0) {
    b.file_off = _file_end;
    _file_end += (long long)((b.bytes + kFileAlign - 1) / kFileAlign * kFileAlign);
  }
  for (size_t o = 0; o < b.bytes; o += kStageBytes) {
    const size_t n = std::min(kStageBytes, b.bytes - o);
    char* dev = (char*)b.payload + o;
    if (write) {
      cuda_ok(cudaMemcpyAsync(_stage, dev, n, cudaMemcpyDeviceToHost, st), "spill D2H (file)");
      cuda_ok(cudaStreamSynchronize(st), "spill D2H sync");
      for (size_t w = 0; w < n;) {
        ssize_t r = pwrite(_fd, (char*)_stage + w, n - w, b.file_off + (long long)(o + w));
        if (r <= 0) throw std::runtime_error("block storage: pwrite to the spill file failed: " + std::string(strerror(errno)));
        w += (size_t)r;
      }
      _stats.file_write_bytes += n;
    } else {
      for (size_t w = 0; w < n;) {
        ssize_t r = pread(_fd, (char*)_stage + w, n - w, b.file_off + (long long)(o + w));
        if (r <= 0) throw std::runtime_error("block storage: pread from the spill file failed");
        w += (size_t)r;
      }
      cuda_ok(cudaMemcpyAsync(dev, _stage, n, cudaMemcpyHostToDevice, st), "reload H2D (file)");
      cuda_ok(cudaStreamSynchronize(st), "reload H2D sync");
      _stats.file_read_bytes += n;
    }
  }
}

// Evicts one resident, unpinned, owned block: its bytes are copied out (unless
// a copy from an earlier eviction is still valid) after its last uses, then
// the payload is freed on the copy stream.
void block_storage_t::_evict(tid_t, block_t& b) {
  for (auto& u : b.uses) wait_on(_out_st, u.second);
  if (b.caller_may_write) wait_on(_out_st, _record(_st));
  if (b.host_valid || b.file_valid) {
    ++_stats.clean_evictions;
  } else if (_stats.host_bytes + b.bytes <= _host_budget) {
    event_ptr last_read;
    b.host = _host_alloc(b.bytes, &last_read);
    wait_on(_out_st, last_read);
    cuda_ok(cudaMemcpyAsync(b.host, b.payload, b.bytes, cudaMemcpyDeviceToHost, _out_st), "spill D2H");
    b.copied = _record(_out_st);
    b.host_valid = true;
    _stats.host_bytes += b.bytes;
    _stats.d2h_bytes += b.bytes;
  } else if (_fd >= 0) {
    _file_io(b, true, _out_st);
    b.file_valid = true;
    _stats.d2h_bytes += b.bytes;
  } else {
    throw std::runtime_error("block storage: the host spill budget is exhausted and no spill file is set");
  }
  cuda_ok(cudaFreeAsync(b.payload, _out_st), "cudaFreeAsync(spill)");
  _lru_remove(b);
  b.payload = nullptr;
  b.tensor()->_meta.set_payload(nullptr);
  b.resident = false;
  b.uses.clear();
  b.loaded.reset();
  b.caller_may_write = false;
  _stats.resident_bytes -= b.bytes;
  ++_stats.evictions;
}

void block_storage_t::_make_room(size_t need, cudaStream_t st) {
  if (!_budget) return;
  if (need > _budget)
    throw std::runtime_error("block storage: a request of " + std::to_string(need) +
                             " bytes exceeds the device budget of " + std::to_string(_budget) + " bytes");
  bool evicted = false;
  while (_stats.resident_bytes + need > _budget) {
    if (_lru[0].empty() && _lru[1].empty())
      throw std::runtime_error("block storage: the device budget of " + std::to_string(_budget) +
                               " bytes is held by blocks in use; " + std::to_string(need) + " more bytes needed");
    tid_t v = _lru[1].empty() ? _lru[0].back() : _lru[1].back();
    _evict(v, _blocks.at(v));
    evicted = true;
  }
  if (evicted) {
    _freed = _record(_out_st);
    wait_on(st, _freed);  // the allocation below may reuse the freed memory
  }
}

void block_storage_t::_reload(block_t& b, cudaStream_t st) {
  _make_room(b.bytes, st);
  void* p = nullptr;
  cuda_ok(cudaMallocFromPoolAsync(&p, b.bytes, _pool, st), "cudaMallocFromPoolAsync(reload)");
  b.payload = p;
  if (b.host_valid) {
    wait_on(st, b.copied);
    cuda_ok(cudaMemcpyAsync(p, b.host, b.bytes, cudaMemcpyHostToDevice, st), "reload H2D");
    b.host_read = _record(st);
  } else if (b.file_valid) {
    _file_io(b, false, st);
  } else {
    throw std::runtime_error("block storage: a spilled block has no copy to reload");
  }
  b.tensor()->_meta.set_payload(p);
  b.resident = true;
  b.loaded = _record(st);
  b.loaded_st = st;
  _stats.resident_bytes += b.bytes;
  _stats.peak_resident_bytes = std::max(_stats.peak_resident_bytes, _stats.resident_bytes);
  _stats.h2d_bytes += b.bytes;
  ++_stats.reloads;
}

tensor_t* block_storage_t::create(tid_t tid, const tensor_meta_t& meta, cudaStream_t st) {
  if (!st) st = _st;
  std::lock_guard<std::recursive_mutex> lk(_m);
  auto it = _blocks.find(tid);
  if (it != _blocks.end()) {
    _free_payload(it->second, st);
    _blocks.erase(it);
  }
  size_t bytes = _tf->get_payload_size(meta);
  _make_room(bytes, st);
  void* p = nullptr;
  if (bytes) cuda_ok(cudaMallocFromPoolAsync(&p, bytes, _pool, st), "cudaMallocFromPoolAsync(block)");
  auto& b = _blocks[tid];
  b.header.reset(new char[sizeof(tensor_meta_t)]);
  std::memcpy(b.header.get(), &meta, sizeof(tensor_meta_t));
  b.tensor()->_meta.set_payload(p);
  b.payload = p;
  b.bytes = bytes;
  b.owned = true;
  _stats.resident_bytes += bytes;
  _stats.peak_resident_bytes = std::max(_stats.peak_resident_bytes, _stats.resident_bytes);
  if (_budget) {
    if (_in_command) {
      _pin(tid, b);
      _scope.push_back(tid);
    } else {
      b.caller_may_write = true;  // filled by work the caller queues on the runtime stream
      _unpin(tid, b);
    }
  }
  return b.tensor();
}

tensor_t* block_storage_t::create_view(tid_t tid, const tensor_meta_t& meta, void* payload, size_t bytes) {
  std::lock_guard<std::recursive_mutex> lk(_m);
  auto it = _blocks.find(tid);
  if (it != _blocks.end()) {
    _free_payload(it->second, _st);
    _blocks.erase(it);
  }
  auto& b = _blocks[tid];
  b.header.reset(new char[sizeof(tensor_meta_t)]);
  std::memcpy(b.header.get(), &meta, sizeof(tensor_meta_t));
  b.tensor()->_meta.set_payload(payload);
  b.payload = payload;
  b.bytes = bytes;
  b.owned = false;  // never counted, never evicted
  return b.tensor();
}

tensor_t* block_storage_t::get(tid_t tid) {
  std::lock_guard<std::recursive_mutex> lk(_m);
  auto it = _blocks.find(tid);
  return it == _blocks.end() ? nullptr : it->second.tensor();
}

block_t* block_storage_t::block(tid_t tid) {
  std::lock_guard<std::recursive_mutex> lk(_m);
  auto it = _blocks.find(tid);
  return it == _blocks.end() ? nullptr : &it->second;
}

bool block_storage_t::remove(tid_t tid, cudaStream_t st) {
  std::lock_guard<std::recursive_mutex> lk(_m);
  auto it = _blocks.find(tid);
  if (it == _blocks.end()) return false;
  _free_payload(it->second, st ? st : _st);
  _blocks.erase(it);
  return true;
}

bool block_storage_t::assign_tid(tid_t from, tid_t to) {
  std::lock_guard<std::recursive_mutex> lk(_m);
  auto it = _blocks.find(from);
  if (it == _blocks.end() || _blocks.count(to)) return false;
  block_t b = std::move(it->second);
  _blocks.erase(it);
  if (b.in_lru) *b.lru_it = to;  // the list node moves with the block
  for (auto& t : _scope)
    if (t == from) t = to;
  _blocks[to] = std::move(b);
  return true;
}

std::vector<tid_t> block_storage_t::tids() const {
  std::vector<tid_t> out;
  for (auto& kv : _blocks) out.push_back(kv.first);
  return out;
}

void block_storage_t::set_budget(size_t device_bytes, size_t host_bytes, const std::string& file) {
  std::lock_guard<std::recursive_mutex> lk(_m);
  if (!_out_st) cuda_ok(cudaStreamCreateWithFlags(&_out_st, cudaStreamNonBlocking), "cudaStreamCreate(spill)");
  // bring every spilled block back first (its copy may be in the file being replaced)
  _budget = 0;
  for (auto& kv : _blocks)
    if (!kv.second.resident) _reload(kv.second, _st);
  _lru[0].clear();
  _lru[1].clear();
  for (auto& kv : _blocks) kv.second.in_lru = false;
  if (file != _file || !device_bytes) {
    for (auto& kv : _blocks) kv.second.file_valid = false, kv.second.file_off = -1;
    if (_fd >= 0) {
      close(_fd);
      unlink(_file.c_str());
      _fd = -1;
    }
    _file = device_bytes ? file : std::string();
    _file_end = 0;
    if (!_file.empty()) {
      _fd = open(_file.c_str(), O_CREAT | O_TRUNC | O_RDWR, 0600);
      if (_fd < 0) throw std::runtime_error("block storage: cannot open the spill file " + _file);
    }
  }
  _budget = device_bytes;
  _host_budget = host_bytes;
  _stats = spill_stats_t{};
  for (auto& kv : _blocks)
    if (kv.second.owned) _stats.resident_bytes += kv.second.bytes;
  _stats.peak_resident_bytes = _stats.resident_bytes;
  for (auto& kv : _blocks) _stats.host_bytes += kv.second.host ? kv.second.bytes : 0;
  if (_budget) {
    for (auto& kv : _blocks) {
      block_t& b = kv.second;
      if (b.owned && b.pins == 0) {
        b.caller_may_write = true;  // writers unknown: wait for the runtime stream
        _unpin(kv.first, b);
      }
    }
    _make_room(0, _st);
    _stats.peak_resident_bytes = _stats.resident_bytes;  // within the budget from here on
  }
  cuda_ok(cudaStreamSynchronize(_st), "set_budget sync");
}

void block_storage_t::begin_command() {
  std::lock_guard<std::recursive_mutex> lk(_m);
  _in_command = true;
  _scope.clear();
}

tensor_t* block_storage_t::acquire(tid_t tid, cudaStream_t st) {
  std::lock_guard<std::recursive_mutex> lk(_m);
  auto it = _blocks.find(tid);
  if (it == _blocks.end()) return nullptr;
  block_t& b = it->second;
  if (!_budget) return b.tensor();
  if (!b.resident) _reload(b, st);
  else if (b.loaded && b.loaded_st != st) wait_on(st, b.loaded);  // reloaded for a command on another stream
  if (_in_command) {
    _pin(tid, b);
    _scope.push_back(tid);
  } else if (b.in_lru) {
    _lru_touch(tid, b);
  }
  return b.tensor();
}

void block_storage_t::end_command(cudaStream_t st) {
  std::lock_guard<std::recursive_mutex> lk(_m);
  _in_command = false;
  if (!_budget || _scope.empty()) {
    _scope.clear();
    return;
  }
  event_ptr e = _record(st);
  for (tid_t t : _scope) {
    auto it = _blocks.find(t);
    if (it == _blocks.end()) continue;  // removed inside the command (a reduce temporary)
    block_t& b = it->second;
    bool found = false;
    for (auto& u : b.uses)
      if (u.first == st) u.second = e, found = true;
    if (!found) b.uses.push_back({st, e});
    _unpin(t, b);
  }
  _scope.clear();
}

void* block_storage_t::caller_payload(tid_t tid, size_t* bytes, bool will_write) {
  std::lock_guard<std::recursive_mutex> lk(_m);
  auto it = _blocks.find(tid);
  if (it == _blocks.end()) return nullptr;
  block_t& b = it->second;
  if (_budget) {
    if (!b.resident) _reload(b, _st);
    else if (b.loaded && b.loaded_st != _st) wait_on(_st, b.loaded);
    if (will_write) {
      b.caller_may_write = true;
      _drop_copies(b);
    }
    if (b.in_lru) _lru_touch(tid, b);
  }
  if (bytes) *bytes = b.bytes;
  return b.payload;
}

std::vector<tid_t> block_storage_t::hold_all() {
  std::lock_guard<std::recursive_mutex> lk(_m);
  std::vector<tid_t> held;
  if (!_budget) return held;
  try {
    for (auto& kv : _blocks) {
      block_t& b = kv.second;
      if (!b.owned) continue;
      if (!b.resident) _reload(b, _st);
      else if (b.loaded && b.loaded_st != _st) wait_on(_st, b.loaded);
      _pin(kv.first, b);
      held.push_back(kv.first);
    }
  } catch (...) {
    for (tid_t t : held) _unpin(t, _blocks.at(t));
    throw;
  }
  cuda_ok(cudaStreamSynchronize(_st), "hold_all sync");
  return held;
}

void block_storage_t::release(const std::vector<tid_t>& tids) {
  std::lock_guard<std::recursive_mutex> lk(_m);
  for (tid_t t : tids) {
    auto it = _blocks.find(t);
    if (it == _blocks.end()) continue;
    it->second.caller_may_write = true;  // the DAG's launches ran on streams the storage does not know
    _unpin(t, it->second);
  }
}

spill_stats_t block_storage_t::stats() const { return _stats; }

// ------------------------------------------------------------------ runtime
runtime_t::runtime_t() {
  tf = std::make_shared<tensor_factory_t>();
  register_b200_formats(*tf);
  udm = std::make_shared<udf_manager_t>(tf);
  register_b200_udfs(*udm);
  cuda_ok(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
  storage = std::make_unique<block_storage_t>(tf, stream);
}

runtime_t::~runtime_t() {
  for (cudaStream_t s : worker_streams) cudaStreamSynchronize(s);
  if (stream) cudaStreamSynchronize(stream);
  storage.reset();
  for (cudaStream_t s : worker_streams) cudaStreamDestroy(s);
  if (stream) cudaStreamDestroy(stream);
}

// The ud kinds the executor understands natively.
node_kind_t classify(const ud_impl_t* impl, bool is_reduce) {
  const std::string& n = impl->impl_name;
  if (starts_with(n, "b200_dense_mult_bf16") || starts_with(n, "b200_dense_mult_e4m3")) return NK_TC;
  if (n == "b200_dense_mult_f32") return NK_SIMT;
  if (n == "b200_dense_add" || n == "b200_dense_bf16_add") return NK_SUM;
  if (is_reduce) return NK_OPAQUE;
  if (starts_with(n, "b200_dense_relu") || starts_with(n, "b200_dense_sigmoid")) return NK_UNARY;
  if (starts_with(n, "b200_dense_hadamard") || starts_with(n, "b200_dense_weighted")) return NK_BINARY;
  if (starts_with(n, "b200_contraction")) return NK_CONTRACT;
  return NK_OPAQUE;
}

int elem_of(const tensor_factory_t& tf, tfid_t id) {
  const std::string& n = tf.fmt_name(id);
  if (n == "dense_bf16") return ELEM_BF16;
  if (n == "dense_e4m3") return ELEM_E4M3;
  return ELEM_F32;
}

op_features_t runtime_t::features(const command_t& cmd, size_t* hint_out) {
  std::vector<tensor_meta_t> metas(cmd.get_num_inputs());
  for (size_t i = 0; i < cmd.get_num_inputs(); ++i) {
    tensor_t* t = storage->get(cmd.get_input(i).tid);
    if (t) metas[i] = t->_meta;
  }
  return features_of(*tf, cmd, udm->get_fn_impl(cmd.fun_id), metas, hint_out);
}

// 12 features: op-kind one-hot (matmul, add, reduce, contraction), log2 m, n, k,
// dtype (0 f32 / 1 bf16 / 2 e4m3), transpose flags, input count, log2 of the
// elements touched.
op_features_t features_of(const tensor_factory_t& tfac, const command_t& cmd, ud_impl_t* impl,
                          std::vector<tensor_meta_t> metas, size_t* hint_out) {
  const tensor_factory_t* tf = &tfac;
  op_features_t f{};
  ud_impl_t::meta_args_t margs(metas);
  ud_impl_t::tensor_params_t params;
  params._params = cmd.get_parameters();
  node_kind_t k = impl ? classify(impl, cmd.is_reduce()) : NK_OPAQUE;
  double m = 1, n = 1, kk = 1;
  int ta = 0, tb = 0, dtype = 0;
  if (impl && (k == NK_TC || k == NK_SIMT)) {
    const auto& ma = metas[0].as<dense_tensor_meta_t>().m();
    const auto& mb = metas[1].as<dense_tensor_meta_t>().m();
    ta = params.get_bool_or_default<0>(false);
    tb = params.get_bool_or_default<1>(false);
    m = ta ? ma.num_cols : ma.num_rows;
    kk = ta ? ma.num_rows : ma.num_cols;
    n = tb ? mb.num_rows : mb.num_cols;
    dtype = elem_of(*tf, metas[0].fmt_id);
  } else if (impl && k == NK_CONTRACT) {
    // lowered GEMM sizes: product of lhs-only+batch..., approximated by cube root split of the hint
    size_t h = impl->get_complexity_hint(params, margs);
    double c = std::cbrt((double)h);
    m = n = kk = c;
    dtype = impl->impl_name == "b200_contraction_bf16" ? 1 : 0;
  } else if (!metas.empty()) {
    const auto& ma = metas[0].as<dense_tensor_meta_t>().m();
    m = ma.num_rows;
    n = ma.num_cols;
    dtype = elem_of(*tf, metas[0].fmt_id);
  }
  int kind_slot = (k == NK_TC || k == NK_SIMT) ? 0 : (k == NK_SUM && !cmd.is_reduce()) ? 1 : cmd.is_reduce() ? 2 : k == NK_CONTRACT ? 3 : 1;
  f.f[kind_slot] = 1.f;
  f.f[4] = (float)std::log2(std::max(1.0, m));
  f.f[5] = (float)std::log2(std::max(1.0, n));
  f.f[6] = (float)std::log2(std::max(1.0, kk));
  f.f[7] = (float)dtype;
  f.f[8] = (float)ta;
  f.f[9] = (float)tb;
  f.f[10] = (float)cmd.get_num_inputs();
  f.f[11] = (float)std::log2(std::max(1.0, m * n * (double)std::max<size_t>(1, cmd.get_num_inputs())));
  const size_t hint = impl ? impl->get_complexity_hint(params, margs) : 0;
  f.hint = (double)hint;
  if (hint_out) *hint_out = hint;
  return f;
}

// Executes one APPLY / REDUCE on the runtime stream (the per-op path).
void execute_command(runtime_t& rt, command_t& cmd, cudaStream_t st) {
  ud_impl_t* impl = rt.udm->get_fn_impl(cmd.fun_id);
  if (!impl) throw std::runtime_error("command " + std::to_string(cmd.id) + ": unknown ud impl");
  ud_impl_t::tensor_params_t params;
  params._params = cmd.get_parameters();
  params.stream = st;
  if (cmd.is_apply()) {
    const size_t ni = cmd.get_num_inputs(), no = cmd.get_num_outputs();
    std::vector<tensor_meta_t> in_meta(ni), out_meta(no);
    ud_impl_t::tensor_args_t in_args(ni);
    for (size_t i = 0; i < ni; ++i) {
      tensor_t* t = rt.storage->acquire(cmd.get_input(i).tid, st);
      if (!t) throw std::runtime_error("APPLY " + std::to_string(cmd.id) + ": input tensor missing");
      in_meta[i] = t->_meta;
      in_args.set(i, *t);
    }
    ud_impl_t::meta_args_t im(in_meta), om(out_meta);
    for (size_t i = 0; i < no; ++i) std::memset(&out_meta[i], 0, sizeof(tensor_meta_t));
    impl->get_out_meta(params, im, om);
    ud_impl_t::tensor_args_t out_args(no);
    for (size_t i = 0; i < no; ++i) {
      out_meta[i].fmt_id = rt.tf->get_tensor_ftm(impl->outputTypes[i]);
      tensor_t* t = rt.storage->create(cmd.get_output(i).tid, out_meta[i], st);
      out_args.set(i, *t);
    }
    impl->call_ud(params, in_args, out_args);
  } else if (cmd.is_reduce()) {
    // n-ary reduce: a native matrix_add reduce reads every input once in one
    // launch; any other associative ud is folded pairwise left to right with
    // a temporary per step, as local_reduce_op_t::apply does.
    const size_t ni = cmd.get_num_inputs();
    std::vector<tensor_t*> ins(ni);
    for (size_t i = 0; i < ni; ++i) {
      ins[i] = rt.storage->acquire(cmd.get_input(i).tid, st);
      if (!ins[i]) throw std::runtime_error("REDUCE " + std::to_string(cmd.id) + ": input tensor missing");
    }
    tid_t out_tid = cmd.get_output(0).tid;
    const tensor_meta_t& m0 = ins[0]->_meta;
    if (impl->impl_name == "b200_dense_add" || impl->impl_name == "b200_dense_bf16_add") {
      tensor_t* out = rt.storage->create(out_tid, m0, st);
      const auto& dm = m0.as<dense_tensor_meta_t>().m();
      const long long n = (long long)dm.num_rows * dm.num_cols;
      const int dt = impl->impl_name == "b200_dense_add" ? BBX_F32 : BBX_BF16;
      if (dt == BBX_F32) {
        std::vector<const float*> ptrs(ni);
        for (size_t i = 0; i < ni; ++i) ptrs[i] = (const float*)ins[i]->_meta.payload();
        bbx_ok(bbx_reduce_f32(ptrs.data(), (int)ni, (float*)out->_meta.payload(), n, 1, st));
      } else {
        // bf16 blocks: chain grouped-stream sums of up to 16 inputs (f32 math)
        std::vector<const void*> pend;
        for (size_t i = 0; i < ni; ++i) pend.push_back(ins[i]->_meta.payload());
        while (!pend.empty()) {
          bbx_stream_op_t s{};
          s.kind = BBX_S_SUM; s.in_dtype = BBX_BF16; s.out_dtype = BBX_BF16; s.kahan = 1; s.n = n;
          int c = 0;
          if (pend.size() != ni) s.in[c++] = out->_meta.payload();
          while (c < BBX_STREAM_MAX_IN && !pend.empty()) { s.in[c++] = pend.front(); pend.erase(pend.begin()); }
          s.n_in = c;
          s.out = out->_meta.payload();
          bbx_ok(bbx_stream_group(&s, 1, st));
        }
      }
    } else {
      tid_t tmp_base = -1000000000;
      tensor_t* lhs = ins[0];
      tid_t lhs_tid = cmd.get_input(0).tid;
      for (size_t i = 1; i < ni; ++i) {
        std::vector<tensor_meta_t> im{lhs->_meta, ins[i]->_meta}, om(1);
        std::memset(&om[0], 0, sizeof(tensor_meta_t));
        ud_impl_t::meta_args_t ima(im), oma(om);
        impl->get_out_meta(params, ima, oma);
        om[0].fmt_id = rt.tf->get_tensor_ftm(impl->outputTypes[0]);
        tid_t t = (i + 1 == ni) ? out_tid : tmp_base - (tid_t)i;
        tensor_t* o = rt.storage->create(t, om[0], st);
        ud_impl_t::tensor_args_t ia(std::vector<tensor_t*>{lhs, ins[i]}), oa(std::vector<tensor_t*>{o});
        impl->call_ud(params, ia, oa);
        if (i > 1) rt.storage->remove(lhs_tid, st);  // drop the previous intermediate
        lhs = o;
        lhs_tid = t;
      }
      if (ni == 1) {
        tensor_t* o = rt.storage->create(out_tid, m0, st);
        cuda_ok(cudaMemcpyAsync(o->_meta.payload(), m0.payload(), rt.tf->get_payload_size(m0),
                                cudaMemcpyDeviceToDevice, st), "reduce copy");
      }
    }
  }
}

void runtime_t::run_per_op(int policy, std::vector<std::pair<op_features_t, float>>* record) {
  reservation_station_t rs(0, 1);
  for (tid_t t : storage->tids()) rs.register_tensor(t);
  std::unordered_map<command_id_t, double> prio, lat_of;
  if (policy == SCHED_LEARNED && predictor) {
    // critical-path priority: predicted latency + the longest predicted path to a sink
    std::unordered_map<tid_t, std::vector<size_t>> readers;
    for (size_t i = 0; i < commands.size(); ++i)
      for (size_t j = 0; j < commands[i]->get_num_inputs(); ++j) readers[commands[i]->get_input(j).tid].push_back(i);
    // metas of every tensor the list will create (get_out_meta propagated in
    // command order), so each command gets real features
    std::unordered_map<tid_t, tensor_meta_t> metas;
    for (tid_t t : storage->tids()) metas[t] = storage->get(t)->_meta;
    std::vector<op_features_t> fs(commands.size());
    std::vector<bool> has(commands.size(), false);
    for (size_t i = 0; i < commands.size(); ++i) {
      auto& c = *commands[i];
      if (c.is_delete()) continue;
      ud_impl_t* impl = udm->get_fn_impl(c.fun_id);
      std::vector<tensor_meta_t> in;
      bool ok = impl != nullptr;
      for (size_t j = 0; j < c.get_num_inputs() && ok; ++j) {
        auto it = metas.find(c.get_input(j).tid);
        ok = it != metas.end();
        if (ok) in.push_back(it->second);
      }
      if (!ok) continue;
      ud_impl_t::tensor_params_t params;
      params._params = c.get_parameters();
      std::vector<tensor_meta_t> out(c.get_num_outputs());
      for (auto& m : out) std::memset(&m, 0, sizeof(m));
      if (c.is_apply()) {
        ud_impl_t::meta_args_t im(in), om(out);
        impl->get_out_meta(params, im, om);
        for (size_t o = 0; o < out.size(); ++o) out[o].fmt_id = tf->get_tensor_ftm(impl->outputTypes[o]);
      } else {
        out[0] = in[0];
      }
      for (size_t o = 0; o < out.size(); ++o) metas[c.get_output(o).tid] = out[o];
      fs[i] = features_of(*tf, c, impl, in, nullptr);
      has[i] = true;
    }
    std::vector<op_features_t> batch;
    for (size_t i = 0; i < commands.size(); ++i) if (has[i]) batch.push_back(fs[i]);
    std::vector<double> lat_b = batch_predictor ? batch_predictor(batch) : std::vector<double>();
    std::vector<double> lat(commands.size(), 1.0);
    for (size_t i = 0, k = 0; i < commands.size(); ++i)
      if (has[i]) lat[i] = k < lat_b.size() ? lat_b[k++] : predictor(fs[i]);
    std::vector<double> up(commands.size(), 0.0);
    for (size_t ii = commands.size(); ii-- > 0;) {
      auto& c = *commands[ii];
      if (c.is_delete()) continue;
      double best = 0;
      for (size_t o = 0; o < c.get_num_outputs(); ++o)
        for (size_t r : readers[c.get_output(o).tid]) best = std::max(best, up[r]);
      up[ii] = lat[ii] + best;
      prio[c.id] = up[ii];
      lat_of[c.id] = lat[ii];
    }
    rs.set_priority([&prio](const command_t& c) { auto it = prio.find(c.id); return it == prio.end() ? 0.0 : it->second; });
  }
  for (auto& c : commands) {
    if (!rs.queue_command(c->clone())) throw std::runtime_error("reservation station rejected command " + std::to_string(c->id));
  }
  rs.execute_scheduled_async();

  // ---- worker streams (one = the runtime stream itself)
  const int K = record ? 1 : std::max(1, std::min(workers, 16));
  while ((int)worker_streams.size() < K && K > 1) {
    cudaStream_t s;
    cuda_ok(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate(worker)");
    worker_streams.push_back(s);
  }
  std::vector<cudaStream_t> ws;
  if (K == 1) ws.push_back(stream);
  else ws.assign(worker_streams.begin(), worker_streams.begin() + K);
  std::vector<cudaEvent_t> events;
  auto new_event = [&]() {
    cudaEvent_t e;
    cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    events.push_back(e);
    return e;
  };
  std::unordered_map<tid_t, cudaEvent_t> ready;                              // producer's completion
  std::unordered_map<tid_t, std::vector<std::pair<cudaEvent_t, int>>> reads;  // readers' completions + stream
  if (K > 1) {
    cudaEvent_t start = new_event();  // everything queued on the runtime stream so far comes first
    cuda_ok(cudaEventRecord(start, stream), "record start");
    for (cudaStream_t s : ws) cuda_ok(cudaStreamWaitEvent(s, start, 0), "wait start");
  }
  // a deleted block is freed on the stream of its last reader, after the other
  // readers' completions, so its memory returns to the pool only when unused
  auto free_block = [&](tid_t t) {
    if (K == 1) {
      storage->remove(t);
      return;
    }
    cudaStream_t s = stream;
    auto it = reads.find(t);
    if (it != reads.end() && !it->second.empty()) {
      const int si = it->second.back().second;
      s = ws[si];
      for (auto& er : it->second)
        if (er.second != si) cuda_ok(cudaStreamWaitEvent(s, er.first, 0), "wait reader");
    } else {
      auto r = ready.find(t);
      if (r != ready.end()) cuda_ok(cudaStreamWaitEvent(s, r->second, 0), "wait producer");
    }
    storage->remove(t, s);
    reads.erase(t);
    ready.erase(t);
  };
  // eviction hint under a storage budget: queued reads left per block
  const bool hint_readers = storage->budget() > 0;
  std::unordered_map<tid_t, int> readers_left;
  if (hint_readers) {
    for (auto& c : commands)
      if (!c->is_delete())
        for (size_t j = 0; j < c->get_num_inputs(); ++j) ++readers_left[c->get_input(j).tid];
    for (tid_t t : storage->tids()) {
      auto r = readers_left.find(t);
      storage->set_readers_left(t, r == readers_left.end() ? 0 : r->second);
    }
  }
  std::vector<double> avail(K, 0.0);             // predicted time each stream frees up
  std::unordered_map<tid_t, double> t_ready;     // predicted time each block is written
  int rr = 0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> evs;
  std::vector<op_features_t> feats;
  while (true) {
    tid_t dead;
    while (rs.try_get_to_remove(&dead)) {
      free_block(dead);
      rs.retire_remove(dead);
    }
    command_ptr_t cmd = rs.try_get_next_command();
    if (!cmd) {
      if (rs.num_to_retire() == 0) break;
      throw std::runtime_error("DAG stalled: commands wait for tensors nothing produces");
    }
    int si = 0;
    if (K > 1) {
      auto lit = lat_of.find(cmd->id);
      if (policy == SCHED_LEARNED && lit != lat_of.end()) {
        // list scheduling: the stream on which the command is predicted to finish first
        double rdy = 0;
        for (size_t j = 0; j < cmd->get_num_inputs(); ++j) {
          auto r = t_ready.find(cmd->get_input(j).tid);
          if (r != t_ready.end()) rdy = std::max(rdy, r->second);
        }
        for (int k = 1; k < K; ++k)
          if (std::max(avail[k], rdy) < std::max(avail[si], rdy)) si = k;
        avail[si] = std::max(avail[si], rdy) + lit->second;
        for (size_t o = 0; o < cmd->get_num_outputs(); ++o) t_ready[cmd->get_output(o).tid] = avail[si];
      } else {
        si = rr++ % K;  // the reference's workers take commands as they come
      }
      for (size_t j = 0; j < cmd->get_num_inputs(); ++j) {
        auto r = ready.find(cmd->get_input(j).tid);
        if (r != ready.end()) cuda_ok(cudaStreamWaitEvent(ws[si], r->second, 0), "wait input");
      }
    }
    cudaStream_t s = ws[si];
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (record) {
      size_t hint;
      feats.push_back(features(*cmd, &hint));
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      cudaEventRecord(e0, s);
    }
    storage->begin_command();
    try {
      execute_command(*this, *cmd, s);
    } catch (...) {
      storage->end_command(s);
      throw;
    }
    storage->end_command(s);
    if (hint_readers) {
      for (size_t j = 0; j < cmd->get_num_inputs(); ++j) {
        const tid_t t = cmd->get_input(j).tid;
        storage->set_readers_left(t, --readers_left[t]);
      }
      for (size_t o = 0; o < cmd->get_num_outputs(); ++o) {
        const tid_t t = cmd->get_output(o).tid;
        auto r = readers_left.find(t);
        storage->set_readers_left(t, r == readers_left.end() ? 0 : r->second);
      }
    }
    if (record) {
      cudaEventRecord(e1, s);
      evs.push_back({e0, e1});
    }
    if (K > 1) {
      cudaEvent_t done = new_event();
      cuda_ok(cudaEventRecord(done, s), "record done");
      for (size_t o = 0; o < cmd->get_num_outputs(); ++o) ready[cmd->get_output(o).tid] = done;
      for (size_t j = 0; j < cmd->get_num_inputs(); ++j) reads[cmd->get_input(j).tid].push_back({done, si});
    }
    rs.retire_command(std::move(cmd));
  }
  tid_t dead;
  while (rs.try_get_to_remove(&dead)) {
    free_block(dead);
    rs.retire_remove(dead);
  }
  if (K > 1) {
    // join: the runtime stream continues after every worker's last command
    for (cudaStream_t s : ws) {
      cudaEvent_t e = new_event();
      cuda_ok(cudaEventRecord(e, s), "record join");
      cuda_ok(cudaStreamWaitEvent(stream, e, 0), "wait join");
    }
  }
  for (cudaEvent_t e : events) cudaEventDestroy(e);  // released once the device has passed them
  if (record) {
    cuda_ok(cudaStreamSynchronize(stream), "run_per_op sync");
    for (size_t i = 0; i < evs.size(); ++i) {
      float ms = 0;
      cudaEventElapsedTime(&ms, evs[i].first, evs[i].second);
      record->push_back({feats[i], ms * 1000.f});
      cudaEventDestroy(evs[i].first);
      cudaEventDestroy(evs[i].second);
    }
  }
}

}  // namespace bbts
