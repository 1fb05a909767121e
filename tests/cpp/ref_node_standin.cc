// A stand-in for the reference node's side of the plugin boundary.
//
// The reference's coordinator dlopen()s a plugin and calls its two unmangled
// entry points with its own objects (src/server/coordinator.cc:509-532):
//   register_tensors(tensor_factory_ptr_t)   register_udfs(udf_manager_ptr)
// A plugin compiled against the reference's headers calls back into the
// node's exported member functions (register_fmt, register_udf,
// register_udf_impl) and hands the node ud_impl_t objects that the node then
// calls through fn / get_out_meta / get_complexity_hint.
//
// This program plays the node: the classes below restate the reference's
// data members in the reference's order and types (tensor.h:20-52,
// tensor_factory.h:12-41, ud_function.h:33-265, udf_manager.h:31-66,
// command_utils.h:8-13, raw_vector.h), written here independently of this
// library's headers; the static_asserts pin the offsets those declarations
// imply. The member functions are defined here and exported (-rdynamic), so
// the plugin's calls bind to them, as they bind to a real node's.
// register_udf_impl wraps GPU impls the way the reference's does
// (udf_manager.cc:98-111): fn moves to gpu_fn and fn goes through the node's
// GPU scheduler.
//
// Usage: ref_node_standin <path to libbbts_b200.so> [gpu]
// Without "gpu" it checks the registrations and the metadata callbacks only;
// with "gpu" it also runs impls on reference-layout dense tensors in managed
// memory (payload right after the 260-byte header, as the node allocates them).
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace bbts {

using tid_t = int32_t;
using tfid_t = int32_t;

struct tensor_meta_t {
  tfid_t fmt_id;
  char _blob[256];
};

struct tensor_t {
  tensor_meta_t _meta;
  char _blob[0];
};

struct tensor_creation_fs_t {
  std::function<size_t(const tensor_meta_t&)> get_size;
  std::function<tensor_t&(void* here, const tensor_meta_t&)> init_tensor;
  std::function<void(const void* here, std::stringstream& ss)> print;
};

class tensor_factory_t {
 public:
  tensor_factory_t();
  tfid_t register_fmt(const std::string& _fmt_name, const tensor_creation_fs_t& _fmt_funs);
  tfid_t get_tensor_ftm(const std::string& _fmt_name);
  size_t get_tensor_size(const tensor_meta_t& _meta);
  tensor_t& init_tensor(tensor_t* here, const tensor_meta_t& _meta);
  // inspection by this test (private in the reference; same order)
  std::unordered_map<std::string, tfid_t> _reg_fmts;
  std::vector<tensor_creation_fs_t> _fmt_fs;
};
using tensor_factory_ptr_t = std::shared_ptr<tensor_factory_t>;

union command_param_t {
  float f;
  int32_t i;
  uint32_t u;
  bool b;
};

template <class T>
struct raw_vector_t {
  T* _data;
  size_t _num_elements;
};
using command_param_list_t = raw_vector_t<command_param_t>;

using ud_id_t = int32_t;
using ud_impl_local_t = int32_t;
struct ud_impl_id_t {
  ud_id_t ud_id;
  ud_impl_local_t impl_id;
};

// cuTENSOR 1.x's handle is an opaque struct of 512 int64 words held by value.
struct cutensor_handle_standin_t {
  int64_t fields[512];
};

struct ud_impl_t {
  template <class T>
  struct ud_impl_args_t {
    ud_impl_args_t() = default;
    ud_impl_args_t(std::vector<T*> in_arg) : arguments(std::move(in_arg)) {}
    std::vector<T*> arguments;
  };
  using tensor_args_t = ud_impl_args_t<tensor_t>;
  using meta_args_t = ud_impl_args_t<tensor_meta_t>;

  struct tensor_params_t {
    command_param_list_t _params;
    cudaStream_t stream;
    void* cublas_handle;
    cutensor_handle_standin_t cutensor_handle;
  };

  using ud_impl_callable =
      std::function<void(const tensor_params_t& params, const tensor_args_t& _in, tensor_args_t& _out)>;

  ud_impl_id_t impl_id;
  std::string impl_name;
  std::string ud_name;
  std::vector<std::string> inputTypes;
  std::vector<int32_t> inputInplace;
  std::vector<std::string> outputTypes;
  bool is_gpu;

  virtual ~ud_impl_t() = default;

  ud_impl_callable fn;
  ud_impl_callable gpu_fn;

  virtual size_t get_complexity_hint(const tensor_params_t& params, const meta_args_t& _in) = 0;
  virtual void get_out_meta(const tensor_params_t& params, const meta_args_t& _in, meta_args_t& _out) const = 0;
};
using ud_impl_ptr_t = std::unique_ptr<ud_impl_t>;

struct ud_func_t {
  ud_id_t id;
  std::string ud_name;
  bool is_ass;
  bool is_com;
  size_t num_in;
  size_t num_out;
  std::vector<ud_impl_ptr_t> impls;
};
using ud_func_ptr_t = std::unique_ptr<ud_func_t>;

// The node's GPU scheduler, reduced to what the wrapper needs: run the impl's
// gpu_fn on the scheduler's stream and wait (gpu_scheduler_impl.cc:34-112
// prefetches managed memory around the same call).
struct gpu_scheduler_t {
  cudaStream_t stream = nullptr;
  int calls = 0;
  void execute(ud_impl_t* me, const ud_impl_t::tensor_params_t* params, const ud_impl_t::tensor_args_t* in,
               ud_impl_t::tensor_args_t* out) {
    ++calls;
    ud_impl_t::tensor_params_t p = *params;
    p.stream = stream;
    me->gpu_fn(p, *in, *out);
    if (cudaStreamSynchronize(stream) != cudaSuccess) throw std::runtime_error("scheduler sync failed");
  }
};
using gpu_scheduler_ptr_t = std::shared_ptr<gpu_scheduler_t>;

class udf_manager_t {
 public:
  udf_manager_t(tensor_factory_ptr_t _tensor_factory, gpu_scheduler_ptr_t _gpu_scheduler);
  ud_id_t register_udf(ud_func_ptr_t _fun);
  ud_impl_id_t register_udf_impl(ud_impl_ptr_t _impl);
  // inspection by this test (private in the reference; same order)
  gpu_scheduler_ptr_t _gpu_scheduler;
  tensor_factory_ptr_t _tensor_factory;
  std::vector<ud_func_ptr_t> _udfs;
  std::unordered_map<std::string, ud_id_t> _udfs_name_to_id;
};
using udf_manager_ptr = std::shared_ptr<udf_manager_t>;

static_assert(sizeof(tensor_meta_t) == 260, "tensor_meta_t");
static_assert(offsetof(ud_impl_t::tensor_params_t, stream) == 16, "params.stream");
static_assert(offsetof(ud_impl_t::tensor_params_t, cutensor_handle) == 32, "params.cutensor_handle");
static_assert(sizeof(ud_impl_t::tensor_params_t) == 32 + 4096, "params size");
static_assert(offsetof(udf_manager_t, _tensor_factory) == 16, "manager: the scheduler comes first");

// ---------------------------------------------------------------- node-side definitions
tensor_factory_t::tensor_factory_t() {
  // the node's own "dense" format: payload right after the header
  tensor_creation_fs_t fs;
  fs.get_size = [](const tensor_meta_t& m) {
    const uint32_t* rc = (const uint32_t*)m._blob;
    return sizeof(tensor_meta_t) + (size_t)rc[0] * rc[1] * sizeof(float);
  };
  fs.init_tensor = [](void* here, const tensor_meta_t& m) -> tensor_t& {
    auto& t = *(tensor_t*)here;
    t._meta = m;
    return t;
  };
  fs.print = [](const void*, std::stringstream&) {};
  register_fmt("dense", fs);
}

tfid_t tensor_factory_t::register_fmt(const std::string& name, const tensor_creation_fs_t& fs) {
  if (_reg_fmts.find(name) == _reg_fmts.end()) {
    _reg_fmts[name] = (tfid_t)_fmt_fs.size();
    _fmt_fs.emplace_back(fs);
  }
  return -1;
}

tfid_t tensor_factory_t::get_tensor_ftm(const std::string& name) {
  auto it = _reg_fmts.find(name);
  return it == _reg_fmts.end() ? -1 : it->second;
}

size_t tensor_factory_t::get_tensor_size(const tensor_meta_t& m) { return _fmt_fs.at(m.fmt_id).get_size(m); }

tensor_t& tensor_factory_t::init_tensor(tensor_t* here, const tensor_meta_t& m) {
  tensor_t& out = _fmt_fs.at(m.fmt_id).init_tensor(here, m);
  out._meta.fmt_id = m.fmt_id;
  return out;
}

udf_manager_t::udf_manager_t(tensor_factory_ptr_t tf, gpu_scheduler_ptr_t gs)
    : _gpu_scheduler(std::move(gs)), _tensor_factory(std::move(tf)) {
  // the node's builtin uds come first (udf_manager.cc:42-76)
  for (const char* name : {"matrix_add", "matrix_mult", "uniform"}) {
    auto f = std::make_unique<ud_func_t>();
    f->ud_name = name;
    f->is_ass = true;
    f->is_com = std::string(name) == "matrix_add";
    f->num_in = std::string(name) == "uniform" ? 0 : 2;
    f->num_out = 1;
    register_udf(std::move(f));
  }
}

ud_id_t udf_manager_t::register_udf(ud_func_ptr_t fun) {
  if (_udfs_name_to_id.count(fun->ud_name)) return -1;
  ud_id_t id = (ud_id_t)_udfs.size();
  fun->id = id;
  _udfs_name_to_id[fun->ud_name] = id;
  _udfs.emplace_back(std::move(fun));
  return id;
}

static int g_node_impl_registrations = 0;  // calls that reached the node's own definition

ud_impl_id_t udf_manager_t::register_udf_impl(ud_impl_ptr_t impl) {
  ++g_node_impl_registrations;
  if (impl->is_gpu) {
    impl->gpu_fn = impl->fn;
    impl->fn = [this, me = impl.get()](const ud_impl_t::tensor_params_t& p, const ud_impl_t::tensor_args_t& in,
                                       ud_impl_t::tensor_args_t& out) { _gpu_scheduler->execute(me, &p, &in, &out); };
  }
  auto it = _udfs_name_to_id.find(impl->ud_name);
  if (it == _udfs_name_to_id.end()) return {-1, -1};
  auto& f = _udfs[it->second];
  ud_impl_local_t local = (ud_impl_local_t)f->impls.size();
  impl->impl_id = {f->id, local};
  f->impls.emplace_back(std::move(impl));
  return f->impls.back()->impl_id;
}

}  // namespace bbts

using namespace bbts;

static int g_fail = 0;
#define EXPECT(c)                                                  \
  do {                                                             \
    if (!(c)) {                                                    \
      std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c);     \
      ++g_fail;                                                    \
    }                                                              \
  } while (0)

static ud_impl_t* find_impl(udf_manager_t& m, const char* ud, const char* impl) {
  auto it = m._udfs_name_to_id.find(ud);
  if (it == m._udfs_name_to_id.end()) return nullptr;
  for (auto& p : m._udfs[it->second]->impls)
    if (p->impl_name == impl) return p.get();
  return nullptr;
}

static tensor_meta_t dense_meta(tfid_t id, uint32_t rows, uint32_t cols) {
  tensor_meta_t m;
  std::memset(&m, 0, sizeof(m));  // the node value-initialises metas (a zeroed blob)
  m.fmt_id = id;
  ((uint32_t*)m._blob)[0] = rows;
  ((uint32_t*)m._blob)[1] = cols;
  return m;
}

// A node-allocated dense tensor: header + payload in one managed allocation,
// initialised by the node's own "dense" format.
static tensor_t* node_tensor(tensor_factory_t& tf, uint32_t rows, uint32_t cols) {
  tensor_meta_t m = dense_meta(tf.get_tensor_ftm("dense"), rows, cols);
  void* mem = nullptr;
  if (cudaMallocManaged(&mem, tf.get_tensor_size(m)) != cudaSuccess) throw std::runtime_error("managed alloc");
  return &tf.init_tensor((tensor_t*)mem, m);
}

static float* node_data(tensor_t* t) { return (float*)((char*)t + sizeof(tensor_meta_t)); }

int main(int argc, char** argv) {
  if (argc < 2) {
    std::printf("usage: %s <libbbts_b200.so> [gpu]\n", argv[0]);
    return 2;
  }
  const bool gpu = argc > 2 && std::string(argv[2]) == "gpu";
  auto tf = std::make_shared<tensor_factory_t>();
  auto sched = std::make_shared<gpu_scheduler_t>();
  auto udm = std::make_shared<udf_manager_t>(tf, sched);
  const size_t builtin_uds = udm->_udfs.size();

  void* so = dlopen(argv[1], RTLD_LOCAL | RTLD_NOW);
  if (!so) {
    std::printf("FAIL dlopen: %s\n", dlerror());
    return 1;
  }
  using reg_tensors_f = void(tensor_factory_ptr_t);
  using reg_udfs_f = void(udf_manager_ptr);
  auto* reg_tensors = (reg_tensors_f*)dlsym(so, "register_tensors");
  auto* reg_udfs = (reg_udfs_f*)dlsym(so, "register_udfs");
  EXPECT(reg_tensors != nullptr);
  EXPECT(reg_udfs != nullptr);
  if (!reg_tensors || !reg_udfs) return 1;

  // ---- formats: the node keeps its own "dense" (id 0); the library adds its formats after it
  reg_tensors(tf);
  EXPECT(tf->get_tensor_ftm("dense") == 0);
  for (const char* f : {"dense_bf16", "dense_e4m3", "ffnn_dense", "cutensor", "labels"}) EXPECT(tf->get_tensor_ftm(f) > 0);
  EXPECT(tf->_fmt_fs.size() == 6);
  std::printf("formats registered: %zu\n", tf->_fmt_fs.size());

  // ---- uds and impls: registered through the node's own member functions
  reg_udfs(udm);
  EXPECT(udm->_udfs.size() > builtin_uds);
  EXPECT(udm->_gpu_scheduler == sched && udm->_tensor_factory == tf);  // the node's members are untouched
  size_t n_impls = 0;
  for (auto& f : udm->_udfs)
    for (auto& p : f->impls) {
      ++n_impls;
      EXPECT(p->is_gpu);
      EXPECT(p->impl_name.rfind("b200_", 0) == 0);
      EXPECT((bool)p->gpu_fn && (bool)p->fn);  // wrapped for the node's scheduler
      EXPECT(p->impl_id.ud_id == f->id);
    }
  EXPECT(n_impls >= 20);
  EXPECT(g_node_impl_registrations == (int)n_impls);  // the plugin called the node's register_udf_impl
  std::printf("uds %zu, impls %zu\n", udm->_udfs.size(), n_impls);

  ud_impl_t* mult = find_impl(*udm, "matrix_mult", "b200_dense_mult_f32");
  ud_impl_t* add = find_impl(*udm, "matrix_add", "b200_dense_add");
  ud_impl_t* relu = find_impl(*udm, "matrix_relu", "b200_dense_relu");
  EXPECT(mult && add && relu);
  if (!mult || !add || !relu) return 1;

  // ---- metadata callbacks on node metas (virtual calls across the boundary)
  const tfid_t dense = tf->get_tensor_ftm("dense");
  ud_impl_t::tensor_params_t params;
  std::memset(&params, 0, sizeof(params));
  {
    tensor_meta_t a = dense_meta(dense, 48, 40), b = dense_meta(dense, 40, 56), c = dense_meta(dense, 0, 0);
    ud_impl_t::meta_args_t in({&a, &b}), out({&c});
    mult->get_out_meta(params, in, out);
    EXPECT(((uint32_t*)c._blob)[0] == 48 && ((uint32_t*)c._blob)[1] == 56);
    EXPECT(mult->get_complexity_hint(params, in) == (size_t)48 * 40 * 56);
  }
  std::printf("metadata callbacks ok\n");

  if (gpu) {
    // ---- impls on node-allocated tensors: payload at header + 260 (4-byte aligned)
    const uint32_t M = 48, K = 40, N = 56;
    tensor_t* a = node_tensor(*tf, M, K);
    tensor_t* b = node_tensor(*tf, K, N);
    tensor_t* c = node_tensor(*tf, M, N);
    tensor_t* s = node_tensor(*tf, M, N);
    tensor_t* r = node_tensor(*tf, M, N);
    for (uint32_t i = 0; i < M * K; ++i) node_data(a)[i] = (float)((i * 7) % 13) - 6.0f;
    for (uint32_t i = 0; i < K * N; ++i) node_data(b)[i] = (float)((i * 5) % 11) - 5.0f;
    EXPECT(((uintptr_t)node_data(a) & 15) != 0);  // the reference's unaligned payload
    // C = A B (integers: exact in FP32)
    ud_impl_t::tensor_args_t in({a, b}), out({c});
    mult->fn(params, in, out);
    int bad = 0;
    for (uint32_t i = 0; i < M && !bad; ++i)
      for (uint32_t j = 0; j < N; ++j) {
        double ref = 0;
        for (uint32_t k = 0; k < K; ++k) ref += (double)node_data(a)[i * K + k] * node_data(b)[k * N + j];
        if (node_data(c)[i * N + j] != (float)ref) { bad = 1; break; }
      }
    EXPECT(!bad);
    EXPECT(((uint32_t*)c->_meta._blob)[0] == M && ((uint32_t*)c->_meta._blob)[1] == N);
    // S = C + C, then R = relu(S - ...) via relu of S
    ud_impl_t::tensor_args_t in2({c, c}), out2({s});
    add->fn(params, in2, out2);
    ud_impl_t::tensor_args_t in3({s}), out3({r});
    relu->fn(params, in3, out3);
    bad = 0;
    for (uint32_t i = 0; i < M * N; ++i) {
      const float sum = node_data(c)[i] + node_data(c)[i];
      if (node_data(s)[i] != sum || node_data(r)[i] != (sum > 0.f ? sum : 0.f)) bad = 1;
    }
    EXPECT(!bad);
    EXPECT(sched->calls == 3);  // every call went through the node's scheduler
    std::printf("impls on node tensors ok (scheduler calls %d)\n", sched->calls);
    for (tensor_t* t : {a, b, c, s, r}) cudaFree(t);
  }

  if (g_fail) {
    std::printf("%d failures\n", g_fail);
    return 1;
  }
  std::printf("plugin boundary ok\n");
  return 0;
}
