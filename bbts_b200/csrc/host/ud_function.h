// User-defined block functions: the registration API of BarbaTOS
// (src/ud_functions/ud_function.h:33-265, src/commands/command_utils.h:8-13),
// kept so that a plugin written against the reference registers unchanged.
//
// The classes a plugin touches keep the reference's data members, in the
// reference's order and sizes, so the plugin entry points can run against a
// reference node's objects: ud_impl_t, ud_func_t, tensor_params_t (its cuTENSOR
// 1.x handle is a 4 KiB struct held by value, ud_function.h:164) and
// udf_manager_t (whose first member is the node's GPU scheduler,
// udf_manager.h:55-66).
//
// Differences from the reference, by design:
//  * tensor_params_t keeps the `stream` / `cublas_handle` / `cutensor_handle`
//    fields, but this library never reads the handles: no cuBLAS or cuTENSOR
//    is used.
//  * a GPU impl's `fn` is called directly and is stream-ordered on
//    params.stream (it returns after enqueueing), instead of being funnelled
//    through the reference's blocking 3-stream GPU scheduler
//    (src/ud_functions/gpu_scheduler_impl.cc:34-112).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>
#include "tensor.h"

namespace bbts {

union command_param_t {
  float f;
  int32_t i;
  uint32_t u;
  bool b;
};

// Non-owning view of a contiguous array (src/utils/raw_vector.h).
template <class T>
struct raw_vector_t {
  T* _data = nullptr;
  size_t _num_elements = 0;
  T& operator[](size_t i) const { return _data[i]; }
  size_t size() const { return _num_elements; }
  T* begin() const { return _data; }
  T* end() const { return _data + _num_elements; }
};
using command_param_list_t = raw_vector_t<command_param_t>;

using ud_id_t = int32_t;
using ud_impl_local_t = int32_t;
struct ud_impl_id_t {
  ud_id_t ud_id;
  ud_impl_local_t impl_id;
};

// Stand-in with the size and alignment of cuTENSOR 1.x's cutensorHandle_t,
// an opaque struct of 512 int64 words passed by address to the library.
struct cutensor_handle_t {
  int64_t fields[512];
};

struct ud_impl_t {
  template <class T>
  struct ud_impl_args_t {
    ud_impl_args_t() = default;
    ud_impl_args_t(std::vector<T*> in) : arguments(std::move(in)) {}
    ud_impl_args_t(std::vector<T>& in) { reinit(in); }
    explicit ud_impl_args_t(size_t n) : arguments(n) {}
    size_t num_args() const { return arguments.size(); }
    template <size_t n> T& get() { return *arguments[n]; }
    template <size_t n> const T& get() const { return *arguments[n]; }
    const T& get_by_idx(size_t i) const { return *arguments[i]; }
    T& get_by_idx(size_t i) { return *arguments[i]; }
    template <size_t n> void set(T& v) { arguments[n] = &v; }
    void set(size_t n, T& v) { arguments[n] = &v; }
    void reinit(std::vector<T>& in) {
      arguments.resize(in.size());
      for (size_t i = 0; i < in.size(); ++i) arguments[i] = &in[i];
    }

   private:
    std::vector<T*> arguments;
  };
  using tensor_args_t = ud_impl_args_t<tensor_t>;
  using meta_args_t = ud_impl_args_t<tensor_meta_t>;

  struct tensor_params_t {
    template <size_t n> float get_float() const { return _params[n].f; }
    template <size_t n> int32_t get_int() const { return _params[n].i; }
    template <size_t n> uint32_t get_uint() const { return _params[n].u; }
    template <size_t n> uint32_t get_bool() const { return _params[n].b; }
    template <size_t n> float get_float_or_default(float v) const { return n < _params.size() ? _params[n].f : v; }
    template <size_t n> int32_t get_int_or_default(int32_t v) const { return n < _params.size() ? _params[n].i : v; }
    template <size_t n> uint32_t get_uint_or_default(uint32_t v) const { return n < _params.size() ? _params[n].u : v; }
    template <size_t n> uint32_t get_bool_or_default(bool v) const { return n < _params.size() ? _params[n].b : v; }
    command_param_t get_raw(size_t n) const { return _params[n]; }
    size_t num_parameters() const { return _params.size(); }

    command_param_list_t _params;
    cudaStream_t stream = nullptr;
    void* cublas_handle = nullptr;       // never read by this library
    cutensor_handle_t cutensor_handle{};  // never read by this library
  };

  using ud_impl_callable =
      std::function<void(const tensor_params_t& params, const tensor_args_t& in, tensor_args_t& out)>;

  ud_impl_id_t impl_id{-1, -1};
  std::string impl_name;
  std::string ud_name;
  std::vector<std::string> inputTypes;
  std::vector<int32_t> inputInplace;
  std::vector<std::string> outputTypes;
  bool is_gpu = false;

  virtual ~ud_impl_t() = default;

  void call_ud(const tensor_params_t& p, const tensor_args_t& in, tensor_args_t& out) const { fn(p, in, out); }
  void call_gpu_ud(const tensor_params_t& p, const tensor_args_t& in, tensor_args_t& out) const {
    (gpu_fn ? gpu_fn : fn)(p, in, out);
  }

  ud_impl_callable fn;
  ud_impl_callable gpu_fn;

  virtual size_t get_complexity_hint(const tensor_params_t& params, const meta_args_t& in) = 0;
  virtual void get_out_meta(const tensor_params_t& params, const meta_args_t& in, meta_args_t& out) const = 0;
};
using ud_impl_ptr_t = std::unique_ptr<ud_impl_t>;

struct ud_func_t {
  ud_id_t id = -1;
  std::string ud_name;
  bool is_ass = false;
  bool is_com = false;
  size_t num_in = 0;
  size_t num_out = 0;
  std::vector<ud_impl_ptr_t> impls;

  ud_impl_id_t add_impl(ud_impl_ptr_t impl) {
    auto local = (ud_impl_local_t)impls.size();
    impl->impl_id = ud_impl_id_t{id, local};
    impls.emplace_back(std::move(impl));
    return impls.back()->impl_id;
  }
};
using ud_func_ptr_t = std::unique_ptr<ud_func_t>;

// Finds an implementation whose input and output formats all match
// (src/ud_functions/udf_manager.cc:10-37 intends this; its `continue`s make
// the type checks no-ops, so here the types are actually compared).
class udf_matcher {
 public:
  explicit udf_matcher(std::vector<ud_impl_ptr_t>& impls) : _impls(impls) {}
  ud_impl_t* findMatch(const std::vector<std::string>& inputs, const std::vector<std::string>& outputs,
                       bool require_gpu = false);

 private:
  std::vector<ud_impl_ptr_t>& _impls;
};
using udf_matcher_ptr = std::unique_ptr<udf_matcher>;

class udf_manager_t {
 public:
  explicit udf_manager_t(tensor_factory_ptr_t factory);
  ud_id_t register_udf(ud_func_ptr_t fun);
  ud_impl_id_t register_udf_impl(ud_impl_ptr_t impl);
  udf_matcher_ptr get_matcher_for(const std::string& ud_name);
  udf_matcher_ptr get_matcher_for(const std::string& ud_name, bool is_commutative, bool is_associative);
  ud_impl_t* get_fn_impl(ud_impl_id_t id);
  ud_func_t* get_udf(const std::string& ud_name);
  ud_func_t* get_udf(ud_id_t id);
  const tensor_factory_ptr_t& factory() const { return _tensor_factory; }

 private:
  // the reference node's GPU scheduler (gpu_scheduler_ptr_t); this library
  // schedules on streams and leaves it empty
  std::shared_ptr<void> _gpu_scheduler;
  tensor_factory_ptr_t _tensor_factory;
  std::vector<ud_func_ptr_t> _udfs;
  std::unordered_map<std::string, ud_id_t> _udfs_name_to_id;
};
using udf_manager_ptr = std::shared_ptr<udf_manager_t>;

// Registers the B200 formats and ud implementations of this library; the same
// code runs behind the plugin entry points register_tensors / register_udfs.
void register_b200_formats(tensor_factory_t& tf);
void register_b200_udfs(udf_manager_t& udm);

}  // namespace bbts

// Plugin entry points with the reference's names and argument types
// (libraries/cutensor.cc:16-31, found with dlsym at src/server/coordinator.cc:509-532).
extern "C" {
void register_tensors(bbts::tensor_factory_ptr_t tensor_factory);
void register_udfs(bbts::udf_manager_ptr udf_manager);
}
