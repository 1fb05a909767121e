// The ud registry (src/ud_functions/udf_manager.cc).
#include <stdexcept>
#include "ud_function.h"

namespace bbts {

ud_impl_t* udf_matcher::findMatch(const std::vector<std::string>& inputs,
                                  const std::vector<std::string>& outputs, bool require_gpu) {
  for (const auto& f : _impls) {
    if (f->is_gpu != require_gpu) continue;
    if (f->inputTypes.size() != inputs.size() || f->outputTypes.size() != outputs.size()) continue;
    bool ok = true;
    for (size_t i = 0; i < inputs.size() && ok; ++i) ok = inputs[i] == f->inputTypes[i];
    for (size_t i = 0; i < outputs.size() && ok; ++i) ok = outputs[i] == f->outputTypes[i];
    if (ok) return f.get();
  }
  return nullptr;
}

udf_manager_t::udf_manager_t(tensor_factory_ptr_t factory) : _tensor_factory(std::move(factory)) {}

ud_id_t udf_manager_t::register_udf(ud_func_ptr_t fun) {
  if (_udfs_name_to_id.count(fun->ud_name)) return -1;
  ud_id_t id = (ud_id_t)_udfs.size();
  fun->id = id;
  _udfs_name_to_id[fun->ud_name] = id;
  _udfs.emplace_back(std::move(fun));
  return id;
}

ud_impl_id_t udf_manager_t::register_udf_impl(ud_impl_ptr_t impl) {
  auto it = _udfs_name_to_id.find(impl->ud_name);
  if (it == _udfs_name_to_id.end()) return {-1, -1};
  auto& f = _udfs[it->second];
  // both counts must match (the reference's `&&` accepts a mismatch in one of them)
  if (impl->inputTypes.size() != f->num_in || impl->outputTypes.size() != f->num_out) return {-1, -1};
  return f->add_impl(std::move(impl));
}

udf_matcher_ptr udf_manager_t::get_matcher_for(const std::string& ud_name) {
  auto it = _udfs_name_to_id.find(ud_name);
  if (it == _udfs_name_to_id.end()) return nullptr;
  return std::make_unique<udf_matcher>(_udfs[it->second]->impls);
}

udf_matcher_ptr udf_manager_t::get_matcher_for(const std::string& ud_name, bool is_commutative,
                                               bool is_associative) {
  auto it = _udfs_name_to_id.find(ud_name);
  if (it == _udfs_name_to_id.end()) return nullptr;
  auto& f = _udfs[it->second];
  if ((!f->is_ass && is_associative) || (!f->is_com && is_commutative)) return nullptr;
  return std::make_unique<udf_matcher>(f->impls);
}

ud_impl_t* udf_manager_t::get_fn_impl(ud_impl_id_t id) {
  if (id.ud_id < 0 || (size_t)id.ud_id >= _udfs.size()) return nullptr;
  auto& f = _udfs[id.ud_id];
  if (id.impl_id < 0 || (size_t)id.impl_id >= f->impls.size()) return nullptr;
  return f->impls[id.impl_id].get();
}

ud_func_t* udf_manager_t::get_udf(const std::string& ud_name) {
  auto it = _udfs_name_to_id.find(ud_name);
  return it == _udfs_name_to_id.end() ? nullptr : _udfs[it->second].get();
}

ud_func_t* udf_manager_t::get_udf(ud_id_t id) {
  return (id >= 0 && (size_t)id < _udfs.size()) ? _udfs[id].get() : nullptr;
}

}  // namespace bbts
