// Built-in block formats and the format registry.
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <stdexcept>
#include "tensor.h"

namespace bbts {

namespace {

// Copies `bytes` of a payload (device or host, UVA) into a host vector for printing.
std::vector<char> fetch(const void* p, size_t bytes) {
  std::vector<char> h(bytes);
  if (bytes && cudaMemcpy(h.data(), p, bytes, cudaMemcpyDefault) != cudaSuccess) {
    cudaGetLastError();
    std::memcpy(h.data(), p, bytes);
  }
  return h;
}

float elem_as_float(const char* base, size_t i, int32_t elem, float scale) {
  if (elem == ELEM_F32) return ((const float*)base)[i];
  if (elem == ELEM_BF16) return __bfloat162float(((const __nv_bfloat16*)base)[i]);
  __nv_fp8_e4m3 q;
  std::memcpy(&q, base + i, 1);
  return float(q) * scale;
}

}  // namespace

tensor_creation_fs_t dense_creation_fs(int32_t elem) {
  auto init = [](void* here, const tensor_meta_t& meta) -> tensor_t& {
    auto& t = *(tensor_t*)here;
    t._meta = meta;
    t._meta.set_payload((char*)here + sizeof(tensor_meta_t));
    return t;
  };
  auto size = [elem](const tensor_meta_t& meta) {
    auto& m = meta.as<dense_tensor_meta_t>().m();
    return sizeof(tensor_meta_t) + (size_t)m.num_rows * m.num_cols * elem_size(elem);
  };
  auto print = [elem](const void* here, std::stringstream& ss) {
    auto& t = *(const dense_tensor_t*)here;
    auto& m = t.meta().m();
    auto h = fetch(t.raw(), (size_t)m.num_rows * m.num_cols * elem_size(elem));
    for (uint32_t r = 0; r < m.num_rows; ++r) {
      ss << "[";
      for (uint32_t c = 0; c < m.num_cols; ++c)
        ss << elem_as_float(h.data(), (size_t)r * m.num_cols + c, elem, m.scale)
           << (c + 1 == m.num_cols ? "" : ",");
      ss << "]\n";
    }
  };
  return tensor_creation_fs_t{size, init, print};
}

tensor_creation_fs_t ffnn_dense_creation_fs() {
  auto init = [](void* here, const tensor_meta_t& meta) -> tensor_t& {
    auto& t = *(tensor_t*)here;
    t._meta = meta;
    t._meta.set_payload((char*)here + sizeof(tensor_meta_t));
    return t;
  };
  auto size = [](const tensor_meta_t& meta) {
    auto& m = meta.as<ffnn_dense_meta_t>().m();
    size_t n = (size_t)m.num_rows * m.num_cols + (m.has_bias ? m.num_cols : 0);
    return sizeof(tensor_meta_t) + n * sizeof(float);
  };
  auto print = [](const void* here, std::stringstream& ss) {
    auto& t = *(const ffnn_dense_t*)here;
    auto& m = t.meta().m();
    auto h = fetch(t.data(), (size_t)m.num_rows * m.num_cols * 4);
    const float* d = (const float*)h.data();
    for (uint32_t r = 0; r < m.num_rows; ++r) {
      ss << "[";
      for (uint32_t c = 0; c < m.num_cols; ++c) ss << d[(size_t)r * m.num_cols + c] << (c + 1 == m.num_cols ? "" : ",");
      ss << "]\n";
    }
  };
  return tensor_creation_fs_t{size, init, print};
}

tensor_creation_fs_t cutensor_creation_fs() {
  auto init = [](void* here, const tensor_meta_t& meta) -> tensor_t& {
    auto& t = *(tensor_t*)here;
    t._meta = meta;
    t._meta.set_payload((char*)here + sizeof(tensor_meta_t));
    return t;
  };
  auto size = [](const tensor_meta_t& meta) {
    return sizeof(tensor_meta_t) + meta.as<cu_meta_t>().num_elem() * sizeof(float);
  };
  auto print = [](const void* here, std::stringstream& ss) {
    auto& t = *(const cu_t*)here;
    size_t n = t.meta().num_elem();
    auto h = fetch(t.data(), n * 4);
    const float* d = (const float*)h.data();
    ss << "dims[";
    for (uint32_t r = 0; r < t.meta().m().rank; ++r) ss << t.meta().m().dims[r] << (r + 1 == t.meta().m().rank ? "" : ",");
    ss << "]\n";
    for (size_t i = 0; i < n; ++i) ss << d[i] << " ";
    ss << "\n";
  };
  return tensor_creation_fs_t{size, init, print};
}

tensor_factory_t::tensor_factory_t() {
  register_fmt("dense", dense_creation_fs(ELEM_F32));
  register_fmt("dense_bf16", dense_creation_fs(ELEM_BF16));
  register_fmt("dense_e4m3", dense_creation_fs(ELEM_E4M3));
}

tfid_t tensor_factory_t::register_fmt(const std::string& name, const tensor_creation_fs_t& fs) {
  auto it = _reg_fmts.find(name);
  if (it != _reg_fmts.end()) return it->second;  // registering twice keeps the first
  tfid_t id = (tfid_t)_fmt_fs.size();
  _reg_fmts[name] = id;
  _fmt_fs.push_back(fs);
  return id;
}

tfid_t tensor_factory_t::get_tensor_ftm(const std::string& name) const {
  auto it = _reg_fmts.find(name);
  return it == _reg_fmts.end() ? -1 : it->second;
}

size_t tensor_factory_t::get_tensor_size(const tensor_meta_t& meta) const {
  if (meta.fmt_id < 0 || (size_t)meta.fmt_id >= _fmt_fs.size())
    throw std::runtime_error("get_tensor_size: format " + std::to_string(meta.fmt_id) + " is not registered");
  return _fmt_fs[meta.fmt_id].get_size(meta);
}

size_t tensor_factory_t::get_payload_size(const tensor_meta_t& meta) const {
  return get_tensor_size(meta) - sizeof(tensor_meta_t);
}

void tensor_factory_t::print_tensor(tensor_t* here, std::stringstream& ss) const {
  if (here->_meta.fmt_id < 0 || (size_t)here->_meta.fmt_id >= _fmt_fs.size())
    throw std::runtime_error("print_tensor: format " + std::to_string(here->_meta.fmt_id) + " is not registered");
  _fmt_fs[here->_meta.fmt_id].print(here, ss);
}

tensor_t& tensor_factory_t::init_tensor(tensor_t* here, const tensor_meta_t& meta) const {
  if (meta.fmt_id < 0 || (size_t)meta.fmt_id >= _fmt_fs.size())
    throw std::runtime_error("init_tensor: format " + std::to_string(meta.fmt_id) + " is not registered");
  tensor_t& out = _fmt_fs[meta.fmt_id].init_tensor(here, meta);
  out._meta.fmt_id = meta.fmt_id;
  return out;
}

const std::string& tensor_factory_t::fmt_name(tfid_t id) const {
  static const std::string none = "";
  for (const auto& kv : _reg_fmts)
    if (kv.second == id) return kv.first;
  return none;
}

}  // namespace bbts
