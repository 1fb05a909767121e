// Tensor handles and formats, laid out like BarbaTOS's
// (src/tensor/tensor.h:20-66): a 4-byte format id followed by a 256-byte
// format-specific meta blob (sizeof(tensor_meta_t) == 260).
//
// B200 residency: a block's payload lives in HBM, not behind its header. The
// last 8 bytes of the meta blob hold the payload address ("payload slot") and
// the 8 bytes before them a tag (the address XOR a constant) that marks the
// slot as set by this library. tensor_factory_t::init_tensor sets the slot to
// the bytes right after the header, which reproduces the reference's
// contiguous layout (builtin_formats.cc:18-21); block storage overrides it
// with a device address. A tensor whose slot is not tagged -- one that a
// reference node created and initialised itself -- has its payload right
// after the 260-byte header, as in the reference (dense_tensor_t::data(),
// builtin_formats.h:36-39); tensor_t::payload() resolves both cases.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

namespace bbts {

using tid_t = int32_t;
const tid_t TID_NONE = -1;
using tfid_t = int32_t;

struct tensor_meta_t {
  static const size_t MAX_META_SIZE = 256;
  static const size_t PAYLOAD_SLOT = MAX_META_SIZE - sizeof(void*);  // offset of the payload address
  static const size_t PAYLOAD_TAG = PAYLOAD_SLOT - sizeof(uint64_t);  // offset of the slot's tag
  static constexpr uint64_t kPayloadMagic = 0x62627862323030ull;      // "bbxb200"

  template <class T>
  T& as() const { return *((T*)this); }

  tfid_t fmt_id;
  char _blob[MAX_META_SIZE];

  // True when this library set the payload slot (the tag matches).
  bool payload_tagged() const {
    uint64_t p, tag;
    std::memcpy(&p, _blob + PAYLOAD_SLOT, sizeof(p));
    std::memcpy(&tag, _blob + PAYLOAD_TAG, sizeof(tag));
    return (tag ^ p) == kPayloadMagic;
  }
  // The payload address this library set (nullptr for a block with no
  // resident payload), or nullptr when the slot is not tagged.
  void* payload() const {
    if (!payload_tagged()) return nullptr;
    uint64_t p;
    std::memcpy(&p, _blob + PAYLOAD_SLOT, sizeof(p));
    return (void*)p;
  }
  void set_payload(void* p) {
    const uint64_t v = (uint64_t)p, tag = v ^ kPayloadMagic;
    std::memcpy(_blob + PAYLOAD_SLOT, &v, sizeof(v));
    std::memcpy(_blob + PAYLOAD_TAG, &tag, sizeof(tag));
  }
};
static_assert(sizeof(tensor_meta_t) == 260, "tensor_meta_t must keep the reference layout");

struct tensor_t {
  tensor_t(const tensor_t&) = delete;
  void operator=(const tensor_t&) = delete;

  template <class T>
  T& as() const { return *((T*)this); }

  // The payload: the tagged slot's address (nullptr for a block with no
  // resident payload), else the bytes after the header (the reference's layout).
  void* payload() const {
    if (_meta.payload_tagged()) return _meta.payload();
    return (void*)((const char*)this + sizeof(tensor_meta_t));
  }

  tensor_meta_t _meta;
  char _blob[0];
};

struct tensor_creation_fs_t {
  std::function<size_t(const tensor_meta_t&)> get_size;
  std::function<tensor_t&(void* here, const tensor_meta_t&)> init_tensor;
  std::function<void(const void* here, std::stringstream& ss)> print;
};

// Element types of block payloads (values match BBX_F32 / BBX_BF16 / BBX_E4M3).
enum elem_t : int32_t { ELEM_F32 = 0, ELEM_BF16 = 1, ELEM_E4M3 = 2 };
inline size_t elem_size(int32_t e) { return e == ELEM_F32 ? 4 : e == ELEM_BF16 ? 2 : 1; }

// "dense": row-major FP32 {num_rows, num_cols} (src/tensor/builtin_formats.h:7-45).
// "dense_bf16" / "dense_e4m3" share the meta and store 2- or 1-byte elements;
// e4m3 blocks carry their dequantisation scale at `scale`.
struct dense_tensor_meta_t : public tensor_meta_t {
  struct m_t {
    uint32_t num_rows;
    uint32_t num_cols;
    float scale;  // e4m3 only
  };
  m_t& m() const { return *((m_t*)_blob); }
  dense_tensor_meta_t(tfid_t id) : tensor_meta_t{} { fmt_id = id; }
  dense_tensor_meta_t(tfid_t id, uint32_t rows, uint32_t cols) : tensor_meta_t{} {
    fmt_id = id;
    m() = {rows, cols, 1.0f};
  }
};

struct dense_tensor_t : public tensor_t {
  dense_tensor_meta_t& meta() const { return *((dense_tensor_meta_t*)&_meta); }
  float* data() const { return (float*)payload(); }
  void* raw() const { return payload(); }
};

// "ffnn_dense": row-major FP32 with an optional bias row stored after the data
// (applications/fnn/ffnn_types.h:7-52, size at ffnn_types.cc:18-26).
struct ffnn_dense_meta_t : public tensor_meta_t {
  struct m_t {
    uint32_t num_rows;
    uint32_t num_cols;
    bool has_bias;
  };
  m_t& m() const { return *((m_t*)_blob); }
  ffnn_dense_meta_t(tfid_t id) : tensor_meta_t{} { fmt_id = id; }
  ffnn_dense_meta_t(tfid_t id, bool has_bias, uint32_t rows, uint32_t cols) : tensor_meta_t{} {
    fmt_id = id;
    m() = {rows, cols, has_bias};
  }
};

struct ffnn_dense_t : public tensor_t {
  ffnn_dense_meta_t& meta() const { return *((ffnn_dense_meta_t*)&_meta); }
  float* data() const { return (float*)payload(); }
  float* bias() const { return data() + (size_t)meta().m().num_rows * meta().m().num_cols; }
};

// "cutensor": column-major FP32, rank <= 4, int64 dims (libraries/cutensor/cu.h:60-169).
struct cu_shape_t {
  uint32_t rank;
  int64_t dims[4];
};
struct cu_meta_t : public tensor_meta_t {
  cu_shape_t& m() const { return *((cu_shape_t*)_blob); }
  cu_meta_t(tfid_t id) : tensor_meta_t{} { fmt_id = id; }
  cu_meta_t(tfid_t id, const std::vector<int64_t>& dims) : tensor_meta_t{} {
    fmt_id = id;
    m().rank = (uint32_t)dims.size();
    for (size_t r = 0; r < dims.size() && r < 4; ++r) m().dims[r] = dims[r];
  }
  size_t num_elem() const {
    size_t n = 1;
    for (uint32_t r = 0; r < m().rank; ++r) n *= (size_t)m().dims[r];
    return n;
  }
};
struct cu_t : public tensor_t {
  cu_meta_t& meta() const { return *((cu_meta_t*)&_meta); }
  void* data() const { return payload(); }
};

// Registry of formats by name (src/tensor/tensor_factory.h:12-41), with the
// reference's data members in the reference's order, so that code of this
// library running on a reference node's factory sees the same layout.
// register_fmt keeps the first registration of a name, as the reference does,
// but returns the format's id (the reference always returns -1).
class tensor_factory_t {
 public:
  tensor_factory_t();
  tfid_t register_fmt(const std::string& name, const tensor_creation_fs_t& fs);
  tfid_t get_tensor_ftm(const std::string& name) const;
  size_t get_tensor_size(const tensor_meta_t& meta) const;
  // payload bytes only (what block storage allocates in HBM)
  size_t get_payload_size(const tensor_meta_t& meta) const;
  void print_tensor(tensor_t* here, std::stringstream& ss) const;
  tensor_t& init_tensor(tensor_t* here, const tensor_meta_t& meta) const;
  const std::string& fmt_name(tfid_t id) const;

 private:
  std::unordered_map<std::string, tfid_t> _reg_fmts;
  std::vector<tensor_creation_fs_t> _fmt_fs;
};
using tensor_factory_ptr_t = std::shared_ptr<tensor_factory_t>;

// Creation functions of the built-in formats.
tensor_creation_fs_t dense_creation_fs(int32_t elem);
tensor_creation_fs_t ffnn_dense_creation_fs();
tensor_creation_fs_t cutensor_creation_fs();

}  // namespace bbts
