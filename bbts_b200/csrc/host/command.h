// Block commands: a flat, memcpy-able record (header + parameters + nodes +
// inputs + outputs), as in BarbaTOS's src/commands/command.h:228-542.
#pragma once
#include <algorithm>
#include <cassert>
#include <cstring>
#include <memory>
#include <sstream>
#include <vector>
#include "ud_function.h"

namespace bbts {

using command_id_t = int32_t;
using node_id_t = int32_t;

struct command_t;
struct command_deleter_t {
  void operator()(command_t* p) { delete[] ((char*)p); }
};
using command_ptr_t = std::unique_ptr<command_t, command_deleter_t>;

struct command_t {
  enum op_type_t : int32_t { APPLY = 0, REDUCE = 1, MOVE = 2, DELETE = 3, SHUTDOWN = 4 };

  struct tid_node_id_t {
    tid_t tid;
    node_id_t node;
  };
  using tensor_id_list_t = raw_vector_t<tid_node_id_t>;
  using node_list_t = raw_vector_t<node_id_t>;

  command_id_t id;
  op_type_t type;
  ud_impl_id_t fun_id = {-1, -1};
  union {
    size_t num_bytes;
    bool is_gpu;
  } nfo;

  size_t get_num_inputs() const { return _num_inputs; }
  size_t get_num_outputs() const { return _num_outputs; }
  tid_node_id_t& get_input(int32_t i) { return _inputs()[i]; }
  const tid_node_id_t& get_input(int32_t i) const { return _inputs()[i]; }
  tid_node_id_t& get_output(int32_t i) { return _outputs()[i]; }
  const tid_node_id_t& get_output(int32_t i) const { return _outputs()[i]; }
  tensor_id_list_t get_inputs() const { return {_inputs(), _num_inputs}; }
  tensor_id_list_t get_outputs() const { return {_outputs(), _num_outputs}; }
  node_list_t get_nodes() const { return {_nodes(), _num_nodes}; }
  command_param_list_t get_parameters() const { return {_params(), _num_parameters}; }
  node_id_t get_root_node() const { return _nodes()[0]; }

  bool is_apply() const { return type == APPLY; }
  bool is_reduce() const { return type == REDUCE; }
  bool is_delete() const { return type == DELETE; }
  bool is_move() const { return type == MOVE && _num_outputs == 1; }
  bool is_broadcast() const { return type == MOVE && _num_outputs != 1; }
  bool is_local_reduce(node_id_t n) const {
    if (type != REDUCE) return false;
    for (auto x : get_nodes()) if (x != n) return false;
    return true;
  }
  bool uses_node(node_id_t n) const {
    for (auto x : get_nodes()) if (x == n) return true;
    return false;
  }
  size_t num_bytes() const { return _bytes(_num_parameters, _num_nodes, _num_inputs, _num_outputs); }

  command_ptr_t clone() const {
    char* p = new char[num_bytes()];
    std::memcpy(p, this, num_bytes());
    return command_ptr_t((command_t*)p);
  }

  void print(std::stringstream& ss) const {
    static const char* names[] = {"APPLY", "REDUCE", "MOVE", "DELETE", "SHUTDOWN"};
    ss << "{.id : " << id << " .type : " << names[type] << " .inputs : [";
    for (size_t i = 0; i < _num_inputs; ++i) ss << "(" << get_input(i).tid << ", " << get_input(i).node << "),";
    ss << "] .outputs : [";
    for (size_t i = 0; i < _num_outputs; ++i) ss << "(" << get_output(i).tid << ", " << get_output(i).node << "),";
    ss << "]}\n";
  }

  static command_ptr_t create_apply(command_id_t id, ud_impl_id_t fun, bool is_gpu,
                                    const std::vector<command_param_t>& params,
                                    const std::vector<tid_node_id_t>& in, const std::vector<tid_node_id_t>& out) {
    auto c = _alloc(params.size(), 1, in.size(), out.size());
    c->id = id; c->type = APPLY; c->fun_id = fun; c->nfo.num_bytes = 0; c->nfo.is_gpu = is_gpu;
    c->_nodes()[0] = out.empty() ? (in.empty() ? 0 : in[0].node) : out[0].node;
    c->_fill(params, in, out);
    return c;
  }

  static command_ptr_t create_reduce(command_id_t id, ud_impl_id_t fun, bool is_gpu,
                                     const std::vector<command_param_t>& params,
                                     const std::vector<tid_node_id_t>& in, const tid_node_id_t& out) {
    std::vector<node_id_t> nodes{out.node};
    for (auto& i : in)
      if (std::find(nodes.begin(), nodes.end(), i.node) == nodes.end()) nodes.push_back(i.node);
    auto c = _alloc(params.size(), nodes.size(), in.size(), 1);
    c->id = id; c->type = REDUCE; c->fun_id = fun; c->nfo.num_bytes = 0; c->nfo.is_gpu = is_gpu;
    for (size_t i = 0; i < nodes.size(); ++i) c->_nodes()[i] = nodes[i];
    c->_fill(params, in, {out});
    return c;
  }

  static command_ptr_t create_move(command_id_t id, tid_node_id_t in, tid_node_id_t out) {
    auto c = _alloc(0, 2, 1, 1);
    c->id = id; c->type = MOVE; c->fun_id = {-1, -1}; c->nfo.num_bytes = 0;
    c->_nodes()[0] = in.node;
    c->_nodes()[1] = out.node;
    c->_fill({}, {in}, {out});
    return c;
  }

  static command_ptr_t create_broadcast(command_id_t id, tid_node_id_t in, const std::vector<tid_node_id_t>& out) {
    auto c = _alloc(0, 1 + out.size(), 1, out.size());
    c->id = id; c->type = MOVE; c->fun_id = {-1, -1}; c->nfo.num_bytes = 0;
    c->_nodes()[0] = in.node;
    for (size_t i = 0; i < out.size(); ++i) c->_nodes()[1 + i] = out[i].node;
    c->_fill({}, {in}, out);
    return c;
  }

  static command_ptr_t create_delete(command_id_t id, const std::vector<tid_node_id_t>& in) {
    auto c = _alloc(0, 1, in.size(), 0);
    c->id = id; c->type = DELETE; c->fun_id = {-1, -1}; c->nfo.num_bytes = 0;
    c->_nodes()[0] = in.empty() ? 0 : in[0].node;
    c->_fill({}, in, {});
    return c;
  }

  static command_ptr_t create_shutdown(node_id_t node) {
    auto c = _alloc(0, 1, 0, 0);
    c->id = -1; c->type = SHUTDOWN; c->fun_id = {-1, -1}; c->nfo.num_bytes = 0;
    c->_nodes()[0] = node;
    return c;
  }

 private:
  uint16_t _num_parameters, _num_nodes, _num_inputs, _num_outputs;
  uint16_t _params_offset, _node_offset, _input_offset, _output_offset;

  static size_t _bytes(size_t np, size_t nn, size_t ni, size_t no) {
    return sizeof(command_t) + np * sizeof(command_param_t) + nn * sizeof(node_id_t) +
           (ni + no) * sizeof(tid_node_id_t);
  }
  static command_ptr_t _alloc(size_t np, size_t nn, size_t ni, size_t no) {
    size_t bytes = _bytes(np, nn, ni, no);
    char* p = new char[bytes];
    std::memset(p, 0, bytes);
    command_ptr_t c((command_t*)p);
    c->_num_parameters = (uint16_t)np;
    c->_num_nodes = (uint16_t)nn;
    c->_num_inputs = (uint16_t)ni;
    c->_num_outputs = (uint16_t)no;
    size_t off = sizeof(command_t);
    c->_params_offset = (uint16_t)off; off += np * sizeof(command_param_t);
    c->_node_offset = (uint16_t)off; off += nn * sizeof(node_id_t);
    c->_input_offset = (uint16_t)off; off += ni * sizeof(tid_node_id_t);
    c->_output_offset = (uint16_t)off;
    return c;
  }
  void _fill(const std::vector<command_param_t>& params, const std::vector<tid_node_id_t>& in,
             const std::vector<tid_node_id_t>& out) {
    for (size_t i = 0; i < params.size(); ++i) _params()[i] = params[i];
    for (size_t i = 0; i < in.size(); ++i) _inputs()[i] = in[i];
    for (size_t i = 0; i < out.size(); ++i) _outputs()[i] = out[i];
  }
  command_param_t* _params() const { return (command_param_t*)((char*)this + _params_offset); }
  node_id_t* _nodes() const { return (node_id_t*)((char*)this + _node_offset); }
  tid_node_id_t* _inputs() const { return (tid_node_id_t*)((char*)this + _input_offset); }
  tid_node_id_t* _outputs() const { return (tid_node_id_t*)((char*)this + _output_offset); }
};

}  // namespace bbts
