// .sbbts / .bbts programs and their single-node compilation.
#include "compiler.h"

#include <cstring>
#include <fstream>
#include <stdexcept>

namespace bbts {

// ------------------------------------------------------------------ .sbbts text
void abstract_ud_spec_t::write(std::ostream& f) const {
  f << id << " " << ud_name << " " << input_types.size() << " ";
  for (auto& s : input_types) f << s << " ";
  f << output_types.size() << " ";
  for (auto& s : output_types) f << s << " ";
  f << "\n";
}

void abstract_ud_spec_t::read(std::istream& f) {
  size_t ni = 0, no = 0;
  if (!(f >> id >> ud_name >> ni)) throw std::runtime_error("sbbts: truncated function spec");
  input_types.resize(ni);
  for (auto& s : input_types) f >> s;
  f >> no;
  output_types.resize(no);
  for (auto& s : output_types) f >> s;
  if (!f) throw std::runtime_error("sbbts: truncated function spec");
}

void abstract_command_t::write(std::ostream& f) const {
  const char* t = type == abstract_command_type_t::APPLY ? "APPLY" : type == abstract_command_type_t::REDUCE ? "REDUCE" : "DELETE";
  f << ud_id << " " << t << " " << input_tids.size() << " ";
  for (auto x : input_tids) f << x << " ";
  f << output_tids.size() << " ";
  for (auto x : output_tids) f << x << " ";
  f << params.size() << " ";
  for (size_t i = 0; i < params.size(); ++i) {
    char pt = i < param_types.size() ? param_types[i] : 'i';
    if (pt == 'f') f << "float " << params[i].f << " ";
    else if (pt == 'u') f << "uint " << params[i].u << " ";
    else f << "int " << params[i].i << " ";
  }
  f << "\n";
}

void abstract_command_t::read(std::istream& f) {
  std::string ts;
  size_t ni = 0, no = 0, np = 0;
  if (!(f >> ud_id >> ts >> ni)) throw std::runtime_error("sbbts: truncated command");
  if (ts == "APPLY") type = abstract_command_type_t::APPLY;
  else if (ts == "REDUCE") type = abstract_command_type_t::REDUCE;
  else if (ts == "DELETE") type = abstract_command_type_t::DELETE;
  else throw std::runtime_error("sbbts: unknown command type " + ts);
  if (type == abstract_command_type_t::REDUCE && ni == 0) throw std::runtime_error("sbbts: REDUCE without inputs");
  input_tids.resize(ni);
  for (auto& x : input_tids) f >> x;
  f >> no;
  output_tids.resize(no);
  for (auto& x : output_tids) f >> x;
  f >> np;
  params.clear();
  param_types.clear();
  for (size_t i = 0; i < np; ++i) {
    std::string pt;
    command_param_t p;
    f >> pt;
    if (pt == "int") { f >> p.i; param_types.push_back('i'); }
    else if (pt == "float") { f >> p.f; param_types.push_back('f'); }
    else if (pt == "uint") { f >> p.u; param_types.push_back('u'); }
    else throw std::runtime_error("sbbts: unknown parameter type " + pt);
    params.push_back(p);
  }
  if (!f) throw std::runtime_error("sbbts: truncated command");
}

void compile_source_file_t::write(std::ostream& f) const {
  f << function_specs.size() << "\n";
  for (auto& s : function_specs) s.write(f);
  f << commands.size() << "\n";
  for (auto& c : commands) c.write(f);
}

void compile_source_file_t::read(std::istream& f) {
  size_t nf = 0, nc = 0;
  if (!(f >> nf)) throw std::runtime_error("sbbts: empty file");
  function_specs.resize(nf);
  for (auto& s : function_specs) s.read(f);
  if (!(f >> nc)) throw std::runtime_error("sbbts: missing command count");
  commands.resize(nc);
  for (auto& c : commands) c.read(f);
}

std::vector<command_ptr_t> compile_single_node(const compile_source_file_t& src, udf_manager_t& udm,
                                               command_id_t first_id) {
  // resolve every spec to the GPU impl whose types match
  std::unordered_map<int32_t, ud_impl_t*> impl_of;
  for (auto& s : src.function_specs) {
    auto m = udm.get_matcher_for(s.ud_name);
    if (!m) throw std::runtime_error("Could not match ud " + s.ud_name);
    ud_impl_t* impl = m->findMatch(s.input_types, s.output_types, true);
    if (!impl) throw std::runtime_error("Could not find a matching ud function for " + s.ud_name);
    impl_of[s.id] = impl;
  }
  std::vector<command_ptr_t> out;
  command_id_t cur = first_id;
  for (auto& c : src.commands) {
    if (c.type == abstract_command_type_t::DELETE) {
      std::vector<command_t::tid_node_id_t> in;
      for (auto t : c.input_tids) in.push_back({t, 0});
      if (!in.empty()) out.push_back(command_t::create_delete(cur++, in));
      continue;
    }
    auto it = impl_of.find(c.ud_id);
    if (it == impl_of.end()) throw std::runtime_error("command names unknown function spec " + std::to_string(c.ud_id));
    ud_impl_t* impl = it->second;
    std::vector<command_t::tid_node_id_t> in, o;
    for (auto t : c.input_tids) in.push_back({t, 0});
    for (auto t : c.output_tids) o.push_back({t, 0});
    if (c.type == abstract_command_type_t::APPLY) {
      out.push_back(command_t::create_apply(cur++, impl->impl_id, true, c.params, in, o));
    } else {
      ud_func_t* f = udm.get_udf(impl->impl_id.ud_id);
      if (!f || !f->is_ass || !f->is_com) throw std::runtime_error("REDUCE needs an associative, commutative ud");
      if (o.size() != 1) throw std::runtime_error("REDUCE has exactly one output");
      out.push_back(command_t::create_reduce(cur++, impl->impl_id, true, c.params, in, o[0]));
    }
  }
  return out;
}

// ------------------------------------------------------------------ .bbts binary
// Layout (little endian): u64 count; per command: i32 type; string ud_name;
// u8 is_gpu; u64 n + strings input types; u64 n + strings output types;
// u64 n + n x 8-byte (tid, node) tuples for inputs and for outputs;
// u64 n + n x 4-byte parameters. Strings are u64 length + bytes. The 8-byte
// tuples are std::tuple<tid_t, node_id_t> written as raw memory by the
// reference, whose libstdc++ layout stores the node first and the tid second.
namespace {
template <class T> void put(std::ofstream& f, T v) { f.write((const char*)&v, sizeof(T)); }
template <class T> T get(std::ifstream& f) {
  T v{};
  f.read((char*)&v, sizeof(T));
  if (!f) throw std::runtime_error("bbts: truncated file");
  return v;
}
void put_str(std::ofstream& f, const std::string& s) {
  put<uint64_t>(f, s.size());
  f.write(s.data(), (std::streamsize)s.size());
}
std::string get_str(std::ifstream& f) {
  uint64_t n = get<uint64_t>(f);
  if (n > (1u << 20)) throw std::runtime_error("bbts: implausible string length");
  std::string s(n, '\0');
  f.read(s.data(), (std::streamsize)n);
  return s;
}
void put_tids(std::ofstream& f, const std::vector<std::pair<tid_t, node_id_t>>& v) {
  put<uint64_t>(f, v.size());
  for (auto& x : v) {
    put<int32_t>(f, x.second);
    put<int32_t>(f, x.first);
  }
}
std::vector<std::pair<tid_t, node_id_t>> get_tids(std::ifstream& f) {
  uint64_t n = get<uint64_t>(f);
  if (n > (1u << 24)) throw std::runtime_error("bbts: implausible tensor count");
  std::vector<std::pair<tid_t, node_id_t>> v(n);
  for (auto& x : v) {
    x.second = get<int32_t>(f);
    x.first = get<int32_t>(f);
  }
  return v;
}
}  // namespace

bool parsed_command_list_t::serialize(const std::string& path) const {
  std::ofstream f(path, std::ios::out | std::ios::trunc | std::ios::binary);
  if (!f.is_open()) return false;
  put<uint64_t>(f, commands.size());
  for (auto& c : commands) {
    put<int32_t>(f, (int32_t)c.type);
    put_str(f, c.def.ud_name);
    put<uint8_t>(f, c.def.is_gpu ? 1 : 0);
    put<uint64_t>(f, c.def.input_types.size());
    for (auto& s : c.def.input_types) put_str(f, s);
    put<uint64_t>(f, c.def.output_types.size());
    for (auto& s : c.def.output_types) put_str(f, s);
    put_tids(f, c.inputs);
    put_tids(f, c.outputs);
    put<uint64_t>(f, c.parameters.size());
    for (auto& p : c.parameters) put<uint32_t>(f, p.u);
  }
  return (bool)f;
}

bool parsed_command_list_t::deserialize(const std::string& path) {
  std::ifstream f(path, std::ios::in | std::ios::binary);
  if (!f.is_open()) return false;
  commands.clear();
  uint64_t n = get<uint64_t>(f);
  for (uint64_t i = 0; i < n; ++i) {
    parsed_command_t c;
    c.type = (parsed_command_t::op_type_t)get<int32_t>(f);
    c.def.ud_name = get_str(f);
    c.def.is_gpu = get<uint8_t>(f) != 0;
    uint64_t ni = get<uint64_t>(f);
    for (uint64_t j = 0; j < ni; ++j) c.def.input_types.push_back(get_str(f));
    uint64_t no = get<uint64_t>(f);
    for (uint64_t j = 0; j < no; ++j) c.def.output_types.push_back(get_str(f));
    c.inputs = get_tids(f);
    c.outputs = get_tids(f);
    uint64_t np = get<uint64_t>(f);
    for (uint64_t j = 0; j < np; ++j) {
      command_param_t p;
      p.u = get<uint32_t>(f);
      c.parameters.push_back(p);
    }
    commands.push_back(std::move(c));
  }
  return true;
}

std::vector<command_ptr_t> load_parsed(const parsed_command_list_t& cmds, udf_manager_t& udm,
                                       command_id_t first_id) {
  std::vector<command_ptr_t> out;
  command_id_t cur = first_id;
  auto single = [](const std::vector<std::pair<tid_t, node_id_t>>& v) {
    for (auto& x : v)
      if (x.second != 0) throw std::runtime_error("command names node " + std::to_string(x.second) + "; this runtime has one node");
  };
  for (auto& c : cmds.commands) {
    single(c.inputs);
    single(c.outputs);
    switch (c.type) {
      case parsed_command_t::op_type_t::MOVE:
        if (c.inputs.size() != 1 || c.outputs.empty()) throw std::runtime_error("malformed MOVE");
        break;  // node 0 to node 0: nothing to do
      case parsed_command_t::op_type_t::DELETE: {
        if (!c.outputs.empty()) throw std::runtime_error("A delete operation must have no outputs.");
        if (c.inputs.empty()) throw std::runtime_error("A delete operation must have at least one input.");
        std::vector<command_t::tid_node_id_t> in;
        for (auto& x : c.inputs) in.push_back({x.first, x.second});
        out.push_back(command_t::create_delete(cur++, in));
        break;
      }
      case parsed_command_t::op_type_t::APPLY:
      case parsed_command_t::op_type_t::REDUCE: {
        const bool apply = c.type == parsed_command_t::op_type_t::APPLY;
        if (c.outputs.empty()) throw std::runtime_error("An APPLY must have at least one output.");
        auto m = apply ? udm.get_matcher_for(c.def.ud_name) : udm.get_matcher_for(c.def.ud_name, true, true);
        if (!m) throw std::runtime_error("Could not find function " + c.def.ud_name + (apply ? " in APPLY." : " in REDUCE (it must be associative and commutative)."));
        // every impl of this library runs on the GPU; a CPU request is served by the GPU impl
        ud_impl_t* ud = m->findMatch(c.def.input_types, c.def.output_types, true);
        if (!ud) throw std::runtime_error("No matching implementation for the function " + c.def.ud_name + ".");
        std::vector<command_t::tid_node_id_t> in, o;
        for (auto& x : c.inputs) in.push_back({x.first, x.second});
        for (auto& x : c.outputs) o.push_back({x.first, x.second});
        if (apply) {
          out.push_back(command_t::create_apply(cur++, ud->impl_id, true, c.parameters, in, o));
        } else {
          if (o.size() != 1) throw std::runtime_error("A reduce must have exactly one output.");
          out.push_back(command_t::create_reduce(cur++, ud->impl_id, true, c.parameters, in, o[0]));
        }
        break;
      }
    }
  }
  return out;
}

}  // namespace bbts
