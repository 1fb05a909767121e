// On-disk command programs and their single-node compilation.
//
// .sbbts  text "compile source" of abstract ud specs + abstract commands
//         (src/commands/command_compiler.h:33-85 specs, :391-501 commands,
//         :977-1027 file), compiled like command_compiler_t::compile
//         (:503-975) with every command placed on node 0 and the GPU impl of
//         each spec picked by real type matching;
// .bbts   binary parsed command list (src/commands/parsed_command.h:194-383),
//         compiled like command_loader_t::compile (command_loader.h:10-182).
#pragma once
#include <istream>
#include <ostream>
#include <string>
#include <vector>
#include "command.h"
#include "ud_function.h"

namespace bbts {

enum class abstract_command_type_t : int32_t { APPLY = 0, REDUCE = 1, DELETE = 2 };

struct abstract_ud_spec_t {
  int32_t id = 0;
  std::string ud_name;
  std::vector<std::string> input_types, output_types;
  void write(std::ostream& f) const;
  void read(std::istream& f);
};

struct abstract_command_t {
  int32_t ud_id = 0;
  abstract_command_type_t type = abstract_command_type_t::APPLY;
  std::vector<tid_t> input_tids, output_tids;
  std::vector<command_param_t> params;
  std::vector<char> param_types;  // 'i', 'f', 'u' per parameter (kept for round trips)
  void write(std::ostream& f) const;
  void read(std::istream& f);
};

struct compile_source_file_t {
  std::vector<abstract_ud_spec_t> function_specs;
  std::vector<abstract_command_t> commands;
  void write(std::ostream& f) const;
  void read(std::istream& f);
};

// Compiles an abstract program for one node; command ids start at first_id.
std::vector<command_ptr_t> compile_single_node(const compile_source_file_t& src, udf_manager_t& udm,
                                               command_id_t first_id);

struct parsed_command_t {
  enum class op_type_t : int32_t { APPLY = 0, REDUCE = 1, MOVE = 2, DELETE = 3 };
  struct ud_def_t {
    std::string ud_name;
    std::vector<std::string> input_types, output_types;
    bool is_gpu = false;
  };
  op_type_t type = op_type_t::APPLY;
  ud_def_t def;
  std::vector<std::pair<tid_t, node_id_t>> inputs, outputs;
  std::vector<command_param_t> parameters;
};

struct parsed_command_list_t {
  std::vector<parsed_command_t> commands;
  bool serialize(const std::string& path) const;
  bool deserialize(const std::string& path);
};

// command_loader_t::compile for one node: MOVE / broadcast between node 0
// and itself are dropped; anything naming another node is refused.
std::vector<command_ptr_t> load_parsed(const parsed_command_list_t& cmds, udf_manager_t& udm,
                                       command_id_t first_id);

}  // namespace bbts
