// Per-node dataflow scheduler (src/commands/reservation_station.h:17-74).
//
// Tracks, per tensor, the number of pending readers, whether a command is
// writing it, whether it exists, and whether a DELETE is waiting for it; a
// command becomes ready when all its inputs exist. The ready list is popped
// LIFO exactly like the reference (reservation_station.cc:213-214) unless a
// priority function is installed, in which case the highest-priority ready
// command is popped first (this is how the learned cost model orders the
// station). Deletes are deferred until the last reader retires.
//
// Single node: commands whose root is another node are rejected (the
// multi-node notification machinery rides on MPI, which this build drops).
#pragma once
#include <condition_variable>
#include <functional>
#include <mutex>
#include <unordered_map>
#include <vector>
#include "command.h"

namespace bbts {

class reservation_station_t {
 public:
  reservation_station_t(node_id_t node_id, int32_t num_nodes);

  bool queue_command(command_ptr_t cmd);
  bool retire_command(command_ptr_t cmd);
  command_ptr_t get_next_command();       // blocks until a command is ready or shutdown
  command_ptr_t try_get_next_command();   // non-blocking; nullptr if nothing is ready
  void register_tensor(tid_t tid);
  tid_t get_to_remove();                  // blocks; -1 on shutdown
  bool try_get_to_remove(tid_t* tid);     // non-blocking
  void retire_remove(tid_t tid);
  void shutdown();
  void clear();
  void wait_until_finished();
  void execute_scheduled_async();
  void stop_executing();

  // Higher value = popped earlier. An empty function restores LIFO order.
  void set_priority(std::function<double(const command_t&)> prio);

  template <class fn> void add_queued_hook(fn f) { _queued_hook = f; }
  template <class fn> void add_scheduled_hook(fn f) { _scheduled_hook = f; }
  template <class fn> void add_retired_hook(fn f) { _retired_hook = f; }

  size_t num_ready() {
    std::lock_guard<std::mutex> lk(_m);
    return _execute.size();
  }
  size_t num_to_retire() {
    std::lock_guard<std::mutex> lk(_m);
    return _num_local_to_retire;
  }

 private:
  struct tensor_state_t {
    int32_t num_to_read = 0;
    bool writing_tensor = false;
    bool is_created = false;
    bool scheduled_for_deletion = false;
  };

  bool _queue_local(command_ptr_t cmd);
  bool _retire_local(command_ptr_t cmd);
  void _tensor_created(tid_t tid);
  void _schedule(command_ptr_t cmd);
  void _remove_tensor(tid_t tid);
  command_ptr_t _pop_locked();

  std::mutex _m;
  std::condition_variable _cv, _retire_cv, _deletion_cv;
  bool _is_executing = false;
  bool _shutdown = false;
  size_t _num_local_to_retire = 0;
  size_t _num_to_delete = 0;
  node_id_t _my_rank;
  int32_t _num_nodes;
  command_id_t _last_cmd = -1;
  std::vector<command_ptr_t> _execute;
  std::unordered_map<command_id_t, std::pair<command_ptr_t, int32_t>> _local_commands;
  std::unordered_multimap<tid_t, command_id_t> _waiting_for;
  std::unordered_map<tid_t, tensor_state_t> _tensors;
  std::vector<tid_t> _to_delete;
  std::function<double(const command_t&)> _priority;
  std::function<void(command_id_t)> _queued_hook = [](command_id_t) {};
  std::function<void(command_id_t)> _scheduled_hook = [](command_id_t) {};
  std::function<void(command_id_t)> _retired_hook = [](command_id_t) {};
};
using reservation_station_ptr_t = std::shared_ptr<reservation_station_t>;

}  // namespace bbts
