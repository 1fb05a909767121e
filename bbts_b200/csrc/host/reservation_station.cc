// Reservation station (src/commands/reservation_station.cc:20-761, local part).
#include "reservation_station.h"

namespace bbts {

reservation_station_t::reservation_station_t(node_id_t node_id, int32_t num_nodes)
    : _my_rank(node_id), _num_nodes(num_nodes) {}

bool reservation_station_t::queue_command(command_ptr_t cmd) {
  std::unique_lock<std::mutex> lk(_m);
  const auto id = cmd->id;
  if (_last_cmd >= id) return false;  // commands must be queued in increasing id order
  if (cmd->get_root_node() != _my_rank) return false;
  bool ok = _queue_local(std::move(cmd));
  if (ok) _last_cmd = id;
  lk.unlock();
  _queued_hook(id);
  return ok;
}

bool reservation_station_t::_queue_local(command_ptr_t cmd) {
  if (cmd->is_delete()) {
    for (size_t i = 0; i < cmd->get_num_inputs(); ++i) {
      tid_t tid = cmd->get_input(i).tid;
      auto& s = _tensors[tid];
      if (s.is_created && s.num_to_read == 0 && !s.writing_tensor) {
        _remove_tensor(tid);
      } else {
        if (s.scheduled_for_deletion) return false;
        s.scheduled_for_deletion = true;
      }
      ++_num_to_delete;
    }
    return true;
  }
  int32_t missing = 0;
  for (size_t i = 0; i < cmd->get_num_inputs(); ++i) {
    const auto& in = cmd->get_input(i);
    if (in.node != _my_rank) return false;
    auto& s = _tensors[in.tid];
    if (s.scheduled_for_deletion) return false;  // read after a queued delete
    ++s.num_to_read;
    if (!s.is_created) {
      ++missing;
      _waiting_for.insert({in.tid, cmd->id});
    }
  }
  for (size_t i = 0; i < cmd->get_num_outputs(); ++i) {
    const auto& out = cmd->get_output(i);
    if (out.node != _my_rank) continue;
    auto& s = _tensors[out.tid];
    if (s.scheduled_for_deletion && s.is_created) return false;
    s.writing_tensor = true;
  }
  ++_num_local_to_retire;
  if (missing == 0) {
    _execute.emplace_back(std::move(cmd));
    _cv.notify_all();
  } else {
    const auto id = cmd->id;
    _local_commands[id] = {std::move(cmd), missing};
  }
  return true;
}

bool reservation_station_t::retire_command(command_ptr_t cmd) {
  std::unique_lock<std::mutex> lk(_m);
  const auto id = cmd->id;
  bool ok = _retire_local(std::move(cmd));
  lk.unlock();
  _retired_hook(id);
  return ok;
}

void reservation_station_t::_tensor_created(tid_t tid) {
  auto range = _waiting_for.equal_range(tid);
  for (auto it = range.first; it != range.second;) {
    auto jt = _local_commands.find(it->second);
    if (jt != _local_commands.end() && --jt->second.second == 0) {
      _schedule(std::move(jt->second.first));
      _local_commands.erase(jt);
    }
    it = _waiting_for.erase(it);
  }
}

bool reservation_station_t::_retire_local(command_ptr_t cmd) {
  if (cmd->is_delete()) {
    for (size_t i = 0; i < cmd->get_num_inputs(); ++i) _remove_tensor(cmd->get_input(i).tid);
    return true;
  }
  for (size_t i = 0; i < cmd->get_num_outputs(); ++i) {
    const auto& out = cmd->get_output(i);
    if (out.node != _my_rank) continue;
    auto& s = _tensors[out.tid];
    s.is_created = true;
    s.writing_tensor = false;
    const bool drop = s.num_to_read == 0 && s.scheduled_for_deletion;
    _tensor_created(out.tid);
    if (drop) _remove_tensor(out.tid);
  }
  for (size_t i = 0; i < cmd->get_num_inputs(); ++i) {
    const auto& in = cmd->get_input(i);
    if (in.node != _my_rank) continue;
    auto it = _tensors.find(in.tid);
    if (it == _tensors.end()) continue;
    auto& s = it->second;
    --s.num_to_read;
    if (s.num_to_read == 0 && !s.writing_tensor && s.scheduled_for_deletion) _remove_tensor(in.tid);
  }
  --_num_local_to_retire;
  if (_num_to_delete == 0 && _num_local_to_retire == 0) _retire_cv.notify_all();
  return true;
}

void reservation_station_t::register_tensor(tid_t tid) {
  std::lock_guard<std::mutex> lk(_m);
  auto& s = _tensors[tid];
  s.is_created = true;
  s.writing_tensor = false;
  _tensor_created(tid);
}

command_ptr_t reservation_station_t::_pop_locked() {
  if (_execute.empty()) return nullptr;
  size_t pick = _execute.size() - 1;  // LIFO
  if (_priority) {
    double best = _priority(*_execute[pick]);
    for (size_t i = _execute.size() - 1; i-- > 0;) {
      double v = _priority(*_execute[i]);
      if (v > best) { best = v; pick = i; }
    }
  }
  command_ptr_t c = std::move(_execute[pick]);
  _execute.erase(_execute.begin() + pick);
  return c;
}

command_ptr_t reservation_station_t::get_next_command() {
  std::unique_lock<std::mutex> lk(_m);
  _cv.wait(lk, [&] { return (!_execute.empty() && _is_executing) || _shutdown; });
  if (_shutdown) return nullptr;
  auto c = _pop_locked();
  lk.unlock();
  _scheduled_hook(c->id);
  return c;
}

command_ptr_t reservation_station_t::try_get_next_command() {
  std::unique_lock<std::mutex> lk(_m);
  if (_shutdown || _execute.empty()) return nullptr;
  auto c = _pop_locked();
  lk.unlock();
  _scheduled_hook(c->id);
  return c;
}

tid_t reservation_station_t::get_to_remove() {
  std::unique_lock<std::mutex> lk(_m);
  _deletion_cv.wait(lk, [&] { return !_to_delete.empty() || _shutdown; });
  if (_to_delete.empty()) return -1;
  tid_t t = _to_delete.back();
  _to_delete.pop_back();
  return t;
}

bool reservation_station_t::try_get_to_remove(tid_t* tid) {
  std::lock_guard<std::mutex> lk(_m);
  if (_to_delete.empty()) return false;
  *tid = _to_delete.back();
  _to_delete.pop_back();
  return true;
}

void reservation_station_t::retire_remove(tid_t) {
  std::lock_guard<std::mutex> lk(_m);
  if (_num_to_delete > 0) --_num_to_delete;
  if (_num_to_delete == 0 && _num_local_to_retire == 0) _retire_cv.notify_all();
}

void reservation_station_t::shutdown() {
  std::lock_guard<std::mutex> lk(_m);
  _shutdown = true;
  _cv.notify_all();
  _deletion_cv.notify_all();
  _retire_cv.notify_all();
}

void reservation_station_t::clear() {
  std::lock_guard<std::mutex> lk(_m);
  _last_cmd = -1;
  _execute.clear();
  _local_commands.clear();
  _waiting_for.clear();
  _tensors.clear();
  _to_delete.clear();
  _num_local_to_retire = 0;
  _num_to_delete = 0;
  _shutdown = false;
}

void reservation_station_t::wait_until_finished() {
  std::unique_lock<std::mutex> lk(_m);
  _retire_cv.wait(lk, [&] { return (_num_local_to_retire == 0 && _num_to_delete == 0) || _shutdown; });
}

void reservation_station_t::execute_scheduled_async() {
  std::lock_guard<std::mutex> lk(_m);
  _is_executing = true;
  _cv.notify_all();
}

void reservation_station_t::stop_executing() {
  std::lock_guard<std::mutex> lk(_m);
  _is_executing = false;
  _last_cmd = -1;
}

void reservation_station_t::set_priority(std::function<double(const command_t&)> prio) {
  std::lock_guard<std::mutex> lk(_m);
  _priority = std::move(prio);
}

void reservation_station_t::_schedule(command_ptr_t cmd) {
  _execute.emplace_back(std::move(cmd));
  _cv.notify_all();
}

void reservation_station_t::_remove_tensor(tid_t tid) {
  _to_delete.push_back(tid);
  _tensors.erase(tid);
  _deletion_cv.notify_all();
}

}  // namespace bbts
