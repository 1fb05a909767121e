// Single-GPU runtime around the block kernels: device-resident block storage,
// the per-op command runner (reference: src/commands/command_runner.cc:18-259
// with the local reduce of src/operations/local_reduce_op.cc:23-91) and the
// grouped DAG executor (one grouped tensor-core launch + one grouped streaming
// launch per wave, captured into a CUDA graph).
#pragma once
#include <cuda_runtime.h>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>
#include "bbts_b200.h"
#include "command.h"
#include "reservation_station.h"
#include "ud_function.h"

namespace bbts {

// Completion marker of stream work, shared by the blocks that wait on it.
using event_ptr = std::shared_ptr<CUevent_st>;

// One block: a host-side header in the reference layout whose payload slot
// points at HBM while the block is resident. A spilled block keeps its header;
// its bytes live in pinned host memory (host tier) or in the spill file (file
// tier) until a command needs it again.
struct block_t {
  std::unique_ptr<char[]> header;  // sizeof(tensor_meta_t) bytes
  void* payload = nullptr;         // HBM; null while spilled
  size_t bytes = 0;
  bool owned = true;               // payload allocated by storage (freed by it)
  bool resident = true;
  // spill copies; blocks are written once by the command that creates them,
  // so a copy stays valid across reloads until a caller is handed the
  // payload pointer (it may write through it)
  void* host = nullptr;
  bool host_valid = false;
  long long file_off = -1;
  bool file_valid = false;
  bool caller_may_write = false;   // last writer may be work the caller queued on the runtime stream
  int pins = 0;                    // commands (or compiled DAGs) holding the payload
  std::vector<std::pair<cudaStream_t, event_ptr>> uses;  // last use per stream while resident
  event_ptr copied;                // the D2H that filled the host copy
  event_ptr host_read;             // the last H2D that read the host copy
  event_ptr loaded;                // the reload that made the payload resident again
  cudaStream_t loaded_st = nullptr;
  int readers_left = -1;           // commands still to read it in the running list (-1: unknown)
  bool in_lru = false;
  int lru_list = 0;                // 0: blocks still to be read, 1: blocks no queued command reads
  std::list<tid_t>::iterator lru_it;
  tensor_t* tensor() const { return (tensor_t*)header.get(); }
};

// Spill counters (bytes and counts since the budget was set).
struct spill_stats_t {
  unsigned long long evictions = 0, reloads = 0, d2h_bytes = 0, h2d_bytes = 0;
  unsigned long long file_write_bytes = 0, file_read_bytes = 0, clean_evictions = 0;
  unsigned long long resident_bytes = 0, peak_resident_bytes = 0, host_bytes = 0;
};

// tid -> block. Payloads come from a memory pool the storage owns,
// stream-ordered on the stream each call names (the runtime stream by
// default). The pool keeps freed memory for reuse instead of returning it to
// the driver at every synchronisation, so a block freed and re-created costs
// no new mapping.
//
// With a device budget (set_budget), resident payload bytes stay within it:
// making room evicts the least recently used unpinned blocks, copying each
// to pinned host memory while the host budget lasts and to the spill file
// after that, and a spilled block is copied back when a command acquires it
// (reference: nvme_storage_t, src/storage/nvme_storage.h:26-467 and
// nvme_storage.cc:355-637 -- LRU of unreferenced tensors, eviction to a file
// by pwrite, reload by pread, "Can not process this." when one request alone
// exceeds the budget). Device-to-host spill copies run on a copy stream that
// waits for the block's last uses; the streams that allocate next wait for
// those frees.
class block_storage_t {
 public:
  block_storage_t(tensor_factory_ptr_t tf, cudaStream_t st);
  ~block_storage_t();
  tensor_t* create(tid_t tid, const tensor_meta_t& meta, cudaStream_t st = nullptr);  // allocates the payload
  tensor_t* create_view(tid_t tid, const tensor_meta_t& meta, void* payload, size_t bytes);
  tensor_t* get(tid_t tid);        // header only; the payload slot is null while spilled
  block_t* block(tid_t tid);
  bool remove(tid_t tid, cudaStream_t st = nullptr);
  bool assign_tid(tid_t from, tid_t to);
  size_t size() const { return _blocks.size(); }
  std::vector<tid_t> tids() const;

  // ---- spill tier
  // device_bytes 0 = no budget (nothing is ever spilled). host_bytes: pinned
  // host memory the spill may hold; past it blocks go to `file` (none = error).
  void set_budget(size_t device_bytes, size_t host_bytes, const std::string& file);
  size_t budget() const { return _budget; }
  // Commands: blocks acquired or created between begin_command and
  // end_command stay resident until end_command records their use on `st`.
  void begin_command();
  tensor_t* acquire(tid_t tid, cudaStream_t st);  // resident + held for the current command
  void end_command(cudaStream_t st);
  // Resident payload for a caller outside a command (reads, and writes when
  // will_write, queued on the runtime stream); valid until the next call that
  // may evict.
  void* caller_payload(tid_t tid, size_t* bytes, bool will_write);
  // Eviction hint from the per-op runner: how many queued commands still read
  // `tid` (0 = none: it is evicted before blocks that will be read again).
  void set_readers_left(tid_t tid, int n);
  // Compiled DAGs hold every existing block resident until released.
  std::vector<tid_t> hold_all();
  void release(const std::vector<tid_t>& tids);
  spill_stats_t stats() const;

 private:
  void _lru_remove(block_t& b);
  void _lru_touch(tid_t tid, block_t& b);
  void _make_room(size_t need, cudaStream_t st);
  void _evict(tid_t tid, block_t& b);
  void _reload(block_t& b, cudaStream_t st);
  void _pin(tid_t tid, block_t& b);
  void _unpin(tid_t tid, block_t& b);
  void _drop_copies(block_t& b);
  void _free_payload(block_t& b, cudaStream_t st);
  void* _host_alloc(size_t bytes, event_ptr* last_read);
  void _file_io(block_t& b, bool write, cudaStream_t st);
  event_ptr _record(cudaStream_t st);

  tensor_factory_ptr_t _tf;
  cudaStream_t _st;
  cudaMemPool_t _pool = nullptr;
  std::recursive_mutex _m;
  std::unordered_map<tid_t, block_t> _blocks;
  // spill state
  size_t _budget = 0, _host_budget = 0;
  std::string _file;
  int _fd = -1;
  long long _file_end = 0;
  cudaStream_t _out_st = nullptr;  // device-to-host spill copies and the frees after them
  event_ptr _freed;                // after the latest eviction's free
  // resident unpinned owned blocks, front = most recently used; eviction takes
  // the blocks no queued command reads (results, list 1) before the others
  std::list<tid_t> _lru[2];
  std::vector<tid_t> _scope;       // blocks held by the command being issued
  bool _in_command = false;
  std::multimap<size_t, std::pair<void*, event_ptr>> _host_cache;  // pinned buffers free for reuse
  std::vector<void*> _host_all;
  void* _stage = nullptr;          // pinned staging for the file tier
  spill_stats_t _stats;
};

// Op features for the learned cost model: the 12 MLP inputs, plus the ud's
// own get_complexity_hint (the heuristic cost), which is not an MLP input.
struct op_features_t {
  float f[12];
  double hint = 0.0;
};

// A compiled DAG: every launch of a whole command list, captured in a CUDA graph.
struct dag_t;

enum sched_policy_t : int {
  SCHED_HEURISTIC = 0,  // reservation-station LIFO order + complexity hints
  SCHED_LEARNED = 1,    // critical-path / LPT order from the MLP's predicted latencies
};

class runtime_t {
 public:
  runtime_t();
  ~runtime_t();

  tensor_factory_ptr_t tf;
  udf_manager_ptr udm;
  cudaStream_t stream = nullptr;
  std::unique_ptr<block_storage_t> storage;
  std::vector<command_ptr_t> commands;  // the queued command list (compiled DAG)

  // predicted latency (us) for a node / a batch of nodes, installed by the learned cost model
  std::function<double(const op_features_t&)> predictor;
  std::function<std::vector<double>(const std::vector<op_features_t>&)> batch_predictor;
  // predicted time of a grouped tensor-core launch per tile (dag_build with
  // tile_n = -2), from tile_features rows; installed from a trained MLP
  std::function<std::vector<double>(const std::vector<op_features_t>&)> tile_predictor;
  // kernel of a compiled DAG's grouped streaming launches (BBX_STREAM_KERNEL_*)
  int dag_stream_kernel = 0;

  // Worker streams of the per-op path: the reference pulls ready commands from
  // the reservation station with num_threads workers (src/server/node.cc:67-69);
  // here each worker is a CUDA stream and a command waits only on the events
  // of the commands that produced its inputs. 1 = the plain path (one stream,
  // one launch after another).
  int workers = 1;
  std::vector<cudaStream_t> worker_streams;

  // Per-op execution of `commands` through the reservation station with
  // `workers` streams. Heuristic: LIFO pop, round-robin streams. Learned:
  // critical-path pop by predicted latency, each command on the stream with
  // the earliest predicted finish. With record != null (always one stream)
  // the launches of each command are bracketed by CUDA events and their
  // (features, latency) pairs appended.
  void run_per_op(int policy, std::vector<std::pair<op_features_t, float>>* record);

  op_features_t features(const command_t& cmd, size_t* hint_out);
};

// The ud kinds the executor launches natively (grouped) or through the impl's fn.
enum node_kind_t { NK_TC = 0, NK_SIMT = 1, NK_SUM = 2, NK_UNARY = 3, NK_BINARY = 4, NK_CONTRACT = 5, NK_OPAQUE = 6 };
node_kind_t classify(const ud_impl_t* impl, bool is_reduce);
op_features_t features_of(const tensor_factory_t& tf, const command_t& cmd, ud_impl_t* impl,
                          std::vector<tensor_meta_t> in_metas, size_t* hint_out);
int elem_of(const tensor_factory_t& tf, tfid_t id);
void execute_command(runtime_t& rt, command_t& cmd, cudaStream_t st);

dag_t* dag_build(runtime_t* rt, int policy, int tile_n);
// Recording of the autotuner's timings as learned-tile training samples
// (features of a group run with one tile, us per launch); on clears them.
void tile_record(bool on);
std::vector<std::pair<op_features_t, float>> tile_samples();
void dag_launch(dag_t* d, cudaStream_t st);
void dag_destroy(dag_t* d);
struct dag_stats_t {
  int waves, tc_launches, stream_launches, opaque_launches, nodes;
  int register_waves;  // waves whose streaming launches run the register kernel (per-wave choice)
  double flops, bytes;
  size_t arena_bytes;
};
dag_stats_t dag_stats(const dag_t* d);
// kind: 0 contraction input gathers, 1 grouped streaming ops, 2 ops called
// through their impls, 3 grouped tcgen05 GEMM, 4 contraction output gathers
struct dag_group_profile_t {
  int kind, wave;
  float ms;
  double flops, bytes;
};
std::vector<dag_group_profile_t> dag_profile(dag_t* d, cudaStream_t st);
int dag_num_groups(const dag_t* d);

}  // namespace bbts
