// Single-GPU runtime around the block kernels: device-resident block storage,
// the per-op command runner (reference: src/commands/command_runner.cc:18-259
// with the local reduce of src/operations/local_reduce_op.cc:23-91) and the
// grouped DAG executor (one grouped tensor-core launch + one grouped streaming
// launch per wave, captured into a CUDA graph).
#pragma once
#include <cuda_runtime.h>
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

// One block: a host-side header in the reference layout whose payload slot
// points at HBM.
struct block_t {
  std::unique_ptr<char[]> header;  // sizeof(tensor_meta_t) bytes
  void* payload = nullptr;
  size_t bytes = 0;
  bool owned = true;               // payload allocated by storage (freed by it)
  tensor_t* tensor() const { return (tensor_t*)header.get(); }
};

// tid -> block. Payload allocations are stream-ordered on the runtime stream.
// Payloads come from a memory pool the storage owns, stream-ordered on the
// stream each call names (the runtime stream by default). The pool keeps freed
// memory for reuse instead of returning it to the driver at every
// synchronisation, so a block freed and re-created costs no new mapping.
class block_storage_t {
 public:
  block_storage_t(tensor_factory_ptr_t tf, cudaStream_t st);
  ~block_storage_t();
  tensor_t* create(tid_t tid, const tensor_meta_t& meta, cudaStream_t st = nullptr);  // allocates the payload
  tensor_t* create_view(tid_t tid, const tensor_meta_t& meta, void* payload, size_t bytes);
  tensor_t* get(tid_t tid);
  block_t* block(tid_t tid);
  bool remove(tid_t tid, cudaStream_t st = nullptr);
  bool assign_tid(tid_t from, tid_t to);
  size_t size() const { return _blocks.size(); }
  std::vector<tid_t> tids() const;

 private:
  tensor_factory_ptr_t _tf;
  cudaStream_t _st;
  cudaMemPool_t _pool = nullptr;
  std::mutex _m;
  std::unordered_map<tid_t, block_t> _blocks;
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
void dag_launch(dag_t* d, cudaStream_t st);
void dag_destroy(dag_t* d);
struct dag_stats_t {
  int waves, tc_launches, stream_launches, opaque_launches, nodes;
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
