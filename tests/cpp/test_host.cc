// Host-side tests of the runtime's C++ layer, no GPU needed: tensor factory,
// ud registry with real type matching, command records, reservation station.
// Modelled on the reference's tests/test_builtin_dense.cc,
// tests/test_builtin_ud.cc, tests/test_parsed_command.cc and
// tests/test_reservation_station.cc (FewLocalCommands*, the deferred-delete
// scenarios). Built and run by tests/test_host_cpp.py.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <cstdio>
#include <cstdlib>
#include <set>
#include <thread>
#include <sstream>
#include <tuple>
#include <vector>
#include "bbts_b200.h"
#include "command.h"
#include "compiler.h"
#include "contraction.h"
#include "reservation_station.h"
#include "tensor.h"
#include "tile_order.h"
#include "ud_function.h"

using namespace bbts;

static int g_fail = 0;
#define EXPECT(c)                                                              \
  do {                                                                         \
    if (!(c)) {                                                                \
      std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c);                 \
      ++g_fail;                                                                \
    }                                                                          \
  } while (0)

struct fake_impl : ud_impl_t {
  fake_impl(const char* ud, const char* name, std::vector<std::string> in, std::vector<std::string> out, bool gpu) {
    ud_name = ud;
    impl_name = name;
    inputTypes = std::move(in);
    outputTypes = std::move(out);
    is_gpu = gpu;
    fn = [](const tensor_params_t&, const tensor_args_t&, tensor_args_t&) {};
  }
  size_t get_complexity_hint(const tensor_params_t&, const meta_args_t&) override { return 1; }
  void get_out_meta(const tensor_params_t&, const meta_args_t&, meta_args_t&) const override {}
};

static void test_dense_format() {
  tensor_factory_t tf;
  tfid_t id = tf.get_tensor_ftm("dense");
  EXPECT(id == 0);
  EXPECT(tf.get_tensor_ftm("nope") == -1);
  dense_tensor_meta_t m(id, 100, 200);
  // builtin_formats.cc:18-21: header + rows*cols*4
  EXPECT(tf.get_tensor_size(m) == sizeof(tensor_meta_t) + 100 * 200 * 4);
  EXPECT(sizeof(tensor_meta_t) == 260);
  // reference layout on the host: payload right after the header
  std::vector<char> mem(tf.get_tensor_size(m));
  auto& t = tf.init_tensor((tensor_t*)mem.data(), m).as<dense_tensor_t>();
  EXPECT((char*)t.data() == mem.data() + sizeof(tensor_meta_t));
  EXPECT(t.meta().m().num_rows == 100 && t.meta().m().num_cols == 200);
  // payload slot: tagged by this library; an untagged header (a tensor the
  // reference initialised, zeroed or garbage blob) has its payload inline
  {
    std::vector<char> raw(sizeof(tensor_meta_t) + 16, 0);
    tensor_t* u = (tensor_t*)raw.data();
    u->_meta.fmt_id = id;
    EXPECT(!u->_meta.payload_tagged() && u->_meta.payload() == nullptr);
    EXPECT((char*)u->payload() == raw.data() + sizeof(tensor_meta_t));
    for (size_t i = 0; i < tensor_meta_t::MAX_META_SIZE; ++i) u->_meta._blob[i] = (char)(i * 37 + 11);
    EXPECT(!u->_meta.payload_tagged() && (char*)u->payload() == raw.data() + sizeof(tensor_meta_t));
    int dev_word = 0;
    u->_meta.set_payload(&dev_word);  // a device address placed by this library
    EXPECT(u->_meta.payload_tagged() && u->payload() == &dev_word);
    u->_meta.set_payload(nullptr);    // a block with no resident payload (zero bytes, or spilled)
    EXPECT(u->_meta.payload_tagged() && u->payload() == nullptr);
    tensor_meta_t copy = u->_meta;    // the tag travels with the meta
    copy.set_payload(&dev_word);
    EXPECT(copy.payload() == &dev_word);
    copy._blob[tensor_meta_t::PAYLOAD_SLOT] ^= 1;  // a slot changed behind the tag is not trusted
    EXPECT(!copy.payload_tagged());
  }
  // register_fmt returns the new id, and the first one on re-registration
  tfid_t f2 = tf.register_fmt("ffnn_dense", ffnn_dense_creation_fs());
  EXPECT(f2 == tf.get_tensor_ftm("ffnn_dense"));
  EXPECT(tf.register_fmt("ffnn_dense", ffnn_dense_creation_fs()) == f2);
  ffnn_dense_meta_t fm(f2, true, 10, 20);
  EXPECT(tf.get_tensor_size(fm) == sizeof(tensor_meta_t) + (10 * 20 + 20) * 4);
  tfid_t bf = tf.get_tensor_ftm("dense_bf16");
  dense_tensor_meta_t mb(bf, 64, 32);
  EXPECT(tf.get_payload_size(mb) == 64 * 32 * 2);
}

static void test_matcher_types() {
  auto tf = std::make_shared<tensor_factory_t>();
  udf_manager_t udm(tf);
  auto f = std::make_unique<ud_func_t>();
  f->ud_name = "matrix_add";
  f->is_ass = f->is_com = true;
  f->num_in = 2;
  f->num_out = 1;
  EXPECT(udm.register_udf(std::move(f)) == 0);
  auto dup = std::make_unique<ud_func_t>();
  dup->ud_name = "matrix_add";
  EXPECT(udm.register_udf(std::move(dup)) == -1);
  auto a = udm.register_udf_impl(std::make_unique<fake_impl>("matrix_add", "cpu_dense", std::vector<std::string>{"dense", "dense"}, std::vector<std::string>{"dense"}, false));
  auto b = udm.register_udf_impl(std::make_unique<fake_impl>("matrix_add", "gpu_bf16", std::vector<std::string>{"dense_bf16", "dense_bf16"}, std::vector<std::string>{"dense_bf16"}, true));
  auto c = udm.register_udf_impl(std::make_unique<fake_impl>("matrix_add", "gpu_dense", std::vector<std::string>{"dense", "dense"}, std::vector<std::string>{"dense"}, true));
  EXPECT(a.impl_id == 0 && b.impl_id == 1 && c.impl_id == 2);
  // wrong arity is refused
  auto bad = udm.register_udf_impl(std::make_unique<fake_impl>("matrix_add", "bad", std::vector<std::string>{"dense"}, std::vector<std::string>{"dense"}, true));
  EXPECT(bad.ud_id == -1);
  auto m = udm.get_matcher_for("matrix_add");
  EXPECT(m != nullptr);
  // the reference's matcher returns the first GPU impl regardless of types; here types decide
  ud_impl_t* g = m->findMatch({"dense", "dense"}, {"dense"}, true);
  EXPECT(g && g->impl_name == "gpu_dense");
  ud_impl_t* h = m->findMatch({"dense_bf16", "dense_bf16"}, {"dense_bf16"}, true);
  EXPECT(h && h->impl_name == "gpu_bf16");
  EXPECT(m->findMatch({"dense", "dense_bf16"}, {"dense"}, true) == nullptr);
  EXPECT(m->findMatch({"dense", "dense"}, {"dense"}, false)->impl_name == "cpu_dense");
  EXPECT(udm.get_matcher_for("nope") == nullptr);
  EXPECT(udm.get_matcher_for("matrix_add", true, true) != nullptr);
  EXPECT(udm.get_fn_impl({0, 2})->impl_name == "gpu_dense");
  EXPECT(udm.get_fn_impl({0, 9}) == nullptr);
}

static void test_command_layout() {
  std::vector<command_param_t> p(3);
  p[0].i = 7;
  p[1].f = 2.5f;
  p[2].b = true;
  auto c = command_t::create_apply(5, {1, 2}, true, p, {{10, 0}, {11, 0}}, {{12, 0}});
  EXPECT(c->id == 5 && c->is_apply() && c->get_num_inputs() == 2 && c->get_num_outputs() == 1);
  EXPECT(c->get_input(1).tid == 11 && c->get_output(0).tid == 12);
  EXPECT(c->get_parameters()[1].f == 2.5f && c->get_parameters()[0].i == 7);
  auto d = c->clone();  // flat, memcpy-able (command.h:459-542)
  EXPECT(d->num_bytes() == c->num_bytes() && d->get_input(0).tid == 10 && d->get_parameters()[2].b);
  auto r = command_t::create_reduce(6, {0, 0}, true, {}, {{1, 0}, {2, 0}, {3, 0}}, {4, 0});
  EXPECT(r->is_reduce() && r->is_local_reduce(0) && !r->is_local_reduce(1) && r->get_num_inputs() == 3);
  auto del = command_t::create_delete(7, {{1, 0}, {2, 0}});
  EXPECT(del->is_delete() && del->get_num_outputs() == 0);
  auto mv = command_t::create_move(8, {3, 0}, {3, 1});
  EXPECT(mv->is_move() && mv->get_nodes().size() == 2);
}

// APPLY a, b -> c ; APPLY c -> d ; DELETE a, b, c : readiness, LIFO order and deferred deletes
static void test_reservation_station_basic() {
  reservation_station_t rs(0, 1);
  std::vector<command_id_t> scheduled, retired;
  rs.add_scheduled_hook([&](command_id_t id) { scheduled.push_back(id); });
  rs.add_retired_hook([&](command_id_t id) { retired.push_back(id); });
  rs.register_tensor(0);
  rs.register_tensor(1);
  EXPECT(rs.queue_command(command_t::create_apply(0, {0, 0}, true, {}, {{0, 0}, {1, 0}}, {{2, 0}})));
  EXPECT(rs.queue_command(command_t::create_apply(1, {0, 0}, true, {}, {{2, 0}}, {{3, 0}})));
  EXPECT(rs.queue_command(command_t::create_delete(2, {{0, 0}, {1, 0}, {2, 0}})));
  EXPECT(!rs.queue_command(command_t::create_apply(1, {0, 0}, true, {}, {{0, 0}}, {{9, 0}})));  // id order
  rs.execute_scheduled_async();
  auto c0 = rs.try_get_next_command();
  EXPECT(c0 && c0->id == 0);
  EXPECT(rs.try_get_next_command() == nullptr);  // command 1 waits for tensor 2
  tid_t t;
  EXPECT(!rs.try_get_to_remove(&t));             // a, b still have a reader
  rs.retire_command(std::move(c0));
  std::set<tid_t> removed;
  while (rs.try_get_to_remove(&t)) { removed.insert(t); rs.retire_remove(t); }
  EXPECT(removed == std::set<tid_t>({0, 1}));   // deleted as soon as their reader retired
  auto c1 = rs.try_get_next_command();
  EXPECT(c1 && c1->id == 1);
  rs.retire_command(std::move(c1));
  while (rs.try_get_to_remove(&t)) { removed.insert(t); rs.retire_remove(t); }
  EXPECT(removed.count(2) == 1);
  EXPECT(rs.num_to_retire() == 0);
  rs.wait_until_finished();
  EXPECT(scheduled == std::vector<command_id_t>({0, 1}));
  EXPECT(retired == std::vector<command_id_t>({0, 1}));
}

// Ready commands pop LIFO (reservation_station.cc:213-214), or by priority when installed.
static void test_reservation_station_order() {
  for (int prio = 0; prio < 2; ++prio) {
    reservation_station_t rs(0, 1);
    rs.register_tensor(0);
    for (int i = 0; i < 5; ++i)
      rs.queue_command(command_t::create_apply(i, {0, 0}, true, {}, {{0, 0}}, {{100 + i, 0}}));
    if (prio) rs.set_priority([](const command_t& c) { return (double)((c.id * 3) % 5); });
    rs.execute_scheduled_async();
    std::vector<command_id_t> order;
    while (auto c = rs.try_get_next_command()) {
      order.push_back(c->id);
      rs.retire_command(std::move(c));
    }
    if (!prio) EXPECT(order == std::vector<command_id_t>({4, 3, 2, 1, 0}));
    else EXPECT(order == std::vector<command_id_t>({3, 1, 4, 2, 0}));  // priorities 4,3,2,1,0
  }
}

// A delete queued before the readers of a not-yet-created tensor waits for them;
// reading a tensor after its delete was queued is refused.
static void test_reservation_station_delete_rules() {
  reservation_station_t rs(0, 1);
  rs.register_tensor(0);
  EXPECT(rs.queue_command(command_t::create_apply(0, {0, 0}, true, {}, {{0, 0}}, {{1, 0}})));
  EXPECT(rs.queue_command(command_t::create_delete(1, {{1, 0}})));
  EXPECT(!rs.queue_command(command_t::create_apply(2, {0, 0}, true, {}, {{1, 0}}, {{2, 0}})));
  rs.execute_scheduled_async();
  auto c = rs.try_get_next_command();
  tid_t t;
  EXPECT(!rs.try_get_to_remove(&t));
  rs.retire_command(std::move(c));
  EXPECT(rs.try_get_to_remove(&t) && t == 1);  // created with no readers and scheduled: dropped
  rs.retire_remove(t);
}

// A diamond of 100 commands run by 4 worker threads; every tensor is deleted
// exactly once and every command retires (the shape of the reference's
// threaded reservation-station scenarios).
static void test_reservation_station_threads() {
  reservation_station_t rs(0, 1);
  rs.register_tensor(0);
  const int N = 100;
  int id = 0;
  for (int i = 0; i < N; ++i)
    rs.queue_command(command_t::create_apply(id++, {0, 0}, true, {}, {{0, 0}}, {{1 + i, 0}}));
  std::vector<command_t::tid_node_id_t> ins;
  for (int i = 0; i < N; ++i) ins.push_back({1 + i, 0});
  rs.queue_command(command_t::create_reduce(id++, {0, 0}, true, {}, ins, {1000, 0}));
  rs.queue_command(command_t::create_delete(id++, ins));
  std::atomic<int> executed{0};
  std::mutex rm_mu;
  std::set<tid_t> removed;
  rs.execute_scheduled_async();
  std::vector<std::thread> th;
  for (int w = 0; w < 4; ++w)
    th.emplace_back([&] {
      while (auto c = rs.get_next_command()) {
        ++executed;
        rs.retire_command(std::move(c));
      }
    });
  std::thread deleter([&] {
    tid_t t;
    while ((t = rs.get_to_remove()) != -1) {
      { std::lock_guard<std::mutex> lk(rm_mu); removed.insert(t); }
      rs.retire_remove(t);
    }
  });
  rs.wait_until_finished();
  rs.shutdown();
  for (auto& x : th) x.join();
  deleter.join();
  EXPECT(executed == N + 1);
  EXPECT((int)removed.size() == N);
}

// .sbbts text round trip + single-node compilation (command_compiler.h:977-1027)
static void test_sbbts_compile() {
  const char* text =
      "2\n"
      "0 matrix_mult 2 dense dense 1 dense \n"
      "1 matrix_add 2 dense dense 1 dense \n"
      "4\n"
      "0 APPLY 2 0 1 1 2 2 int 0 int 0 \n"
      "0 APPLY 2 0 1 1 3 0 \n"
      "1 REDUCE 2 2 3 1 4 1 float 0.5 \n"
      "0 DELETE 2 2 3 0 0 \n";
  std::istringstream in(text);
  compile_source_file_t src;
  src.read(in);
  EXPECT(src.function_specs.size() == 2 && src.commands.size() == 4);
  EXPECT(src.commands[2].type == abstract_command_type_t::REDUCE && src.commands[2].params[0].f == 0.5f);
  std::ostringstream out;
  src.write(out);
  std::istringstream in2(out.str());
  compile_source_file_t again;
  again.read(in2);
  EXPECT(again.commands.size() == 4 && again.commands[1].output_tids[0] == 3);

  auto tf = std::make_shared<tensor_factory_t>();
  udf_manager_t udm(tf);
  for (auto [name, ass, com] : {std::tuple<const char*, bool, bool>{"matrix_mult", true, false},
                                std::tuple<const char*, bool, bool>{"matrix_add", true, true}}) {
    auto f = std::make_unique<ud_func_t>();
    f->ud_name = name; f->is_ass = ass; f->is_com = com; f->num_in = 2; f->num_out = 1;
    udm.register_udf(std::move(f));
    udm.register_udf_impl(std::make_unique<fake_impl>(name, "gpu", std::vector<std::string>{"dense", "dense"}, std::vector<std::string>{"dense"}, true));
  }
  auto cmds = compile_single_node(src, udm, 10);
  EXPECT(cmds.size() == 4);
  EXPECT(cmds[0]->id == 10 && cmds[0]->is_apply() && cmds[0]->get_root_node() == 0);
  EXPECT(cmds[2]->is_reduce() && cmds[2]->get_num_inputs() == 2 && cmds[2]->get_output(0).tid == 4);
  EXPECT(cmds[3]->is_delete() && cmds[3]->get_num_inputs() == 2);
  // a REDUCE over a non-commutative ud is refused
  std::istringstream bad("1\n0 matrix_mult 2 dense dense 1 dense \n1\n0 REDUCE 2 0 1 1 2 0 \n");
  compile_source_file_t sbad;
  sbad.read(bad);
  bool threw = false;
  try { compile_single_node(sbad, udm, 0); } catch (const std::exception&) { threw = true; }
  EXPECT(threw);
}

// .bbts binary round trip (parsed_command.h:194-383) and the loader
static void test_bbts_roundtrip() {
  parsed_command_list_t list;
  parsed_command_t a;
  a.type = parsed_command_t::op_type_t::APPLY;
  a.def = {"matrix_add", {"dense", "dense"}, {"dense"}, true};
  a.inputs = {{0, 0}, {1, 0}};
  a.outputs = {{2, 0}};
  command_param_t p;
  p.f = 1.5f;
  a.parameters = {p};
  parsed_command_t d;
  d.type = parsed_command_t::op_type_t::DELETE;
  d.inputs = {{0, 0}};
  list.commands = {a, d};
  const char* path = "/tmp/bbx_test_roundtrip.bbts";
  EXPECT(list.serialize(path));
  parsed_command_list_t back;
  EXPECT(back.deserialize(path));
  EXPECT(back.commands.size() == 2);
  EXPECT(back.commands[0].def.ud_name == "matrix_add" && back.commands[0].def.is_gpu);
  EXPECT(back.commands[0].inputs[1].first == 1 && back.commands[0].outputs[0].first == 2);
  EXPECT(back.commands[0].parameters[0].f == 1.5f);
  // on disk each (tid, node) pair is stored node first (std::tuple layout)
  FILE* f = std::fopen(path, "rb");
  std::vector<unsigned char> raw(4096);
  size_t n = std::fread(raw.data(), 1, raw.size(), f);
  std::fclose(f);
  EXPECT(n > 8);
  auto tf = std::make_shared<tensor_factory_t>();
  udf_manager_t udm(tf);
  auto fn = std::make_unique<ud_func_t>();
  fn->ud_name = "matrix_add"; fn->is_ass = fn->is_com = true; fn->num_in = 2; fn->num_out = 1;
  udm.register_udf(std::move(fn));
  udm.register_udf_impl(std::make_unique<fake_impl>("matrix_add", "gpu", std::vector<std::string>{"dense", "dense"}, std::vector<std::string>{"dense"}, true));
  auto cmds = load_parsed(back, udm, 0);
  EXPECT(cmds.size() == 2 && cmds[0]->is_apply() && cmds[1]->is_delete());
  std::remove(path);
}

// The bf16 contraction lowering's GEMM orientation: the longer of the lhs-only
// (nm) and rhs-only (nn) output extents becomes M. With nm > nn the GEMM is
// A = Lc, B = Rc, column-major C; otherwise A = Rc, B = Lc, row-major C. Both
// keep the staging layouts, pitches and per-batch offsets.
static void test_contraction_orientation() {
  char* lc = (char*)0x100000;
  char* rc = (char*)0x200000;
  char* ct = (char*)0x400000;
  {  // 'ijk,kl->ijl': i, j lhs-only (nm = 960), l rhs-only (nn = 32), k summed
    const long long dl[3] = {40, 24, 16}, dr[2] = {16, 32};
    const int ml[3] = {0, 1, 2}, mr[2] = {2, 3}, mo[3] = {0, 1, 3};
    bbx::ContractionLowering L;
    EXPECT(bbx::lower_contraction(3, dl, ml, 2, dr, mr, 3, mo, true, &L) == 0);
    EXPECT(L.nm == 960 && L.nn == 32 && L.kdim == 16 && L.nb == 1);
    EXPECT(L.lc_mn && !L.rc_mn && L.direct);
    const bbx::ContractionGemm g = bbx::contraction_gemm(L, lc, rc, ct, 0);
    EXPECT(g.m == 960 && g.n == 32 && g.k == 16);
    EXPECT(g.flags == BBX_EPI_C_COLMAJOR && g.ldc == 960 && g.c == ct);
    EXPECT(g.a == lc && g.trans_a == 1 && g.lda == L.pm);  // Lc[k][m]
    EXPECT(g.b == rc && g.trans_b == 1 && g.ldb == L.pk);  // Rc[n][k]
  }
  {  // batched 'ikb,klb->ilb' (b = 3): nm = 40 > nn = 32, offsets of batch 2
    const long long dl[3] = {40, 16, 3}, dr[3] = {16, 32, 3};
    const int ml[3] = {0, 2, 4}, mr[3] = {2, 3, 4}, mo[3] = {0, 3, 4};
    bbx::ContractionLowering L;
    EXPECT(bbx::lower_contraction(3, dl, ml, 3, dr, mr, 3, mo, true, &L) == 0);
    EXPECT(L.nb == 3 && L.nm == 40 && L.nn == 32);
    const bbx::ContractionGemm g = bbx::contraction_gemm(L, lc, rc, ct, 2);
    EXPECT(g.flags == BBX_EPI_C_COLMAJOR && g.m == 40 && g.n == 32);
    EXPECT(g.a == lc + 2 * 2 * L.kdim * L.pm);   // bf16 Lc[b][k][m]
    EXPECT(g.b == rc + 2 * 2 * L.nn * L.pk);     // bf16 Rc[b][n][k]
    EXPECT(g.c == ct + 4 * 2 * L.nn * L.nm);     // f32 Ct[b][n][m]
  }
  {  // 'ik,kl->il' with the rhs side longer (nm = 16 < nn = 64): row-major C
    const long long dl[2] = {16, 8}, dr[2] = {8, 64};
    const int ml[2] = {0, 2}, mr[2] = {2, 3}, mo[2] = {0, 3};
    bbx::ContractionLowering L;
    EXPECT(bbx::lower_contraction(2, dl, ml, 2, dr, mr, 2, mo, true, &L) == 0);
    const bbx::ContractionGemm g = bbx::contraction_gemm(L, lc, rc, ct, 0);
    EXPECT(g.m == 64 && g.n == 16 && g.k == 8 && g.flags == 0 && g.ldc == 16);
    EXPECT(g.a == rc && g.trans_a == 0 && g.lda == L.pk);  // Rc[n][k]
    EXPECT(g.b == lc && g.trans_b == 0 && g.ldb == L.pm);  // Lc[k][m]
  }
}

// The grouped tcgen05 launches' tile order (csrc/tile_order.h): the snake
// rounds of a persistent grid over a group's tile list, and the bands of
// tile-rows inside a problem, each visit every tile exactly once.
static void test_tile_order() {
  unsigned seed = 12345;
  auto rnd = [&](int lo, int hi) {
    seed = seed * 1103515245u + 12345u;
    return lo + (int)((seed >> 8) % (unsigned)(hi - lo + 1));
  };
  for (int trial = 0; trial < 300; ++trial) {
    const int grid = trial < 4 ? (trial == 0 ? 1 : 148) : rnd(1, 160);
    const int total = trial == 2 ? grid : (trial == 3 ? 3 * grid : rnd(1, 5000));
    std::vector<int> seen(total, 0);
    bool in_range = true;
    for (int b = 0; b < grid; ++b) {
      int prev = -1;
      for (int t0 = b, r = 0; t0 < total; t0 += grid, ++r) {
        const int t = bbx::snake_tile_of(t0, r, total, b, grid);
        if (t < 0 || t >= total) { in_range = false; continue; }
        ++seen[t];
        EXPECT(t / grid == r);  // round r's tiles stay in round r
        EXPECT(t > prev);
        prev = t;
      }
    }
    EXPECT(in_range);
    EXPECT(std::all_of(seen.begin(), seen.end(), [](int c) { return c == 1; }));
  }
  for (int tiles_m = 1; tiles_m <= 40; tiles_m += 3)
    for (int tiles_n = 1; tiles_n <= 9; ++tiles_n) {
      std::vector<int> seen(tiles_m * tiles_n, 0);
      for (int lt = 0; lt < tiles_m * tiles_n; ++lt) {
        int tm = -1, tn = -1;
        bbx::band_tile(lt, tiles_m, tiles_n, tm, tn);
        EXPECT(tm >= 0 && tm < tiles_m && tn >= 0 && tn < tiles_n);
        if (tm >= 0 && tm < tiles_m && tn >= 0 && tn < tiles_n) ++seen[tm * tiles_n + tn];
        EXPECT(tm / bbx::kTileBand == lt / (bbx::kTileBand * tiles_n));  // bands in order
      }
      EXPECT(std::all_of(seen.begin(), seen.end(), [](int c) { return c == 1; }));
    }
}

// The bulk gather's row segments (gather_segment in csrc/contraction.h): over
// random row-path records (outer modes in any source order, destination rows
// padded), the segments write every destination element once and no padding,
// read the source element the mode strides give, and their whole 16-byte
// blocks [c0, c1) lie inside the segment with at most 3 elements on each side.
static void test_gather_segments() {
  unsigned seed = 777;
  auto rnd = [&](int lo, int hi) {
    seed = seed * 1103515245u + 12345u;
    return lo + (int)((seed >> 8) % (unsigned)(hi - lo + 1));
  };
  for (int trial = 0; trial < 200; ++trial) {
    const int rank = rnd(1, 3);
    long long dims[3] = {1, 1, 1};
    for (int d = 0; d < rank; ++d) dims[d] = d == rank - 1 ? rnd(1, 2600) : rnd(1, 7);
    const long long L = dims[rank - 1];
    // source: the outer modes in a random order of strides, the row contiguous
    long long istr[3] = {0, 0, 0};
    {
      int order[2] = {0, 1};
      if (rank == 3 && rnd(0, 1)) std::swap(order[0], order[1]);
      long long st = L;
      for (int q = rank - 2; q >= 0; --q) {
        const int d = rank == 3 ? order[q] : q;
        istr[d] = st;
        st *= dims[d];
      }
      istr[rank - 1] = 1;
    }
    const long long pitch = L + rnd(0, 9);
    long long ostr[3] = {0, 0, 0};
    {
      long long st = pitch;
      for (int d = rank - 2; d >= 0; --d) {
        ostr[d] = st;
        st *= dims[d];
      }
      ostr[rank - 1] = 1;
    }
    bbx::GatherRec R{};
    R.a.rank_o = rank;
    for (int d = 0; d < rank; ++d) {
      R.a.odims[d] = dims[d];
      R.a.istride[d] = istr[d];
      R.a.ostride[d] = ostr[d];
    }
    long long rows = 1;
    for (int d = 0; d + 1 < rank; ++d) rows *= dims[d];
    R.n = rows * L;
    R.row_len = L;
    R.segs = (L + bbx::kGatherSeg - 1) / bbx::kGatherSeg;
    std::vector<int> hit(rows * pitch, 0);
    bool ok = true;
    for (long long local = 0; local < rows * R.segs; ++local) {
      const bbx::GatherSeg g = bbx::gather_segment(R, local);
      ok = ok && g.len > 0 && g.len <= bbx::kGatherSeg && g.so >= 0 && g.so + g.len <= R.n;
      ok = ok && g.c0 % 4 == 0 && g.c1 % 4 == 0 && g.so <= g.c0 && g.c0 <= g.c1 && g.c1 <= g.so + g.len;
      ok = ok && (g.c1 == g.c0 || (g.c0 - g.so <= 3 && g.so + g.len - g.c1 <= 3));
      for (int y = 0; y < g.len && ok; ++y) {
        const long long o = g.dso + y;
        ok = o >= 0 && o < (long long)hit.size();
        if (!ok) break;
        ++hit[o];
        // destination coordinates of o, and the source element they name
        long long rem = o / pitch, x = o % pitch, src = x;
        ok = x < L;
        for (int d = rank - 2; d >= 0; --d) {
          src += (rem % dims[d]) * istr[d];
          rem /= dims[d];
        }
        ok = ok && src == g.so + y;
      }
    }
    EXPECT(ok);
    bool once = true;
    for (long long o = 0; o < (long long)hit.size(); ++o) once = once && hit[o] == ((o % pitch) < L ? 1 : 0);
    EXPECT(once);
  }
}

int main() {
  test_tile_order();
  test_gather_segments();
  test_contraction_orientation();
  test_sbbts_compile();
  test_bbts_roundtrip();
  test_dense_format();
  test_matcher_types();
  test_command_layout();
  test_reservation_station_basic();
  test_reservation_station_order();
  test_reservation_station_delete_rules();
  test_reservation_station_threads();
  if (g_fail) {
    std::printf("%d failure(s)\n", g_fail);
    return 1;
  }
  std::printf("all host tests passed\n");
  return 0;
}
