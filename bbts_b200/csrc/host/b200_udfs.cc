// B200 implementations of BarbaTOS's block ud functions, registered through
// the reference's ud API. Every impl is is_gpu = true, takes device-resident
// payloads, and enqueues its kernels on params.stream through the C ABI;
// a nonzero C-ABI status becomes std::runtime_error, as the reference reports
// failures by throwing.
//
// ud functions and the reference impl each one replaces:
//   matrix_mult   dense_matrix_mult.cc:50-86 / dense_matrix_gpu_mult.cu:51-85
//   matrix_add    dense_matrix_add.cc:46-77 / dense_matrix_gpu_add.cu:47-85
//   uniform       dense_uniform.cc:50-79 (seeded Philox instead of time()-seeded MCG31)
//   matrix_relu, matrix_relu_dif, matrix_sigmoid, matrix_matrix_hadamard,
//   matrix_weighted_sum          dense_matrix_{relu,relu_dif,sigmoid,hadamard,weighted_sum}.cc
//   ffnn_*        applications/fnn/ffnn_*.cc (registered at ffnn_lib_init.cc:20-177)
//   contraction   libraries/cutensor/contraction.h:633-695
//   ffnn_softmax_ce  new: softmax cross-entropy loss + gradient (no reference counterpart)
#include <atomic>
#include <stdexcept>
#include "bbts_b200.h"
#include "ud_function.h"

namespace bbts {

namespace {

void ok(int rc) {
  if (rc != 0) {
    char buf[1024];
    bbx_last_error(buf, sizeof(buf));
    throw std::runtime_error(std::string("bbts_b200: ") + buf);
  }
}

using params_t = ud_impl_t::tensor_params_t;
using targs_t = ud_impl_t::tensor_args_t;
using margs_t = ud_impl_t::meta_args_t;
using hint_fn = std::function<size_t(const params_t&, const margs_t&)>;
using meta_fn = std::function<void(const params_t&, const margs_t&, margs_t&)>;

// A B200 impl assembled from three callables.
struct b200_impl_t : public ud_impl_t {
  hint_fn hint;
  meta_fn meta;
  b200_impl_t(std::string impl, std::string ud, std::vector<std::string> in,
              std::vector<std::string> out, std::vector<int32_t> inplace, ud_impl_callable f,
              hint_fn h, meta_fn m)
      : hint(std::move(h)), meta(std::move(m)) {
    impl_name = std::move(impl);
    ud_name = std::move(ud);
    inputTypes = std::move(in);
    outputTypes = std::move(out);
    inputInplace = std::move(inplace);
    is_gpu = true;
    fn = std::move(f);
    gpu_fn = fn;
  }
  size_t get_complexity_hint(const params_t& p, const margs_t& in) override { return hint(p, in); }
  void get_out_meta(const params_t& p, const margs_t& in, margs_t& out) const override { meta(p, in, out); }
};

const dense_tensor_meta_t::m_t& dm(const tensor_meta_t& t) { return t.as<dense_tensor_meta_t>().m(); }
dense_tensor_meta_t::m_t& dm(tensor_meta_t& t) { return t.as<dense_tensor_meta_t>().m(); }
const ffnn_dense_meta_t::m_t& fm(const tensor_meta_t& t) { return t.as<ffnn_dense_meta_t>().m(); }
ffnn_dense_meta_t::m_t& fm(tensor_meta_t& t) { return t.as<ffnn_dense_meta_t>().m(); }

// ------------------------------------------------------------------ dense matmul
// op(A) is I x K, op(B) is K x J; transpose flags are params b0 / b1
// (dense_matrix_mult.cc:78-79). Leading dimensions are the stored row widths
// (the reference passes K and J, which equals these only for square blocks).
struct mm_shape { uint32_t I, J, K, lda, ldb; bool ta, tb; };
mm_shape mm_dims(const params_t& p, const tensor_meta_t& a, const tensor_meta_t& b) {
  mm_shape s;
  s.ta = p.get_bool_or_default<0>(false);
  s.tb = p.get_bool_or_default<1>(false);
  const auto &ma = dm(a), &mb = dm(b);
  s.I = s.ta ? ma.num_cols : ma.num_rows;
  s.K = s.ta ? ma.num_rows : ma.num_cols;
  s.J = s.tb ? mb.num_rows : mb.num_cols;
  uint32_t kb = s.tb ? mb.num_cols : mb.num_rows;
  if (kb != s.K) throw std::runtime_error("matrix_mult: inner dimensions differ");
  s.lda = ma.num_cols;
  s.ldb = mb.num_cols;
  return s;
}

hint_fn mm_hint = [](const params_t& p, const margs_t& in) -> size_t {
  auto s = mm_dims(p, in.get<0>(), in.get<1>());
  return (size_t)s.I * s.J * s.K;
};
meta_fn mm_meta = [](const params_t& p, const margs_t& in, margs_t& out) {
  auto s = mm_dims(p, in.get<0>(), in.get<1>());
  dm(out.get<0>()) = {s.I, s.J, 1.0f};
};

void mm_tc(const params_t& p, const targs_t& in, targs_t& out, int in_dtype, bool out_bf16) {
  auto& a = in.get<0>().as<dense_tensor_t>();
  auto& b = in.get<1>().as<dense_tensor_t>();
  auto& c = out.get<0>().as<dense_tensor_t>();
  auto s = mm_dims(p, a._meta, b._meta);
  bbx_tc_problem_t q{};
  q.a = a.raw(); q.b = b.raw(); q.c = c.raw();
  q.m = (int)s.I; q.n = (int)s.J; q.k = (int)s.K;
  q.trans_a = s.ta; q.trans_b = s.tb;
  q.lda = s.lda; q.ldb = s.ldb; q.ldc = s.J;
  q.alpha = 1.0f;
  if (in_dtype == BBX_E4M3) q.alpha = dm(a._meta).scale * dm(b._meta).scale;
  q.flags = out_bf16 ? BBX_EPI_OUT_BF16 : 0;
  ok(bbx_matmul_tc(in_dtype, &q, 1, 0, p.stream));
  dm(c._meta) = {s.I, s.J, 1.0f};
}

// ------------------------------------------------------------------ elementwise helpers
hint_fn ew_hint = [](const params_t&, const margs_t& in) -> size_t {
  return (size_t)dm(in.get<0>()).num_rows * dm(in.get<0>()).num_cols;
};
meta_fn same_meta = [](const params_t&, const margs_t& in, margs_t& out) {
  dm(out.get<0>()) = {dm(in.get<0>()).num_rows, dm(in.get<0>()).num_cols, 1.0f};
};

// One grouped-stream op on a dense block of any element type (f32 / bf16).
void dense_stream(const params_t& p, int kind, int op, const std::vector<const tensor_t*>& ins,
                  tensor_t& out, int dtype, float p0, float p1, int out_dtype = -1) {
  bbx_stream_op_t s{};
  s.kind = kind; s.op = op; s.in_dtype = dtype; s.out_dtype = out_dtype < 0 ? dtype : out_dtype;
  s.n_in = (int)ins.size(); s.kahan = 1;
  const auto& m = dm(ins[0]->_meta);
  s.n = (long long)m.num_rows * m.num_cols;
  for (size_t i = 0; i < ins.size(); ++i) s.in[i] = ins[i]->payload();
  s.out = out.payload();
  s.p0 = p0; s.p1 = p1;
  ok(bbx_stream_group(&s, 1, p.stream));
  dm(out._meta) = {m.num_rows, m.num_cols, 1.0f};
}

void check_same(const tensor_meta_t& a, const tensor_meta_t& b, const char* what) {
  if (dm(a).num_rows != dm(b).num_rows || dm(a).num_cols != dm(b).num_cols)
    throw std::runtime_error(std::string(what) + ": block shapes differ");
}

// ------------------------------------------------------------------ ffnn helpers
meta_fn ffnn_same_meta_bias = [](const params_t&, const margs_t& in, margs_t& out) {
  auto& a = fm(in.get<0>());
  fm(out.get<0>()) = {a.num_rows, a.num_cols, a.has_bias};
};
meta_fn ffnn_same_meta_nobias = [](const params_t&, const margs_t& in, margs_t& out) {
  auto& a = fm(in.get<0>());
  fm(out.get<0>()) = {a.num_rows, a.num_cols, false};
};
hint_fn ffnn_ew_hint = [](const params_t&, const margs_t& in) -> size_t {
  return (size_t)fm(in.get<0>()).num_rows * fm(in.get<0>()).num_cols;
};

long long fn_elems(const tensor_meta_t& m) { return (long long)fm(m).num_rows * fm(m).num_cols; }

unsigned long long next_seed() {
  static std::atomic<unsigned long long> ctr{0};
  return 0x5eedull + 0x9E3779B97F4A7C15ull * (ctr++ + 1);
}

// Registers a ud function unless one of that name exists (register_udf then
// returns -1 and drops the new one, here and in the reference,
// udf_manager.cc:78-95). Only the reference's own member functions are called
// on the manager, so this also runs against a reference node's manager.
void register_ud(udf_manager_t& udm, const char* name, bool ass, bool com, size_t nin, size_t nout) {
  auto f = std::make_unique<ud_func_t>();
  f->ud_name = name;
  f->is_ass = ass;
  f->is_com = com;
  f->num_in = nin;
  f->num_out = nout;
  udm.register_udf(std::move(f));
}

void add_impl(udf_manager_t& udm, ud_impl_ptr_t impl) {
  auto id = udm.register_udf_impl(std::move(impl));
  if (id.ud_id < 0) throw std::runtime_error("bbts_b200: failed to register a ud impl");
}

}  // namespace

void register_b200_formats(tensor_factory_t& tf) {
  tf.register_fmt("dense", dense_creation_fs(ELEM_F32));
  tf.register_fmt("dense_bf16", dense_creation_fs(ELEM_BF16));
  tf.register_fmt("dense_e4m3", dense_creation_fs(ELEM_E4M3));
  tf.register_fmt("ffnn_dense", ffnn_dense_creation_fs());
  tf.register_fmt("cutensor", cutensor_creation_fs());
  // int32 class labels, one per row (payload = rows x int32), for ffnn_softmax_ce
  tensor_creation_fs_t labels = dense_creation_fs(ELEM_F32);
  tf.register_fmt("labels", labels);
}

void register_b200_udfs(udf_manager_t& udm) {
  using V = std::vector<std::string>;
  // ---- builtin block uds (src/ud_functions/builtin_functions.cc:4-44)
  register_ud(udm, "matrix_add", true, true, 2, 1);
  register_ud(udm, "matrix_mult", true, false, 2, 1);
  register_ud(udm, "uniform", false, false, 0, 1);
  // compiled-but-unregistered reference impls get ud functions of their own names
  register_ud(udm, "matrix_relu", false, false, 1, 1);
  register_ud(udm, "matrix_relu_dif", false, false, 1, 1);
  register_ud(udm, "matrix_sigmoid", false, false, 1, 1);
  register_ud(udm, "matrix_matrix_hadamard", true, true, 2, 1);
  register_ud(udm, "matrix_weighted_sum", true, false, 2, 1);

  // matrix_mult: the plain FP32 path (SIMT) and the tensor-core paths
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_dense_mult_f32", "matrix_mult", V{"dense", "dense"}, V{"dense"}, std::vector<int32_t>{},
      [](const params_t& p, const targs_t& in, targs_t& out) {
        auto& a = in.get<0>().as<dense_tensor_t>();
        auto& b = in.get<1>().as<dense_tensor_t>();
        auto& c = out.get<0>().as<dense_tensor_t>();
        auto s = mm_dims(p, a._meta, b._meta);
        ok(bbx_matmul_f32(a.data(), b.data(), c.data(), (int)s.I, (int)s.J, (int)s.K, s.lda, s.ldb, s.J,
                          s.ta, s.tb, 1.f, 0.f, nullptr, 0, 1, 0, 0, 0, p.stream));
        dm(c._meta) = {s.I, s.J, 1.0f};
      },
      mm_hint, mm_meta));
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_dense_mult_bf16", "matrix_mult", V{"dense_bf16", "dense_bf16"}, V{"dense"},
      std::vector<int32_t>{},
      [](const params_t& p, const targs_t& in, targs_t& out) { mm_tc(p, in, out, BBX_BF16, false); },
      mm_hint, mm_meta));
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_dense_mult_bf16_out_bf16", "matrix_mult", V{"dense_bf16", "dense_bf16"}, V{"dense_bf16"},
      std::vector<int32_t>{},
      [](const params_t& p, const targs_t& in, targs_t& out) { mm_tc(p, in, out, BBX_BF16, true); },
      mm_hint, mm_meta));
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_dense_mult_e4m3", "matrix_mult", V{"dense_e4m3", "dense_e4m3"}, V{"dense"},
      std::vector<int32_t>{},
      [](const params_t& p, const targs_t& in, targs_t& out) { mm_tc(p, in, out, BBX_E4M3, false); },
      mm_hint, mm_meta));

  // matrix_add (f32 and bf16 blocks); both inputs may be the in-place output
  for (int dt : {BBX_F32, BBX_BF16}) {
    const char* fmt = dt == BBX_F32 ? "dense" : "dense_bf16";
    add_impl(udm, std::make_unique<b200_impl_t>(
        dt == BBX_F32 ? "b200_dense_add" : "b200_dense_bf16_add", "matrix_add", V{fmt, fmt}, V{fmt},
        std::vector<int32_t>{0, 1},
        [dt](const params_t& p, const targs_t& in, targs_t& out) {
          check_same(in.get<0>()._meta, in.get<1>()._meta, "matrix_add");
          if (dt == BBX_F32) {
            auto& a = in.get<0>().as<dense_tensor_t>();
            auto& b = in.get<1>().as<dense_tensor_t>();
            auto& c = out.get<0>().as<dense_tensor_t>();
            long long n = (long long)dm(a._meta).num_rows * dm(a._meta).num_cols;
            ok(bbx_add_f32(a.data(), b.data(), c.data(), n, p.stream));
            dm(c._meta) = {dm(a._meta).num_rows, dm(a._meta).num_cols, 1.0f};
          } else {
            dense_stream(p, BBX_S_SUM, 0, {&in.get<0>(), &in.get<1>()}, out.get<0>(), dt, 0, 0);
          }
        },
        ew_hint, same_meta));
  }

  // uniform: params u0 rows, u1 cols, f2 left (0), f3 right (1), u4 seed (optional)
  for (int dt : {BBX_F32, BBX_BF16}) {
    add_impl(udm, std::make_unique<b200_impl_t>(
        dt == BBX_F32 ? "b200_dense_uniform" : "b200_dense_bf16_uniform", "uniform", V{},
        V{dt == BBX_F32 ? "dense" : "dense_bf16"}, std::vector<int32_t>{},
        [dt](const params_t& p, const targs_t&, targs_t& out) {
          auto& c = out.get<0>().as<dense_tensor_t>();
          uint32_t rows = p.get_uint<0>(), cols = p.get_uint<1>();
          float lo = p.get_float_or_default<2>(0.f), hi = p.get_float_or_default<3>(1.f);
          // explicit seed (param u4) or a per-process call counter, so every block
          // of a program differs (the reference seeds each call with time())
          unsigned long long seed = p.num_parameters() > 4 ? p.get_uint<4>() : next_seed();
          ok(bbx_fill_philox(dt, c.raw(), (long long)rows * cols, seed, 0, lo, hi, p.stream));
          dm(c._meta) = {rows, cols, 1.0f};
        },
        [](const params_t& p, const margs_t&) -> size_t {
          if (p.num_parameters() < 2) throw std::runtime_error("uniform: not enough parameters");
          return (size_t)p.get_uint<0>() * p.get_uint<1>();
        },
        [](const params_t& p, const margs_t&, margs_t& out) {
          dm(out.get<0>()) = {p.get_uint<0>(), p.get_uint<1>(), 1.0f};
        }));
  }

  // elementwise dense uds (f32 and bf16 blocks)
  struct ew_spec { const char* ud; const char* impl; int kind, op, nin; };
  const ew_spec ews[] = {
      {"matrix_relu", "b200_dense_relu", BBX_S_UNARY, BBX_U_RELU, 1},
      {"matrix_relu_dif", "b200_dense_relu_dif", BBX_S_UNARY, BBX_U_RELU_DIF, 1},
      {"matrix_sigmoid", "b200_dense_sigmoid", BBX_S_UNARY, BBX_U_SIGMOID_REF, 1},
      {"matrix_matrix_hadamard", "b200_dense_hadamard", BBX_S_BINARY, BBX_B_HADAMARD, 2},
      {"matrix_weighted_sum", "b200_dense_weighted", BBX_S_BINARY, BBX_B_WEIGHTED, 2},
  };
  for (const auto& e : ews) {
    for (int dt : {BBX_F32, BBX_BF16}) {
      const char* fmt = dt == BBX_F32 ? "dense" : "dense_bf16";
      V ins(e.nin, fmt);
      std::string impl = std::string(e.impl) + (dt == BBX_F32 ? "" : "_bf16");
      add_impl(udm, std::make_unique<b200_impl_t>(
          impl, e.ud, ins, V{fmt}, e.nin == 1 ? std::vector<int32_t>{0} : std::vector<int32_t>{0, 1},
          [e, dt](const params_t& p, const targs_t& in, targs_t& out) {
            std::vector<const tensor_t*> ts;
            for (int i = 0; i < e.nin; ++i) ts.push_back(&in.get_by_idx(i));
            if (e.nin == 2) check_same(ts[0]->_meta, ts[1]->_meta, e.ud);
            float p0 = 0, p1 = 0;
            if (e.op == BBX_B_WEIGHTED && e.kind == BBX_S_BINARY) {
              p0 = p.get_float_or_default<0>(1.f);
              p1 = p.get_float_or_default<1>(1.f);
            }
            dense_stream(p, e.kind, e.op, ts, out.get<0>(), dt, p0, p1);
          },
          ew_hint, same_meta));
    }
  }

  // relu of an f32 block written as bf16 (the activation of a layer whose
  // pre-activation was accumulated in f32)
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_dense_relu_to_bf16", "matrix_relu", V{"dense"}, V{"dense_bf16"}, std::vector<int32_t>{},
      [](const params_t& p, const targs_t& in, targs_t& out) {
        dense_stream(p, BBX_S_UNARY, BBX_U_RELU, {&in.get<0>()}, out.get<0>(), BBX_F32, 0, 0, BBX_BF16);
      },
      ew_hint, same_meta));

  // relu of an f32 block split into hi = bf16(relu(z)) and lo = bf16(relu(z) - hi)
  // (new ud, no reference counterpart): the activation of a layer followed by
  // another ReLU layer, whose masks would flip on a bf16-rounded operand; the
  // next layer multiplies both parts and sums them in f32. (The impl name does
  // not start with "b200_dense_relu": the DAG executor runs it through its fn,
  // not as a one-output streaming relu.)
  register_ud(udm, "matrix_relu_split", false, false, 1, 2);
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_dense_split_relu", "matrix_relu_split", V{"dense"}, V{"dense_bf16", "dense_bf16"},
      std::vector<int32_t>{},
      [](const params_t& p, const targs_t& in, targs_t& out) {
        auto& z = in.get<0>().as<dense_tensor_t>();
        auto& hi = out.get<0>().as<dense_tensor_t>();
        auto& lo = out.get<1>().as<dense_tensor_t>();
        auto& mz = dm(z._meta);
        dm(hi._meta) = {mz.num_rows, mz.num_cols, 1.0f};
        dm(lo._meta) = {mz.num_rows, mz.num_cols, 1.0f};
        ok(bbx_relu_split(z.data(), hi.raw(), lo.raw(), (long long)mz.num_rows * mz.num_cols, p.stream));
      },
      ew_hint,
      [](const params_t&, const margs_t& in, margs_t& out) {
        auto& mz = dm(in.get<0>());
        dm(out.get<0>()) = {mz.num_rows, mz.num_cols, 1.0f};
        dm(out.get<1>()) = {mz.num_rows, mz.num_cols, 1.0f};
      }));

  // ---- FNN application uds (applications/fnn/ffnn_lib_init.cc:20-177)
  register_ud(udm, "ffnn_act_mult", false, false, 2, 1);
  register_ud(udm, "ffnn_add", true, true, 2, 1);
  register_ud(udm, "ffnn_matrix_hadamard", true, true, 2, 1);
  register_ud(udm, "ffnn_mult", false, false, 2, 1);
  register_ud(udm, "ffnn_relu", false, false, 1, 1);  // the reference declares 2 inputs for a 1-input impl
  register_ud(udm, "ffnn_relu_dif", false, false, 1, 1);
  register_ud(udm, "ffnn_sigmoid", false, false, 1, 1);
  register_ud(udm, "ffnn_uniform_data", false, false, 0, 1);
  register_ud(udm, "ffnn_uniform_weights", false, false, 0, 1);
  register_ud(udm, "ffnn_weighted_sum", true, false, 2, 1);
  register_ud(udm, "ffnn_back_mult", false, false, 2, 1);
  register_ud(udm, "ffnn_softmax_ce", false, false, 2, 2);

  const V FF{"ffnn_dense"};
  // X.W + bias (ffnn_activation_mult.cc:56-96): bias fused into the matmul epilogue
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_ffnn_act_mult", "ffnn_act_mult", V{"ffnn_dense", "ffnn_dense"}, FF, std::vector<int32_t>{},
      [](const params_t& p, const targs_t& in, targs_t& out) {
        auto& a = in.get<0>().as<ffnn_dense_t>();
        auto& b = in.get<1>().as<ffnn_dense_t>();
        auto& c = out.get<0>().as<ffnn_dense_t>();
        auto &ma = fm(a._meta), &mb = fm(b._meta);
        if (ma.num_cols != mb.num_rows) throw std::runtime_error("ffnn_act_mult: inner dimensions differ");
        if (!mb.has_bias) throw std::runtime_error("ffnn_act_mult: weights carry no bias");
        fm(c._meta) = {ma.num_rows, mb.num_cols, false};
        ok(bbx_matmul_f32(a.data(), b.data(), c.data(), ma.num_rows, mb.num_cols, ma.num_cols, ma.num_cols,
                          mb.num_cols, mb.num_cols, 0, 0, 1.f, 0.f, b.bias(), 0, 1, 0, 0, 0, p.stream));
      },
      [](const params_t&, const margs_t& in) -> size_t {
        return (size_t)fm(in.get<0>()).num_rows * fm(in.get<0>()).num_cols * fm(in.get<1>()).num_cols;
      },
      [](const params_t&, const margs_t& in, margs_t& out) {
        fm(out.get<0>()) = {fm(in.get<0>()).num_rows, fm(in.get<1>()).num_cols, false};
      }));
  // op(A).op(B) with transpose flags b0/b1 (ffnn_mult.cc:54-93)
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_ffnn_mult", "ffnn_mult", V{"ffnn_dense", "ffnn_dense"}, FF, std::vector<int32_t>{},
      [](const params_t& p, const targs_t& in, targs_t& out) {
        auto& a = in.get<0>().as<ffnn_dense_t>();
        auto& b = in.get<1>().as<ffnn_dense_t>();
        auto& c = out.get<0>().as<ffnn_dense_t>();
        bool ta = p.get_bool_or_default<0>(false), tb = p.get_bool_or_default<1>(false);
        auto &ma = fm(a._meta), &mb = fm(b._meta);
        uint32_t I = ta ? ma.num_cols : ma.num_rows, K = ta ? ma.num_rows : ma.num_cols;
        uint32_t J = tb ? mb.num_rows : mb.num_cols, K2 = tb ? mb.num_cols : mb.num_rows;
        if (K != K2) throw std::runtime_error("ffnn_mult: inner dimensions differ");
        fm(c._meta) = {I, J, false};
        ok(bbx_matmul_f32(a.data(), b.data(), c.data(), I, J, K, ma.num_cols, mb.num_cols, J, ta, tb, 1.f, 0.f,
                          nullptr, 0, 1, 0, 0, 0, p.stream));
      },
      [](const params_t& p, const margs_t& in) -> size_t {
        bool ta = p.get_bool_or_default<0>(false), tb = p.get_bool_or_default<1>(false);
        auto &ma = fm(in.get<0>()), &mb = fm(in.get<1>());
        return (size_t)(ta ? ma.num_cols : ma.num_rows) * (ta ? ma.num_rows : ma.num_cols) *
               (tb ? mb.num_rows : mb.num_cols);
      },
      [](const params_t& p, const margs_t& in, margs_t& out) {
        bool ta = p.get_bool_or_default<0>(false), tb = p.get_bool_or_default<1>(false);
        auto &ma = fm(in.get<0>()), &mb = fm(in.get<1>());
        fm(out.get<0>()) = {ta ? ma.num_cols : ma.num_rows, tb ? mb.num_rows : mb.num_cols, false};
      }));
  // A^T.B with the bias = column sums of B (ffnn_back_mult.cc:52-91; the bias
  // starts from zero here, the reference adds into uninitialised memory)
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_ffnn_back_mult", "ffnn_back_mult", V{"ffnn_dense", "ffnn_dense"}, FF, std::vector<int32_t>{},
      [](const params_t& p, const targs_t& in, targs_t& out) {
        auto& a = in.get<0>().as<ffnn_dense_t>();
        auto& b = in.get<1>().as<ffnn_dense_t>();
        auto& c = out.get<0>().as<ffnn_dense_t>();
        auto &ma = fm(a._meta), &mb = fm(b._meta);
        if (ma.num_rows != mb.num_rows) throw std::runtime_error("ffnn_back_mult: row counts differ");
        fm(c._meta) = {ma.num_cols, mb.num_cols, true};
        ok(bbx_matmul_f32(a.data(), b.data(), c.data(), ma.num_cols, mb.num_cols, ma.num_rows, ma.num_cols,
                          mb.num_cols, mb.num_cols, 1, 0, 1.f, 0.f, nullptr, 0, 1, 0, 0, 0, p.stream));
        ok(bbx_colsum_f32(b.data(), c.bias(), mb.num_rows, mb.num_cols, mb.num_cols, 0, p.stream));
      },
      [](const params_t&, const margs_t& in) -> size_t {
        return (size_t)fm(in.get<0>()).num_cols * fm(in.get<0>()).num_rows * fm(in.get<1>()).num_cols;
      },
      [](const params_t&, const margs_t& in, margs_t& out) {
        fm(out.get<0>()) = {fm(in.get<0>()).num_cols, fm(in.get<1>()).num_cols, true};
      }));
  // ffnn add / weighted sum / hadamard: data, and the bias rows when both carry one
  struct ffb { const char* ud; const char* impl; int op; };
  for (const ffb& e : {ffb{"ffnn_add", "b200_ffnn_add", BBX_B_ADD},
                       ffb{"ffnn_weighted_sum", "b200_ffnn_weighted_sum", BBX_B_WEIGHTED},
                       ffb{"ffnn_matrix_hadamard", "b200_ffnn_matrix_hadamard", BBX_B_HADAMARD}}) {
    add_impl(udm, std::make_unique<b200_impl_t>(
        e.impl, e.ud, V{"ffnn_dense", "ffnn_dense"}, FF, std::vector<int32_t>{0, 1},
        [e](const params_t& p, const targs_t& in, targs_t& out) {
          auto& a = in.get<0>().as<ffnn_dense_t>();
          auto& b = in.get<1>().as<ffnn_dense_t>();
          auto& c = out.get<0>().as<ffnn_dense_t>();
          auto &ma = fm(a._meta), &mb = fm(b._meta);
          if (ma.num_rows != mb.num_rows || ma.num_cols != mb.num_cols)
            throw std::runtime_error(std::string(e.ud) + ": block shapes differ");
          float ca = 1.f, cb = 1.f;
          if (e.op == BBX_B_WEIGHTED) { ca = p.get_float_or_default<0>(1.f); cb = p.get_float_or_default<1>(1.f); }
          const bool both = ma.has_bias && mb.has_bias;
          fm(c._meta) = {ma.num_rows, ma.num_cols, ma.has_bias};
          ok(bbx_binary_f32(e.op, a.data(), b.data(), c.data(), fn_elems(a._meta), ca, cb, p.stream));
          if (both) ok(bbx_binary_f32(e.op, a.bias(), b.bias(), c.bias(), ma.num_cols, ca, cb, p.stream));
        },
        ffnn_ew_hint, ffnn_same_meta_bias));
  }
  struct ffu { const char* ud; const char* impl; int op; };
  for (const ffu& e : {ffu{"ffnn_relu", "b200_ffnn_relu", BBX_U_RELU},
                       ffu{"ffnn_relu_dif", "b200_ffnn_relu_dif", BBX_U_RELU_DIF},
                       ffu{"ffnn_sigmoid", "b200_ffnn_sigmoid", BBX_U_SIGMOID_REF}}) {
    add_impl(udm, std::make_unique<b200_impl_t>(
        e.impl, e.ud, V{"ffnn_dense"}, FF, std::vector<int32_t>{0},
        [e](const params_t& p, const targs_t& in, targs_t& out) {
          auto& a = in.get<0>().as<ffnn_dense_t>();
          auto& c = out.get<0>().as<ffnn_dense_t>();
          fm(c._meta) = {fm(a._meta).num_rows, fm(a._meta).num_cols, false};
          ok(bbx_unary_f32(e.op, a.data(), c.data(), fn_elems(a._meta), 0.f, p.stream));
        },
        ffnn_ew_hint, ffnn_same_meta_nobias));
  }
  // uniform data / weights: params i0 rows, i1 cols, f2 left, f3 right, u4 seed
  for (int w = 0; w < 2; ++w) {
    add_impl(udm, std::make_unique<b200_impl_t>(
        w ? "b200_ffnn_uniform_weights" : "b200_ffnn_uniform_data", w ? "ffnn_uniform_weights" : "ffnn_uniform_data",
        V{}, FF, std::vector<int32_t>{},
        [w](const params_t& p, const targs_t&, targs_t& out) {
          auto& c = out.get<0>().as<ffnn_dense_t>();
          uint32_t rows = p.get_uint<0>(), cols = p.get_uint<1>();
          fm(c._meta) = {rows, cols, (bool)w};
          long long n = (long long)(rows + (w ? 1 : 0)) * cols;  // weights: data + bias row
          ok(bbx_fill_philox(BBX_F32, c.data(), n, p.num_parameters() > 4 ? p.get_uint<4>() : next_seed(), 0,
                             p.get_float_or_default<2>(0.f), p.get_float_or_default<3>(1.f), p.stream));
        },
        [](const params_t& p, const margs_t&) -> size_t {
          if (p.num_parameters() < 2) throw std::runtime_error("ffnn uniform: not enough parameters");
          return (size_t)p.get_uint<0>() * p.get_uint<1>();
        },
        [w](const params_t& p, const margs_t&, margs_t& out) {
          fm(out.get<0>()) = {p.get_uint<0>(), p.get_uint<1>(), (bool)w};
        }));
  }
  // softmax cross-entropy: in (logits ffnn_dense, labels) -> (grad ffnn_dense, loss ffnn_dense rows x 1)
  // param f0 = gradient scale (1/batch for a mean loss)
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_ffnn_softmax_ce", "ffnn_softmax_ce", V{"ffnn_dense", "labels"}, V{"ffnn_dense", "ffnn_dense"},
      std::vector<int32_t>{},
      [](const params_t& p, const targs_t& in, targs_t& out) {
        auto& z = in.get<0>().as<ffnn_dense_t>();
        auto& y = in.get<1>().as<dense_tensor_t>();
        auto& g = out.get<0>().as<ffnn_dense_t>();
        auto& l = out.get<1>().as<ffnn_dense_t>();
        auto& mz = fm(z._meta);
        if (dm(y._meta).num_rows * dm(y._meta).num_cols != mz.num_rows)
          throw std::runtime_error("ffnn_softmax_ce: one label per row expected");
        fm(g._meta) = {mz.num_rows, mz.num_cols, false};
        fm(l._meta) = {mz.num_rows, 1, false};
        ok(bbx_softmax_ce_f32(z.data(), (const int*)y.raw(), l.data(), g.data(), mz.num_rows, mz.num_cols,
                              mz.num_cols, p.get_float_or_default<0>(1.f), p.stream));
      },
      ffnn_ew_hint,
      [](const params_t&, const margs_t& in, margs_t& out) {
        auto& mz = fm(in.get<0>());
        fm(out.get<0>()) = {mz.num_rows, mz.num_cols, false};
        fm(out.get<1>()) = {mz.num_rows, 1, false};
      }));

  // softmax cross-entropy over dense blocks (new ud, no reference counterpart):
  // in (logits "dense" f32, labels) -> (grad dense / dense_bf16, loss dense rows x 1); f0 = grad scale
  register_ud(udm, "matrix_softmax_ce", false, false, 2, 2);
  for (int gdt : {BBX_F32, BBX_BF16}) {
    add_impl(udm, std::make_unique<b200_impl_t>(
        gdt == BBX_F32 ? "b200_dense_softmax_ce" : "b200_dense_softmax_ce_bf16", "matrix_softmax_ce",
        V{"dense", "labels"}, V{gdt == BBX_F32 ? "dense" : "dense_bf16", "dense"}, std::vector<int32_t>{},
        [gdt](const params_t& p, const targs_t& in, targs_t& out) {
          auto& z = in.get<0>().as<dense_tensor_t>();
          auto& y = in.get<1>().as<dense_tensor_t>();
          auto& g = out.get<0>().as<dense_tensor_t>();
          auto& l = out.get<1>().as<dense_tensor_t>();
          auto& mz = dm(z._meta);
          if (dm(y._meta).num_rows * dm(y._meta).num_cols != mz.num_rows)
            throw std::runtime_error("matrix_softmax_ce: one label per row expected");
          dm(g._meta) = {mz.num_rows, mz.num_cols, 1.0f};
          dm(l._meta) = {mz.num_rows, 1, 1.0f};
          ok(bbx_softmax_ce(z.data(), (const int*)y.raw(), l.data(), g.raw(), gdt, mz.num_rows, mz.num_cols,
                            mz.num_cols, p.get_float_or_default<0>(1.f), p.stream));
        },
        ew_hint,
        [](const params_t&, const margs_t& in, margs_t& out) {
          auto& mz = dm(in.get<0>());
          dm(out.get<0>()) = {mz.num_rows, mz.num_cols, 1.0f};
          dm(out.get<1>()) = {mz.num_rows, 1, 1.0f};
        }));
  }

  // ---- reduction / ew / ewb / ewb_castable / expand of the cutensor plugin
  // (libraries/cutensor.cc:20-28 registers them under these names)
  auto cu_shape = [](const tensor_meta_t& m) -> const cu_shape_t& { return m.as<cu_meta_t>().m(); };
  auto cu_elems = [](const cu_shape_t& s) { size_t n = 1; for (uint32_t r = 0; r < s.rank; ++r) n *= (size_t)s.dims[r]; return n; };
  auto ints_from = [](const params_t& p, size_t first) {
    std::vector<int> v;
    for (size_t i = first; i < p.num_parameters(); ++i) v.push_back(p.get_raw(i).i);
    return v;
  };
  const V CU{"cutensor"}, CU2{"cutensor", "cutensor"};
  register_ud(udm, "reduction", false, false, 1, 1);
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_reduction", "reduction", CU, CU, std::vector<int32_t>{},
      [cu_shape, ints_from](const params_t& p, const targs_t& in, targs_t& out) {
        const auto& si = cu_shape(in.get<0>()._meta);
        auto ord = ints_from(p, 2);
        auto& so = out.get<0>().as<cu_t>().meta().m();
        so.rank = (uint32_t)ord.size();
        for (size_t r = 0; r < ord.size(); ++r) so.dims[r] = si.dims[ord[r]];
        std::vector<long long> d(si.dims, si.dims + si.rank);
        ok(bbx_cu_reduction((const float*)in.get<0>().payload(), (int)si.rank, d.data(), p.get_raw(0).i,
                            p.get_raw(1).f, ord.data(), (int)ord.size(), (float*)out.get<0>().payload(), p.stream));
      },
      [cu_shape, cu_elems](const params_t&, const margs_t& in) -> size_t { return cu_elems(cu_shape(in.get<0>())); },
      [cu_shape, ints_from](const params_t& p, const margs_t& in, margs_t& out) {
        const auto& si = cu_shape(in.get<0>());
        auto ord = ints_from(p, 2);
        auto& so = out.get<0>().as<cu_meta_t>().m();
        so.rank = (uint32_t)ord.size();
        for (size_t r = 0; r < ord.size(); ++r) so.dims[r] = si.dims[ord[r]];
      }));
  // ew params: uop, [scalar if uop == 6], alpha, ordering...
  auto ew_parse = [](const params_t& p, int& uop, float& scalar, float& alpha, std::vector<int>& ord) {
    size_t i = 0;
    uop = p.get_raw(i++).i;
    if (uop < 0 || uop > 6) throw std::invalid_argument("is not a valid unary op");
    scalar = uop == 6 ? p.get_raw(i++).f : 0.f;
    alpha = p.get_raw(i++).f;
    ord.clear();
    for (; i < p.num_parameters(); ++i) ord.push_back(p.get_raw(i).i);
  };
  register_ud(udm, "ew", false, false, 1, 1);
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_ew", "ew", CU, CU, std::vector<int32_t>{},
      [cu_shape, ew_parse](const params_t& p, const targs_t& in, targs_t& out) {
        const auto& si = cu_shape(in.get<0>()._meta);
        int uop; float sc, al; std::vector<int> ord;
        ew_parse(p, uop, sc, al, ord);
        if (ord.size() != si.rank) throw std::invalid_argument("input rank is incorrect");
        auto& so = out.get<0>().as<cu_t>().meta().m();
        so.rank = si.rank;
        for (size_t r = 0; r < ord.size(); ++r) so.dims[r] = si.dims[ord[r]];
        std::vector<long long> d(si.dims, si.dims + si.rank);
        ok(bbx_cu_ew((const float*)in.get<0>().payload(), (int)si.rank, d.data(), uop, sc, al, ord.data(),
                     (float*)out.get<0>().payload(), p.stream));
      },
      [cu_shape, cu_elems](const params_t&, const margs_t& in) -> size_t { return cu_elems(cu_shape(in.get<0>())); },
      [cu_shape, ew_parse](const params_t& p, const margs_t& in, margs_t& out) {
        const auto& si = cu_shape(in.get<0>());
        int uop; float sc, al; std::vector<int> ord;
        ew_parse(p, uop, sc, al, ord);
        auto& so = out.get<0>().as<cu_meta_t>().m();
        so.rank = (uint32_t)ord.size();
        for (size_t r = 0; r < ord.size() && r < 4; ++r) so.dims[r] = si.dims[ord[r]];
      }));
  // ewb params: op, alpha, beta, rank_l, ord_l..., rank_r, ord_r...
  auto ewb_parse = [](const params_t& p, int& op, float& al, float& be, std::vector<int>& ol, std::vector<int>& orr) {
    op = p.get_raw(0).i;
    al = p.get_raw(1).f;
    be = p.get_raw(2).f;
    int rl = p.get_raw(3).i;
    size_t i = 4;
    ol.clear();
    orr.clear();
    for (int r = 0; r < rl; ++r) ol.push_back(p.get_raw(i++).i);
    int rr = p.get_raw(i++).i;
    for (int r = 0; r < rr; ++r) orr.push_back(p.get_raw(i++).i);
  };
  auto ewb_meta = [cu_shape](const std::vector<int>& ol, const std::vector<int>& orr, const tensor_meta_t& l,
                             const tensor_meta_t& r, cu_shape_t& so) {
    const auto &sl = cu_shape(l), &sr = cu_shape(r);
    int rank = 0;
    for (int m : ol) rank = std::max(rank, m + 1);
    for (int m : orr) rank = std::max(rank, m + 1);
    so.rank = (uint32_t)rank;
    for (int d = 0; d < 4; ++d) so.dims[d] = 0;
    for (size_t q = 0; q < ol.size(); ++q) so.dims[ol[q]] = sl.dims[q];
    for (size_t q = 0; q < orr.size(); ++q) so.dims[orr[q]] = sr.dims[q];
  };
  register_ud(udm, "ewb", false, false, 2, 1);
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_ewb", "ewb", CU2, CU, std::vector<int32_t>{},
      [cu_shape, ewb_parse, ewb_meta](const params_t& p, const targs_t& in, targs_t& out) {
        int op; float al, be; std::vector<int> ol, orr;
        ewb_parse(p, op, al, be, ol, orr);
        const auto &sl = cu_shape(in.get<0>()._meta), &sr = cu_shape(in.get<1>()._meta);
        ewb_meta(ol, orr, in.get<0>()._meta, in.get<1>()._meta, out.get<0>().as<cu_t>().meta().m());
        std::vector<long long> dl(sl.dims, sl.dims + sl.rank), dr(sr.dims, sr.dims + sr.rank);
        ok(bbx_cu_ewb((const float*)in.get<0>().payload(), (int)sl.rank, dl.data(), ol.data(),
                      (const float*)in.get<1>().payload(), (int)sr.rank, dr.data(), orr.data(), op, al, be,
                      (float*)out.get<0>().payload(), nullptr, nullptr, p.stream));
      },
      [cu_shape, cu_elems](const params_t&, const margs_t& in) -> size_t {
        return std::max(cu_elems(cu_shape(in.get<0>())), cu_elems(cu_shape(in.get<1>())));
      },
      [ewb_parse, ewb_meta](const params_t& p, const margs_t& in, margs_t& out) {
        int op; float al, be; std::vector<int> ol, orr;
        ewb_parse(p, op, al, be, ol, orr);
        ewb_meta(ol, orr, in.get<0>(), in.get<1>(), out.get<0>().as<cu_meta_t>().m());
      }));
  // ewb_castable: same-shape add / max / min / mul (param op), associative and commutative
  register_ud(udm, "ewb_castable", true, true, 2, 1);
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_ewb_castable", "ewb_castable", CU2, CU, std::vector<int32_t>{0, 1},
      [cu_shape](const params_t& p, const targs_t& in, targs_t& out) {
        const auto &sl = cu_shape(in.get<0>()._meta), &sr = cu_shape(in.get<1>()._meta);
        if (sl.rank != sr.rank) throw std::runtime_error("ewb_castable: ranks differ");
        std::vector<int> ord;
        for (uint32_t r = 0; r < sl.rank; ++r) {
          if (sl.dims[r] != sr.dims[r]) throw std::runtime_error("ewb_castable: shapes differ");
          ord.push_back((int)r);
        }
        auto& so = out.get<0>().as<cu_t>().meta().m();
        so = sl;
        int op = p.get_raw(0).i;
        if (op < 0 || op > 3) throw std::invalid_argument("is not a castable operator");
        std::vector<long long> d(sl.dims, sl.dims + sl.rank);
        ok(bbx_cu_ewb((const float*)in.get<0>().payload(), (int)sl.rank, d.data(), ord.data(),
                      (const float*)in.get<1>().payload(), (int)sr.rank, d.data(), ord.data(), op, 1.f, 1.f,
                      (float*)out.get<0>().payload(), nullptr, nullptr, p.stream));
      },
      [cu_shape, cu_elems](const params_t&, const margs_t& in) -> size_t { return cu_elems(cu_shape(in.get<0>())); },
      [cu_shape](const params_t&, const margs_t& in, margs_t& out) {
        out.get<0>().as<cu_meta_t>().m() = cu_shape(in.get<0>());
      }));
  // expand params: per mode (sz_in, sz_out, num, start_in, start_out)
  register_ud(udm, "expand", false, false, 1, 1);
  add_impl(udm, std::make_unique<b200_impl_t>(
      "b200_expand", "expand", CU, CU, std::vector<int32_t>{},
      [](const params_t& p, const targs_t& in, targs_t& out) {
        const int rank = (int)(p.num_parameters() / 5);
        std::vector<int> q(p.num_parameters());
        for (size_t i = 0; i < q.size(); ++i) q[i] = p.get_raw(i).i;
        auto& so = out.get<0>().as<cu_t>().meta().m();
        so.rank = (uint32_t)rank;
        for (int i = 0; i < rank; ++i) so.dims[i] = q[5 * i + 1];
        ok(bbx_cu_expand((const float*)in.get<0>().payload(), q.data(), rank,
                         (float*)out.get<0>().payload(), p.stream));
      },
      [](const params_t& p, const margs_t&) -> size_t {
        size_t t = 1;
        for (size_t i = 0; i + 4 < p.num_parameters(); i += 5) t *= (size_t)p.get_raw(i + 1).i;
        return t;
      },
      [](const params_t& p, const margs_t&, margs_t& out) {
        auto& so = out.get<0>().as<cu_meta_t>().m();
        so.rank = (uint32_t)(p.num_parameters() / 5);
        for (uint32_t i = 0; i < so.rank; ++i) so.dims[i] = p.get_raw(5 * i + 1).i;
      }));

  // ---- contraction of the cutensor plugin (params: rank_l, rank_r, rank_o,
  // modes_l..., modes_r..., modes_o..., alpha; contraction.h:25-55)
  register_ud(udm, "contraction", false, false, 2, 1);
  struct cinfo { std::vector<int> ml, mr, mo; float alpha; };
  auto parse = [](const params_t& p) {
    cinfo c;
    int rl = p.get_raw(0).i, rr = p.get_raw(1).i, ro = p.get_raw(2).i;
    size_t i = 3;
    for (int d = 0; d < rl; ++d) c.ml.push_back(p.get_raw(i++).i);
    for (int d = 0; d < rr; ++d) c.mr.push_back(p.get_raw(i++).i);
    for (int d = 0; d < ro; ++d) c.mo.push_back(p.get_raw(i++).i);
    c.alpha = p.get_raw(i).f;
    return c;
  };
  auto out_dims = [parse](const params_t& p, const tensor_meta_t& l, const tensor_meta_t& r) {
    auto c = parse(p);
    std::vector<int64_t> ext(16, 1);
    auto& sl = l.as<cu_meta_t>().m();
    auto& sr = r.as<cu_meta_t>().m();
    for (size_t d = 0; d < c.ml.size(); ++d) ext[c.ml[d]] = sl.dims[d];
    for (size_t d = 0; d < c.mr.size(); ++d) ext[c.mr[d]] = sr.dims[d];
    std::vector<int64_t> o;
    for (int m : c.mo) o.push_back(ext[m]);
    return o;
  };
  for (int prec : {BBX_F32, BBX_BF16}) {
    add_impl(udm, std::make_unique<b200_impl_t>(
        prec == BBX_F32 ? "b200_contraction" : "b200_contraction_bf16", "contraction",
        V{"cutensor", "cutensor"}, V{"cutensor"}, std::vector<int32_t>{},
        [parse, out_dims, prec](const params_t& p, const targs_t& in, targs_t& out) {
          auto& l = in.get<0>().as<cu_t>();
          auto& r = in.get<1>().as<cu_t>();
          auto& o = out.get<0>().as<cu_t>();
          auto c = parse(p);
          auto od = out_dims(p, l._meta, r._meta);
          auto& so = o.meta().m();
          so.rank = (uint32_t)od.size();
          for (size_t d = 0; d < od.size(); ++d) so.dims[d] = od[d];
          std::vector<long long> dl(l.meta().m().dims, l.meta().m().dims + l.meta().m().rank);
          std::vector<long long> dr(r.meta().m().dims, r.meta().m().dims + r.meta().m().rank);
          ok(bbx_contraction((const float*)l.data(), (int)dl.size(), dl.data(), c.ml.data(), (const float*)r.data(),
                             (int)dr.size(), dr.data(), c.mr.data(), (float*)o.data(), (int)c.mo.size(),
                             c.mo.data(), c.alpha, prec, p.stream));
        },
        [parse](const params_t& p, const margs_t& in) -> size_t {
          auto c = parse(p);
          std::vector<int64_t> ext(16, 1);
          auto& sl = in.get<0>().as<cu_meta_t>().m();
          auto& sr = in.get<1>().as<cu_meta_t>().m();
          for (size_t d = 0; d < c.ml.size(); ++d) ext[c.ml[d]] = sl.dims[d];
          for (size_t d = 0; d < c.mr.size(); ++d) ext[c.mr[d]] = sr.dims[d];
          size_t prod = 1;
          for (auto e : ext) prod *= (size_t)e;
          return prod;
        },
        [out_dims](const params_t& p, const margs_t& in, margs_t& out) {
          auto od = out_dims(p, in.get<0>(), in.get<1>());
          auto& so = out.get<0>().as<cu_meta_t>().m();
          so.rank = (uint32_t)od.size();
          for (size_t d = 0; d < od.size(); ++d) so.dims[d] = od[d];
        }));
  }
}

}  // namespace bbts

extern "C" void register_tensors(bbts::tensor_factory_ptr_t tensor_factory) {
  bbts::register_b200_formats(*tensor_factory);
}

extern "C" void register_udfs(bbts::udf_manager_ptr udf_manager) { bbts::register_b200_udfs(*udf_manager); }
