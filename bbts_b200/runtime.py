"""Python view of the native runtime (bbx_rt_* / bbx_dag_* / bbx_mlp_* in include/bbts_b200.h).

Tensors are addressed by tid like in BarbaTOS; metas are the reference's
260-byte tensor_meta_t (int32 format id + 256-byte blob). Commands are queued
with the reference's APPLY / REDUCE / DELETE semantics and run either on the
per-op path (reservation station, one launch per command) or compiled into a
grouped, graph-captured DAG.
"""
import ctypes as C
import struct

import numpy as np

from ._lib import lib, check

META_BYTES = 260
HEURISTIC, LEARNED = 0, 1
# build_dag tile_n: AUTOTUNE times every candidate tile per group; LEARNED_TILES
# asks the runtime's tile model (set_tile_predictor); 0 = size heuristic
AUTOTUNE, LEARNED_TILES = -1, -2
_NP_OF_FMT = {"dense": np.float32, "ffnn_dense": np.float32, "cutensor": np.float32, "labels": np.int32}


def dense_meta(fmt_id, rows, cols, scale=1.0):
    b = bytearray(META_BYTES)
    struct.pack_into("<iIIf", b, 0, fmt_id, rows, cols, scale)
    return bytes(b)


def ffnn_meta(fmt_id, rows, cols, has_bias):
    b = bytearray(META_BYTES)
    struct.pack_into("<iII?", b, 0, fmt_id, rows, cols, bool(has_bias))
    return bytes(b)


def cutensor_meta(fmt_id, dims):
    b = bytearray(META_BYTES)
    struct.pack_into("<iI", b, 0, fmt_id, len(dims))
    for i, d in enumerate(dims):
        struct.pack_into("<q", b, 4 + 8 + 8 * i, int(d))
    return bytes(b)


def parse_meta(meta):
    fmt_id, rows, cols, scale = struct.unpack_from("<iIIf", meta, 0)
    return {"fmt_id": fmt_id, "rows": rows, "cols": cols, "scale": scale}


def params_words(params):
    """Encodes a parameter list as the raw 4-byte command_param_t words:
    Python float -> f, bool -> b, int -> i."""
    words = []
    for p in params:
        if isinstance(p, bool):
            words.append(int(p))
        elif isinstance(p, float):
            words.append(struct.unpack("<I", struct.pack("<f", p))[0])
        else:
            words.append(int(p) & 0xFFFFFFFF)
    return words


class Runtime:
    def __init__(self):
        self.h = C.c_void_p()
        check(lib.bbx_rt_create(C.byref(self.h)))
        s = C.c_void_p()
        check(lib.bbx_rt_stream(self.h, C.byref(s)))
        self.stream = s
        self._next_cmd = 0

    # ------------------------------------------------------------- registry
    def fmt(self, name):
        v = lib.bbx_rt_fmt_id(self.h, name.encode())
        if v < 0:
            raise KeyError(name)
        return v

    def impl(self, ud_name, in_types, out_types, gpu=True):
        u, i = C.c_int(), C.c_int()
        check(lib.bbx_rt_find_impl(self.h, ud_name.encode(), ",".join(in_types).encode(),
                                   ",".join(out_types).encode(), int(gpu), C.byref(u), C.byref(i)))
        return (u.value, i.value)

    def impl_named(self, ud_name, impl_name, in_types=("cutensor", "cutensor"), out_types=("cutensor",)):
        """The impl of `ud_name` whose impl_name matches (several impls can share types)."""
        ud, _ = self.impl(ud_name, list(in_types), list(out_types))
        buf = C.create_string_buffer(256)
        for i in range(64):
            if lib.bbx_rt_impl_name(self.h, ud, i, buf, 256) != 0:
                break
            if buf.value.decode() == impl_name:
                return (ud, i)
        raise KeyError(impl_name)

    def impl_name(self, impl):
        buf = C.create_string_buffer(256)
        check(lib.bbx_rt_impl_name(self.h, impl[0], impl[1], buf, 256))
        return buf.value.decode()

    # ------------------------------------------------------------- tensors
    def put(self, tid, meta, data=None, device_ptr=None, nbytes=None):
        if device_ptr is not None:
            check(lib.bbx_rt_tensor_put(self.h, tid, meta, C.c_void_p(device_ptr), nbytes, 1))
        elif data is not None:
            arr = np.ascontiguousarray(data)
            check(lib.bbx_rt_tensor_put(self.h, tid, meta, arr.ctypes.data, arr.nbytes, 0))
        else:
            check(lib.bbx_rt_tensor_put(self.h, tid, meta, None, 0, 0))

    def put_dense(self, tid, arr, fmt="dense"):
        arr = np.ascontiguousarray(arr, dtype=np.float32)
        self.put(tid, dense_meta(self.fmt(fmt), arr.shape[0], arr.shape[1]), arr)

    def fill_philox(self, tid, seed, dist=0, a=0.0, b=1.0):
        """Fills tensor `tid`'s payload on the device with the seeded Philox
        generator: dist 0 = U(a, b), 1 = N(a, b^2), in the block's element type
        (f32 unless the format is dense_bf16)."""
        ptr, nbytes = self.payload(tid)
        fmt_id = struct.unpack_from("<i", self.meta(tid), 0)[0]
        bf16 = fmt_id == self.fmt("dense_bf16")
        check(lib.bbx_fill_philox(1 if bf16 else 0, ptr, nbytes // (2 if bf16 else 4), int(seed), int(dist),
                                  float(a), float(b), self.stream))

    def meta(self, tid):
        m = C.create_string_buffer(META_BYTES)
        check(lib.bbx_rt_tensor_get(self.h, tid, m, None, 0, 0))
        return m.raw

    def payload(self, tid):
        p, n = C.c_void_p(), C.c_size_t()
        check(lib.bbx_rt_tensor_payload(self.h, tid, C.byref(p), C.byref(n)))
        return p.value, n.value

    def get_bytes(self, tid):
        _, n = self.payload(tid)
        buf = np.empty(n, np.uint8)
        check(lib.bbx_rt_tensor_get(self.h, tid, None, buf.ctypes.data, n, 0))
        return buf

    def get_dense(self, tid):
        m = parse_meta(self.meta(tid))
        raw = self.get_bytes(tid)
        return raw.view(np.float32).reshape(m["rows"], m["cols"])

    def count(self):
        return lib.bbx_rt_tensor_count(self.h)

    def remove(self, tid):
        check(lib.bbx_rt_tensor_remove(self.h, tid))

    # ------------------------------------------------------------- commands
    def _cid(self, cmd_id):
        if cmd_id is None:
            cmd_id = self._next_cmd
        self._next_cmd = cmd_id + 1
        return cmd_id

    def apply(self, impl, inputs, outputs, params=(), cmd_id=None):
        w = params_words(params)
        pw = (C.c_uint32 * max(1, len(w)))(*w)
        ins = (C.c_int * max(1, len(inputs)))(*inputs)
        outs = (C.c_int * len(outputs))(*outputs)
        check(lib.bbx_rt_queue_apply(self.h, self._cid(cmd_id), impl[0], impl[1], pw, len(w), ins, len(inputs),
                                     outs, len(outputs)))

    def reduce(self, impl, inputs, output, params=(), cmd_id=None):
        w = params_words(params)
        pw = (C.c_uint32 * max(1, len(w)))(*w)
        ins = (C.c_int * len(inputs))(*inputs)
        check(lib.bbx_rt_queue_reduce(self.h, self._cid(cmd_id), impl[0], impl[1], pw, len(w), ins, len(inputs),
                                      output))

    def delete(self, tids, cmd_id=None):
        arr = (C.c_int * len(tids))(*tids)
        check(lib.bbx_rt_queue_delete(self.h, self._cid(cmd_id), arr, len(tids)))

    def clear_commands(self):
        check(lib.bbx_rt_clear_commands(self.h))
        self._next_cmd = 0

    def num_commands(self):
        return lib.bbx_rt_num_commands(self.h)

    def load_program(self, path):
        """Appends a .sbbts (text) or .bbts (binary) program compiled for this node."""
        n = C.c_int()
        fn = lib.bbx_rt_load_sbbts if path.endswith(".sbbts") else lib.bbx_rt_load_bbts
        check(fn(self.h, path.encode(), C.byref(n)))
        self._next_cmd += n.value  # the loader numbers them after the last queued command
        return n.value

    def save_bbts(self, path):
        check(lib.bbx_rt_save_bbts(self.h, path.encode()))

    def run(self, policy=HEURISTIC):
        check(lib.bbx_rt_run(self.h, policy))

    def record(self, policy=HEURISTIC, cap=1 << 20, with_hints=False):
        """Runs the list on one stream, timing every command: (features [n, 12],
        latency us [n]) and, with_hints, the uds' complexity hints [n]."""
        n = self.num_commands()
        cap = max(1, min(cap, n))
        feats = np.empty((cap, 12), np.float32)
        lat = np.empty(cap, np.float32)
        hints = np.empty(cap, np.float64)
        got = C.c_int()
        check(lib.bbx_rt_record(self.h, policy, feats.ctypes.data, lat.ctypes.data, hints.ctypes.data, cap,
                                C.byref(got)))
        k = min(cap, got.value)
        if with_hints:
            return feats[:k].copy(), lat[:k].copy(), hints[:k].copy()
        return feats[:k].copy(), lat[:k].copy()

    def set_workers(self, n):
        """Worker streams of the per-op path (1 = the plain single-stream path)."""
        check(lib.bbx_rt_set_workers(self.h, int(n)))

    SPILL_FIELDS = ("evictions", "reloads", "d2h_bytes", "h2d_bytes", "file_write_bytes", "file_read_bytes",
                    "clean_evictions", "resident_bytes", "peak_resident_bytes", "host_bytes")

    def set_storage_budget(self, device_bytes, host_bytes=1 << 62, spill_file=None):
        """Keep resident block payloads within `device_bytes` by spilling the
        least recently used blocks to pinned host memory (up to `host_bytes`)
        and then to `spill_file`. 0 removes the budget."""
        check(lib.bbx_rt_set_storage_budget(self.h, int(device_bytes), int(host_bytes),
                                            spill_file.encode() if spill_file else None))

    def spill_stats(self):
        out = (C.c_ulonglong * 10)()
        check(lib.bbx_rt_spill_stats(self.h, out, 10))
        return dict(zip(self.SPILL_FIELDS, [int(x) for x in out]))

    def set_hint_predictor(self, a, b):
        """Predicted latency exp(a ln(hint) + b) us from the uds' complexity hints."""
        check(lib.bbx_rt_set_hint_predictor(self.h, float(a), float(b)))
        self._predictor = None

    def set_predictor(self, mlp):
        """The runtime calls into `mlp` whenever it schedules, so it holds a
        reference: a temporary passed here stays alive as long as the runtime."""
        check(lib.bbx_rt_set_predictor(self.h, mlp.h if mlp is not None else None))
        self._predictor = mlp

    def set_tile_predictor(self, mlp):
        """An MLP trained on tile samples (tile_samples) becomes the tile model
        of build_dag(tile_n=LEARNED_TILES); the runtime keeps a reference."""
        check(lib.bbx_rt_set_tile_predictor(self.h, mlp.h if mlp is not None else None))
        self._tile_predictor = mlp

    def set_dag_stream_kernel(self, kernel):
        """Streaming kernel of DAGs built afterwards: 0 = bulk-staged where
        aligned (default), 1 = the register kernel (shares SMs with tensor-core
        launches), 2 = chosen per wave from predicted tensor / streaming times."""
        check(lib.bbx_rt_set_dag_stream_kernel(self.h, int(kernel)))

    def build_dag(self, policy=HEURISTIC, tile_n=0):
        return Dag(self, policy, tile_n)

    def close(self):
        if self.h:
            lib.bbx_rt_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tile_record(on):
    """Record the DAG autotuner's timings as tile samples (on clears them)."""
    check(lib.bbx_tile_record(int(bool(on))))


def tile_samples():
    """(features n x 12 float32, us per launch n) recorded by the autotuner."""
    n = C.c_int()
    check(lib.bbx_tile_samples(None, None, 0, C.byref(n)))
    cap = n.value
    f = np.empty((cap, 12), np.float32)
    t = np.empty(cap, np.float32)
    check(lib.bbx_tile_samples(f.ctypes.data, t.ctypes.data, cap, C.byref(n)))
    k = min(cap, n.value)
    return f[:k].copy(), t[:k].copy()


class Dag:
    def __init__(self, rt, policy, tile_n):
        self.rt = rt
        self.h = C.c_void_p()
        check(lib.bbx_dag_build(rt.h, policy, tile_n, C.byref(self.h)))

    def launch(self, stream=None):
        check(lib.bbx_dag_launch(self.h, stream if stream is not None else self.rt.stream))

    def stats(self):
        fl, by = C.c_double(), C.c_double()
        w, t, s, o = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        ar = C.c_size_t()
        check(lib.bbx_dag_stats(self.h, C.byref(fl), C.byref(by), C.byref(w), C.byref(t), C.byref(s), C.byref(o),
                                C.byref(ar)))
        return {"flops": fl.value, "bytes": by.value, "waves": w.value, "tc_launches": t.value,
                "stream_launches": s.value, "other_launches": o.value, "arena_bytes": ar.value}

    GROUP_KINDS = ("gather_in", "stream", "impl", "tc_gemm", "gather_out")

    def profile(self, stream=None):
        """Each launch group replayed on its own: a list of dicts with kind,
        wave, ms, flops and bytes (the algorithmic work of the launch)."""
        st = stream if stream is not None else self.rt.stream
        n = C.c_int()
        check(lib.bbx_dag_profile(self.h, st, 0, None, None, None, None, None, C.byref(n)))
        cap = n.value
        kinds = np.empty(cap, np.int32)
        waves = np.empty(cap, np.int32)
        ms = np.empty(cap, np.float32)
        fl = np.empty(cap, np.float64)
        by = np.empty(cap, np.float64)
        check(lib.bbx_dag_profile(self.h, st, cap, kinds.ctypes.data, waves.ctypes.data, ms.ctypes.data,
                                  fl.ctypes.data, by.ctypes.data, C.byref(n)))
        return [{"kind": self.GROUP_KINDS[k], "wave": int(w), "ms": float(m), "flops": float(f), "bytes": float(b)}
                for k, w, m, f, b in zip(kinds, waves, ms, fl, by)]

    def tensor(self, tid):
        p = C.c_void_p()
        m = C.create_string_buffer(META_BYTES)
        check(lib.bbx_dag_tensor(self.h, tid, C.byref(p), m))
        return p.value, m.raw

    def read_bytes(self, tid, nbytes):
        buf = np.empty(nbytes, np.uint8)
        check(lib.bbx_dag_read(self.h, tid, buf.ctypes.data, nbytes))
        return buf

    def write(self, tid, src_ptr, nbytes, on_device=False, stream=None):
        """Enqueues a copy of `nbytes` at address `src_ptr` (host, or device
        with on_device) into input block `tid` on `stream` (default: the
        runtime's). Pinned host memory makes it asynchronous."""
        check(lib.bbx_dag_write(self.h, tid, C.c_void_p(src_ptr), nbytes, int(on_device),
                                stream if stream is not None else self.rt.stream))

    def fetch(self, tid, dst_ptr, cap, on_device=False, stream=None):
        """Enqueues a copy of up to `cap` payload bytes of `tid` to `dst_ptr`."""
        check(lib.bbx_dag_fetch(self.h, tid, C.c_void_p(dst_ptr), cap, int(on_device),
                                stream if stream is not None else self.rt.stream))

    def register_waves(self):
        """Waves whose streaming launches run the register kernel."""
        n = lib.bbx_dag_register_waves(self.h)
        if n < 0:
            check(n)
        return n

    def group_tiles(self):
        """Tile of each launch group, in profile order (0 for non-tensor-core groups)."""
        n = C.c_int()
        check(lib.bbx_dag_group_tiles(self.h, 0, None, C.byref(n)))
        out = (C.c_int * max(1, n.value))()
        check(lib.bbx_dag_group_tiles(self.h, n.value, out, C.byref(n)))
        return [int(x) for x in out[:n.value]]

    def close(self):
        if self.h:
            lib.bbx_dag_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mlp:
    """The learned cost model (12 -> 128 -> 128 -> 128 -> 1, ReLU, FP32) on the GPU."""

    def __init__(self, seed=0):
        self.h = C.c_void_p()
        check(lib.bbx_mlp_create(seed, C.byref(self.h)))

    @staticmethod
    def num_params():
        return lib.bbx_mlp_num_params()

    def set_norm(self, mean, std):
        mean = np.ascontiguousarray(mean, np.float32)
        std = np.ascontiguousarray(std, np.float32)
        check(lib.bbx_mlp_set_norm(self.h, mean.ctypes.data, std.ctypes.data))

    def train(self, x, y, epochs=20, batch=512, lr=1e-3):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = C.c_float()
        check(lib.bbx_mlp_train(self.h, x.ctypes.data, y.ctypes.data, len(y), epochs, batch, lr, C.byref(loss)))
        return loss.value

    def predict(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.empty(len(x), np.float32)
        check(lib.bbx_mlp_predict(self.h, x.ctypes.data, len(x), y.ctypes.data))
        return y

    def loss_grad(self, x, y):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = C.c_float()
        g = np.empty(self.num_params(), np.float32)
        check(lib.bbx_mlp_loss_grad(self.h, x.ctypes.data, y.ctypes.data, len(y), C.byref(loss), g.ctypes.data))
        return loss.value, g

    def get_params(self):
        p = np.empty(self.num_params(), np.float32)
        check(lib.bbx_mlp_get_params(self.h, p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        check(lib.bbx_mlp_set_params(self.h, p.ctypes.data))

    def close(self):
        if self.h:
            lib.bbx_mlp_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
