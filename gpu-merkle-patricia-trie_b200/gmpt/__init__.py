"""Python binding of the B200 MPT library through its C ABI (include/gmpt.h).

``MPT`` mirrors the reference's ``GpuMPT::Compress::MPT`` surface
(mpt-with-compress/include/mpt/gpu_mpt.cuh:18-192) for the batched update
path: ``puts_2phase_with_valuehp`` (PhaseNU), ``puts_latching_with_valuehp_v2``
(LockNU), ``hash_onepass_v2`` (PhaseHC), ``gets_parallel`` and
``get_root_hash``.  Every call goes through ``libgmpt_b200.so``; there is no
other implementation behind it, so a missing or unloadable library raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent.parent
LIB_PATH = PKG_DIR / "lib" / "libgmpt_b200.so"

MODE_REF = 0
MODE_GETH = 1

STATUS = {0: "ok", 1: "cuda error", 2: "bad key", 3: "capacity", 4: "retry limit", 5: "bad argument",
          6: "internal"}

# every symbol include/gmpt.h and include/libgmpt.h declare
EXPORTS = [
    "gmpt_version", "gmpt_create", "gmpt_destroy", "gmpt_reset", "gmpt_puts_2phase", "gmpt_puts_latching",
    "gmpt_puts_2phase_device", "gmpt_puts_latching_device", "gmpt_hash_onepass", "gmpt_pending_targets",
    "gmpt_get_root_hash", "gmpt_gets_parallel", "gmpt_get_values", "gmpt_get_stats", "gmpt_set_timing",
    "gmpt_last_error", "gmpt_last_error_message", "gmpt_free_buffer", "gmpt_stream",
    "gmpt_keccak256_batch", "gmpt_keccak256_batch_device", "gmpt_keccak_peak", "gmpt_launch_count",
    "gmpt_keccak256_batch_noalloc", "gmpt_set_option",
    "gmpt_create_forest", "gmpt_max_tries", "gmpt_puts_2phase_forest", "gmpt_puts_latching_forest",
    "gmpt_get_roots", "gmpt_gets_forest", "gmpt_block_update", "gmpt_block_update_device", "gmpt_block_info",
    "gmpt_block_times", "gmpt_reserve", "gmpt_block_timeline", "gmpt_reserve_block",
    "gmpt_reserve_nodes", "gmpt_batch_features_device", "gmpt_puts_pipeline",
    "gmpt_puts_raw", "gmpt_puts_raw_device", "gmpt_puts_pipeline_raw",
    "gmpt_puts_latching_with_read", "gmpt_puts_2phase_with_read", "gmpt_puts_with_read_forest",
    "gmpt_puts_with_read_device", "gmpt_deletes", "gmpt_deletes_device",
    "gmpt_mlp_create", "gmpt_mlp_destroy", "gmpt_mlp_num_params", "gmpt_mlp_get_params", "gmpt_mlp_set_params",
    "gmpt_mlp_forward", "gmpt_mlp_loss_grad", "gmpt_mlp_train",
    "gmpt_puts_forest_device", "gmpt_gets_forest_device", "gmpt_gen_ids", "gmpt_gen_keys", "gmpt_gen_values",
    "gmpt_schedule_count", "gmpt_schedule_name", "gmpt_schedule_info", "gmpt_puts_schedule",
    "gmpt_puts_schedule_device", "gmpt_batch_features", "gmpt_batch_features_trie_device", "gmpt_selector_create",
    "gmpt_selector_destroy", "gmpt_selector_choose", "gmpt_selector_counts", "gmpt_puts_auto",
    "gmpt_puts_auto_device", "gmpt_gets_device", "gmpt_flush_dirty", "gmpt_create_ex",
    "preprocess", "build_mpt_2phase", "build_mpt_olc", "get_all_nodes", "init_mpt", "insert_mpt_2phase",
    "insert_mpt_olc", "free_mpt",
]


class GmptError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Stats(C.Structure):
    _fields_ = ([(n, C.c_uint64) for n in (
        "n_full", "n_short", "n_value", "n_records", "key_bytes", "value_bytes", "last_unique", "last_new",
        "last_pseudo", "last_dirty", "last_levels", "last_hash_levels", "device_bytes")]
        + [("sort_passes", C.c_uint32), ("build_levels", C.c_uint32)]
        + [(n, C.c_float) for n in ("t_stage_ms", "t_sort_ms", "t_walk_ms", "t_build_ms", "t_hash_ms")]
        + [(n, C.c_uint64) for n in ("last_hashed", "last_enc_bytes", "last_keccak_blocks")]
        + [("t_hash_kernels_ms", C.c_float), ("hash_launches", C.c_uint32), ("pad", C.c_uint32)])

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class NodeSet(C.Structure):
    _fields_ = [("hashs", C.c_void_p), ("encs", C.c_void_p), ("encs_indexs", C.c_void_p), ("num", C.c_ulonglong)]


def build(quiet: bool = True) -> Path:
    """Compile libgmpt_b200.so for sm_100a (nvcc; no GPU needed)."""
    r = subprocess.run(["make", "-C", str(PKG_DIR)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("libgmpt_b200 build failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])
    return LIB_PATH


_lib = None


def lib():
    """Load libgmpt_b200.so (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FileNotFoundError(f"{LIB_PATH} is not built; run gmpt.build() / make")
    L = C.CDLL(str(LIB_PATH))
    vp, i32, i64 = C.c_void_p, C.c_int, C.c_int64
    L.gmpt_version.restype = i32
    L.gmpt_create.restype = vp
    L.gmpt_create.argtypes = [i32, i32]
    L.gmpt_create_forest.restype = vp
    L.gmpt_create_forest.argtypes = [i32, i32, i32]
    L.gmpt_create_ex.restype = vp
    L.gmpt_create_ex.argtypes = [i32, i32, i32, C.c_uint]
    L.gmpt_max_tries.argtypes = [vp]
    for f in ("gmpt_puts_2phase_forest", "gmpt_puts_latching_forest"):
        getattr(L, f).argtypes = [vp, vp, vp, vp, vp, vp, vp, i32]
        getattr(L, f).restype = i32
    L.gmpt_get_roots.argtypes = [vp, vp, i32, vp, vp]
    L.gmpt_gets_forest.argtypes = [vp, vp, vp, vp, i32, vp, vp]
    L.gmpt_block_update.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i32, i32, vp, i32, vp, vp]
    L.gmpt_block_update.restype = i32
    L.gmpt_block_update_device.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i32, i32, i64, i64, vp, i32, vp, vp]
    L.gmpt_block_update_device.restype = i32
    L.gmpt_block_info.argtypes = [vp, vp]
    L.gmpt_block_times.argtypes = [vp, vp]
    L.gmpt_block_timeline.argtypes = [vp, vp, i32, vp]
    L.gmpt_reserve.argtypes = [vp, i64, i64, i64]
    L.gmpt_reserve_block.argtypes = [vp, i64, i64, i64, i64]
    L.gmpt_reserve_nodes.argtypes = [vp, i64, i64, i64, i64, i64, i64]
    L.gmpt_mlp_create.restype = vp
    L.gmpt_mlp_create.argtypes = [i32, i32, i32, i32, C.c_uint64]
    L.gmpt_mlp_destroy.argtypes = [vp]
    L.gmpt_mlp_num_params.argtypes = [vp]
    L.gmpt_mlp_get_params.argtypes = [vp, vp]
    L.gmpt_mlp_set_params.argtypes = [vp, vp]
    L.gmpt_mlp_forward.argtypes = [vp, vp, i32, vp]
    L.gmpt_mlp_loss_grad.argtypes = [vp, vp, vp, vp, i32, vp, vp]
    L.gmpt_mlp_train.argtypes = [vp, vp, vp, vp, i32, i32, i32, C.c_float, C.c_uint64, vp]
    L.gmpt_puts_forest_device.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, i32, i64, i64]
    L.gmpt_gets_forest_device.argtypes = [vp, vp, vp, vp, i32, i64, vp, vp]
    L.gmpt_gen_ids.argtypes = [C.c_uint64, i64, i64, i64, C.c_double, C.c_double, vp, vp, vp]
    L.gmpt_gen_keys.argtypes = [C.c_uint64, vp, i64, i32, vp, vp, vp]
    L.gmpt_gen_values.argtypes = [C.c_uint64, i64, i32, vp, vp, vp]
    L.gmpt_batch_features_device.argtypes = [vp, vp, i32, i64, vp, vp]
    L.gmpt_puts_pipeline.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.gmpt_puts_pipeline_raw.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.gmpt_puts_raw.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, i32]
    for f in ("gmpt_puts_latching_with_read", "gmpt_puts_2phase_with_read"):
        getattr(L, f).argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i32, vp, vp]
    L.gmpt_deletes.argtypes = [vp, vp, vp, vp, i32]
    L.gmpt_deletes_device.argtypes = [vp, vp, vp, vp, i32, i64]
    L.gmpt_puts_with_read_forest.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp]
    L.gmpt_puts_with_read_device.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, i32, i64, i64, vp, vp, vp]
    L.gmpt_puts_raw_device.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, i32, i64, i64]
    L.gmpt_destroy.argtypes = [vp]
    L.gmpt_reset.argtypes = [vp]
    for f in ("gmpt_puts_2phase", "gmpt_puts_latching"):
        getattr(L, f).argtypes = [vp, vp, vp, vp, vp, vp, i32]
        getattr(L, f).restype = i32
    for f in ("gmpt_puts_2phase_device", "gmpt_puts_latching_device"):
        getattr(L, f).argtypes = [vp, vp, vp, vp, vp, vp, i32, i64, i64]
        getattr(L, f).restype = i32
    L.gmpt_hash_onepass.argtypes = [vp]
    L.gmpt_pending_targets.argtypes = [vp, vp, vp]
    L.gmpt_get_root_hash.argtypes = [vp, vp, vp]
    L.gmpt_gets_parallel.argtypes = [vp, vp, vp, i32, vp, vp]
    L.gmpt_get_values.argtypes = [vp, vp, vp, i32, vp, i64, vp, vp]
    L.gmpt_get_stats.argtypes = [vp, vp]
    L.gmpt_set_timing.argtypes = [vp, i32]
    L.gmpt_set_option.argtypes = [vp, C.c_char_p, i64]
    L.gmpt_last_error_message.restype = C.c_char_p
    L.gmpt_stream.restype = vp
    L.gmpt_stream.argtypes = [vp]
    L.gmpt_free_buffer.argtypes = [vp]
    L.gmpt_keccak256_batch.argtypes = [vp, vp, i32, vp]
    L.gmpt_keccak256_batch_device.argtypes = [vp, vp, i32, vp, vp]
    L.gmpt_keccak256_batch_noalloc.argtypes = [vp, vp, i32, vp]
    L.gmpt_keccak256_batch_noalloc.restype = i32
    L.gmpt_keccak_peak.argtypes = [i32, vp]
    L.gmpt_launch_count.restype = C.c_uint64
    L.preprocess.restype = i32
    for f in ("build_mpt_2phase", "build_mpt_olc"):
        getattr(L, f).argtypes = [i32, vp, vp, vp, vp, vp, i32]
        getattr(L, f).restype = vp
    for f in ("insert_mpt_2phase", "insert_mpt_olc"):
        getattr(L, f).argtypes = [vp, vp, vp, vp, vp, vp, i32]
        getattr(L, f).restype = vp
    L.get_all_nodes.argtypes = [i32, vp, vp, i32]
    L.get_all_nodes.restype = NodeSet
    L.init_mpt.restype = vp
    L.free_mpt.argtypes = [vp]
    L.gmpt_schedule_name.restype = C.c_char_p
    L.gmpt_schedule_name.argtypes = [i32]
    L.gmpt_schedule_info.argtypes = [i32, vp]
    L.gmpt_puts_schedule.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, i32]
    L.gmpt_puts_schedule_device.argtypes = [vp, i32, vp, vp, vp, vp, vp, i32, i64, i64]
    L.gmpt_batch_features.argtypes = [vp, vp, vp, vp, vp, i32, vp]
    L.gmpt_batch_features_trie_device.argtypes = [vp, vp, vp, i32, i64, i64, i32, i64, vp]
    L.gmpt_selector_create.restype = vp
    L.gmpt_selector_create.argtypes = [i32, C.c_char_p]
    L.gmpt_selector_destroy.argtypes = [vp]
    L.gmpt_selector_choose.argtypes = [vp, vp, vp, vp]
    L.gmpt_selector_counts.argtypes = [vp, vp]
    L.gmpt_puts_auto.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i32, vp]
    L.gmpt_gets_device.argtypes = [vp, vp, vp, vp, i32, i64, vp, vp]
    L.gmpt_flush_dirty.argtypes = [vp, vp, vp, vp, vp]
    L.gmpt_puts_auto_device.argtypes = [vp, vp, vp, vp, vp, vp, vp, i32, i64, i64, i32, i64, vp]
    _lib = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc: int):
    if rc != 0:
        raise GmptError(rc, lib().gmpt_last_error_message().decode())


def _arrays(keys_hexs, keys_indexs, values=None, values_indexs=None):
    kh = np.ascontiguousarray(keys_hexs, dtype=np.uint8)
    ki = np.ascontiguousarray(keys_indexs, dtype=np.int32)
    vb = None if values is None else np.ascontiguousarray(values, dtype=np.uint8)
    vi = None if values_indexs is None else np.ascontiguousarray(values_indexs, dtype=np.int64)
    return kh, ki, vb, vi


def keccak256_batch(messages) -> list:
    """Keccak-256 of each message (bytes) on the GPU."""
    msgs = [bytes(m) for m in messages]
    data = np.frombuffer(b"".join(msgs) + b"\0", dtype=np.uint8)
    idx = np.zeros(2 * len(msgs), dtype=np.int64)
    pos = 0
    for i, m in enumerate(msgs):
        idx[2 * i], idx[2 * i + 1] = pos, pos + len(m) - 1
        pos += len(m)
    out = np.zeros(32 * max(len(msgs), 1), dtype=np.uint8)
    _check(lib().gmpt_keccak256_batch(_p(data), _p(idx), len(msgs), _p(out)))
    return [out[32 * i: 32 * i + 32].tobytes() for i in range(len(msgs))]


def keccak256_rows(msgs: np.ndarray, chunk: int = 1 << 22) -> np.ndarray:
    """Keccak-256 of every row of a 2-D uint8 array (fixed-length messages)
    on the GPU -> [rows, 32] uint8."""
    msgs = np.ascontiguousarray(msgs, dtype=np.uint8)
    rows, width = msgs.shape
    out = np.empty((rows, 32), dtype=np.uint8)
    for a in range(0, rows, chunk):
        m = msgs[a: a + chunk]
        k = len(m)
        idx = np.empty(2 * k, dtype=np.int64)
        starts = np.arange(k, dtype=np.int64) * width
        idx[0::2] = starts
        idx[1::2] = starts + width - 1
        data = np.concatenate([m.reshape(-1), np.zeros(8, np.uint8)])
        o = np.empty(32 * k, dtype=np.uint8)
        _check(lib().gmpt_keccak256_batch(_p(data), _p(idx), k, _p(o)))
        out[a: a + k] = o.reshape(k, 32)
    return out


def gen_ids(seed: int, n: int, n_existing: int, next_new: int, p_new: float, theta: float, d_ids: int,
            stream: int = 0) -> int:
    """Fill d_ids (device int64[n]); returns how many fresh ids were used."""
    nn = C.c_int64()
    _check(lib().gmpt_gen_ids(int(seed) & ((1 << 64) - 1), int(n), int(n_existing), int(next_new), float(p_new),
                              float(theta), C.c_void_p(d_ids), C.byref(nn), C.c_void_p(stream) if stream else None))
    return nn.value


def gen_keys(seed: int, d_ids: int, n: int, key_bytes: int, d_hexs: int, d_idx: int, stream: int = 0):
    _check(lib().gmpt_gen_keys(int(seed) & ((1 << 64) - 1), C.c_void_p(d_ids), int(n), int(key_bytes),
                               C.c_void_p(d_hexs), C.c_void_p(d_idx), C.c_void_p(stream) if stream else None))


def gen_values(seed: int, n: int, value_bytes: int, d_vals: int, d_idx: int, stream: int = 0):
    _check(lib().gmpt_gen_values(int(seed) & ((1 << 64) - 1), int(n), int(value_bytes), C.c_void_p(d_vals),
                                 C.c_void_p(d_idx), C.c_void_p(stream) if stream else None))


def batch_features_device(d_keys: int, d_kidx: int, n: int, keys_bytes: int, stream: int = 0) -> np.ndarray:
    """[mean key nibbles, their std, repeated-sample share, common-prefix share]
    of a device-resident batch (one kernel over 64 sampled keys)."""
    out = np.zeros(4, dtype=np.float32)
    _check(lib().gmpt_batch_features_device(C.c_void_p(d_keys), C.c_void_p(d_kidx), int(n), int(keys_bytes), _p(out),
                                            C.c_void_p(stream) if stream else None))
    return out


def keccak_peak(device: int = 0) -> float:
    v = C.c_double()
    _check(lib().gmpt_keccak_peak(device, C.byref(v)))
    return v.value


def launch_count() -> int:
    return int(lib().gmpt_launch_count())


class Net:
    """The selector's MLP on the GPU (gmpt_mlp_*): hand-written CUDA forward,
    gradient and Adam training kernels."""

    def __init__(self, n_in: int, n_hidden: int, n_out: int, seed: int = 1, device: int = 0):
        self._L = lib()
        self.dims = (n_in, n_hidden, n_out)
        self._h = self._L.gmpt_mlp_create(device, n_in, n_hidden, n_out, seed)
        if not self._h:
            raise GmptError(self._L.gmpt_last_error(), self._L.gmpt_last_error_message().decode())
        self.n_params = self._L.gmpt_mlp_num_params(self._h)

    def close(self):
        if getattr(self, "_h", None):
            self._L.gmpt_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def params(self) -> np.ndarray:
        p = np.zeros(self.n_params, dtype=np.float32)
        _check(self._L.gmpt_mlp_get_params(self._h, _p(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.n_params
        _check(self._L.gmpt_mlp_set_params(self._h, _p(p)))

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.dims[0])
        y = np.zeros((len(x), self.dims[2]), dtype=np.float32)
        _check(self._L.gmpt_mlp_forward(self._h, _p(x), len(x), _p(y)))
        return y

    def loss_grad(self, x, t, m):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        m = np.ascontiguousarray(m, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        g = np.zeros(self.n_params, dtype=np.float32)
        _check(self._L.gmpt_mlp_loss_grad(self._h, _p(x), _p(t), _p(m), len(x), _p(loss), _p(g)))
        return float(loss[0]), g

    def train(self, x, t, m, epochs: int, batch: int = 64, lr: float = 1e-3, seed: int = 7) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        m = np.ascontiguousarray(m, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        _check(self._L.gmpt_mlp_train(self._h, _p(x), _p(t), _p(m), len(x), int(epochs), int(batch), float(lr),
                                      int(seed), _p(loss)))
        return float(loss[0])


def schedules() -> list:
    """The library's insert schedules: [{name, two_phase, persistent,
    local_build, local_sort, latch_ways, latch_dedup, block_grid,
    warp_full_max}] in index order."""
    L = lib()
    out = []
    keys = ("two_phase", "persistent", "local_build", "local_sort", "latch_ways", "latch_dedup", "block_grid",
            "warp_full_max")
    for k in range(L.gmpt_schedule_count()):
        info = np.zeros(8, np.int32)
        _check(L.gmpt_schedule_info(k, _p(info)))
        d = {"name": L.gmpt_schedule_name(k).decode()}
        d.update({kk: (bool(v) if kk in ("two_phase", "persistent") else int(v)) for kk, v in zip(keys, info)})
        out.append(d)
    return out


class CSelector:
    """The library's schedule selector (rule table + optional network),
    loaded from a file written by gmpt.tuner.Selector.save (None: the
    built-in rule)."""

    def __init__(self, device: int = 0, path: str | None = None):
        self._L = lib()
        self._h = self._L.gmpt_selector_create(device, None if path is None else str(path).encode())
        if not self._h:
            raise GmptError(self._L.gmpt_last_error(), self._L.gmpt_last_error_message().decode())

    def choose(self, features) -> tuple:
        f = np.ascontiguousarray(features, dtype=np.float32)
        k, net = C.c_int(-1), C.c_int(0)
        _check(self._L.gmpt_selector_choose(self._h, _p(f), C.byref(k), C.byref(net)))
        return k.value, bool(net.value)

    def counts(self) -> tuple:
        out = np.zeros(2, np.uint64)
        _check(self._L.gmpt_selector_counts(self._h, _p(out)))
        return int(out[0]), int(out[1])

    def close(self):
        if getattr(self, "_h", None):
            self._L.gmpt_selector_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class MPT:
    """A device-resident trie (GpuMPT::Compress::MPT).

    ``max_tries > 1`` makes a forest of independent tries sharing the node
    pools; the ``*_forest`` methods take a trie id per key and every other
    method addresses trie 0."""

    def __init__(self, device: int = 0, mode: int = MODE_REF, max_tries: int = 1, unified: bool = False):
        self._L = lib()
        self._h = self._L.gmpt_create_ex(device, mode, int(max_tries), 1 if unified else 0)
        if not self._h:
            raise GmptError(self._L.gmpt_last_error(), self._L.gmpt_last_error_message().decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.gmpt_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def reset(self):
        _check(self._L.gmpt_reset(self._h))

    # -- puts --------------------------------------------------------------
    def puts_2phase_with_valuehp(self, keys_hexs, keys_indexs, values, values_indexs, values_hps=None):
        kh, ki, vb, vi = _arrays(keys_hexs, keys_indexs, values, values_indexs)
        hp = None if values_hps is None else np.ascontiguousarray(values_hps, dtype=np.uint64)
        _check(self._L.gmpt_puts_2phase(self._h, _p(kh), _p(ki), _p(vb), _p(vi), _p(hp), len(ki) // 2))

    def puts_latching_with_valuehp_v2(self, keys_hexs, keys_indexs, values, values_indexs, values_hps=None):
        kh, ki, vb, vi = _arrays(keys_hexs, keys_indexs, values, values_indexs)
        hp = None if values_hps is None else np.ascontiguousarray(values_hps, dtype=np.uint64)
        _check(self._L.gmpt_puts_latching(self._h, _p(kh), _p(ki), _p(vb), _p(vi), _p(hp), len(ki) // 2))

    def puts_forest(self, two_phase: bool, keys_hexs, keys_indexs, values, values_indexs, trie_ids,
                    values_hps=None):
        kh, ki, vb, vi = _arrays(keys_hexs, keys_indexs, values, values_indexs)
        hp = None if values_hps is None else np.ascontiguousarray(values_hps, dtype=np.uint64)
        tid = np.ascontiguousarray(trie_ids, dtype=np.int32)
        f = self._L.gmpt_puts_2phase_forest if two_phase else self._L.gmpt_puts_latching_forest
        _check(f(self._h, _p(kh), _p(ki), _p(vb), _p(vi), _p(hp), _p(tid), len(ki) // 2))

    # -- schedules ---------------------------------------------------------
    def puts_schedule(self, k: int, keys_hexs, keys_indexs, values, values_indexs, trie_ids=None):
        """Insert under library schedule k (see schedules())."""
        kh, ki, vb, vi = _arrays(keys_hexs, keys_indexs, values, values_indexs)
        tid = None if trie_ids is None else np.ascontiguousarray(trie_ids, dtype=np.int32)
        _check(self._L.gmpt_puts_schedule(self._h, int(k), _p(kh), _p(ki), _p(vb), _p(vi), None, _p(tid),
                                          len(ki) // 2))

    def puts_schedule_device(self, k: int, d_keys, d_kidx, d_vals, d_vidx, n: int, keys_bytes: int,
                             values_bytes: int, d_tids: int = 0):
        v = lambda a: C.c_void_p(a) if a else None  # noqa: E731
        _check(self._L.gmpt_puts_schedule_device(self._h, int(k), v(d_keys), v(d_kidx), v(d_vals), v(d_vidx),
                                                 v(d_tids), int(n), int(keys_bytes), int(values_bytes)))

    def puts_auto(self, keys_hexs, keys_indexs, values, values_indexs, trie_ids=None, selector=None) -> int:
        """Insert under the schedule the selector (None: the library's own)
        picks; returns the schedule index run."""
        kh, ki, vb, vi = _arrays(keys_hexs, keys_indexs, values, values_indexs)
        tid = None if trie_ids is None else np.ascontiguousarray(trie_ids, dtype=np.int32)
        k = C.c_int(-1)
        _check(self._L.gmpt_puts_auto(self._h, selector._h if selector else None, _p(kh), _p(ki), _p(vb), _p(vi),
                                      None, _p(tid), len(ki) // 2, C.byref(k)))
        return k.value

    def puts_auto_device(self, d_keys, d_kidx, d_vals, d_vidx, n: int, keys_bytes: int, values_bytes: int,
                         d_tids: int = 0, tries_touched: int = 0, trie_keys: int = -1, selector=None) -> int:
        v = lambda a: C.c_void_p(a) if a else None  # noqa: E731
        k = C.c_int(-1)
        _check(self._L.gmpt_puts_auto_device(self._h, selector._h if selector else None, v(d_keys), v(d_kidx),
                                             v(d_vals), v(d_vidx), v(d_tids), int(n), int(keys_bytes),
                                             int(values_bytes), int(tries_touched), int(trie_keys), C.byref(k)))
        return k.value

    def features(self, keys_hexs, keys_indexs, values_indexs, trie_ids=None) -> np.ndarray:
        """The selector's 8 features of a host batch put into this trie."""
        kh, ki, _, vi = _arrays(keys_hexs, keys_indexs, None, values_indexs)
        tid = None if trie_ids is None else np.ascontiguousarray(trie_ids, dtype=np.int32)
        out = np.zeros(8, np.float32)
        _check(self._L.gmpt_batch_features(self._h, _p(kh), _p(ki), _p(vi), _p(tid), len(ki) // 2, _p(out)))
        return out

    def features_device(self, d_keys, d_kidx, n: int, keys_bytes: int, values_bytes: int,
                        tries_touched: int = 0, trie_keys: int = -1) -> np.ndarray:
        out = np.zeros(8, np.float32)
        _check(self._L.gmpt_batch_features_trie_device(self._h, C.c_void_p(d_keys), C.c_void_p(d_kidx), int(n),
                                                       int(keys_bytes), int(values_bytes), int(tries_touched),
                                                       int(trie_keys), _p(out)))
        return out

    def deletes(self, keys_hexs, keys_indexs, trie_ids=None):
        """Remove keys (absent keys are ignored); hash_onepass_v2 afterwards."""
        kh, ki, _, _ = _arrays(keys_hexs, keys_indexs)
        tid = None if trie_ids is None else np.ascontiguousarray(trie_ids, dtype=np.int32)
        _check(self._L.gmpt_deletes(self._h, _p(kh), _p(ki), _p(tid), len(ki) // 2))

    def deletes_device(self, d_keys, d_kidx, n: int, keys_bytes: int, d_tids: int = 0):
        v = lambda a: C.c_void_p(a) if a else None  # noqa: E731
        _check(self._L.gmpt_deletes_device(self._h, v(d_keys), v(d_kidx), v(d_tids), int(n), int(keys_bytes)))

    def puts_with_read(self, two_phase: bool, keys_hexs, keys_indexs, rw_flags, values, values_indexs,
                       trie_ids=None, values_hps=None):
        """Mixed batch (rw_flags[i] 0 = read, 1 = write), applied as if in
        index order; returns (hps, sizes) of the reads in read order."""
        kh, ki, vb, vi = _arrays(keys_hexs, keys_indexs, values, values_indexs)
        n = len(ki) // 2
        rw = np.ascontiguousarray(rw_flags, dtype=np.uint8)
        hp = None if values_hps is None else np.ascontiguousarray(values_hps, dtype=np.uint64)
        tid = None if trie_ids is None else np.ascontiguousarray(trie_ids, dtype=np.int32)
        out_hp = np.zeros(max(n, 1), dtype=np.uint64)
        out_len = np.zeros(max(n, 1), dtype=np.int32)
        cnt = C.c_int(0)
        _check(self._L.gmpt_puts_with_read_forest(self._h, 1 if two_phase else 0, _p(kh), _p(ki), _p(rw), _p(vb),
                                                  _p(vi), _p(hp), _p(tid), n, _p(out_hp), _p(out_len),
                                                  C.byref(cnt)))
        return out_hp[:cnt.value], out_len[:cnt.value]

    def puts_with_read_device(self, two_phase: bool, d_keys, d_kidx, d_rw, d_vals, d_vidx, n: int, keys_bytes: int,
                              values_bytes: int, d_out_hp, d_out_len, d_tids: int = 0) -> int:
        """Mixed batch from device memory; results into device arrays; returns the read count."""
        v = lambda a: C.c_void_p(a) if a else None  # noqa: E731
        cnt = C.c_int(0)
        _check(self._L.gmpt_puts_with_read_device(self._h, 1 if two_phase else 0, v(d_keys), v(d_kidx), v(d_rw),
                                                  v(d_vals), v(d_vidx), None, v(d_tids), int(n), int(keys_bytes),
                                                  int(values_bytes), v(d_out_hp), v(d_out_len), C.byref(cnt)))
        return cnt.value

    def get_roots(self, trie_ids=None, n: int | None = None) -> list:
        """Root bytes of each trie in trie_ids (default: tries 0..n-1)."""
        ids = None if trie_ids is None else np.ascontiguousarray(trie_ids, dtype=np.int32)
        cnt = len(ids) if ids is not None else int(n)
        out = np.zeros(32 * max(cnt, 1), dtype=np.uint8)
        sizes = np.zeros(max(cnt, 1), dtype=np.int32)
        _check(self._L.gmpt_get_roots(self._h, _p(ids), cnt, _p(out), _p(sizes)))
        return [out[32 * i: 32 * i + sizes[i]].tobytes() for i in range(cnt)]

    def gets_forest(self, keys_hexs, keys_indexs, trie_ids):
        kh, ki, _, _ = _arrays(keys_hexs, keys_indexs)
        n = len(ki) // 2
        tid = np.ascontiguousarray(trie_ids, dtype=np.int32)
        hps = np.zeros(n, dtype=np.uint64)
        sizes = np.zeros(n, dtype=np.int32)
        _check(self._L.gmpt_gets_forest(self._h, _p(kh), _p(ki), _p(tid), n, _p(hps), _p(sizes)))
        return hps, sizes

    def block_update(self, keys_hexs, keys_indexs, values, values_indexs, trie_ids, n0: int, out_ids,
                     patch_trie=None, patch_off=None) -> list:
        """One persistent launch: stage 0 = keys [0, n0), stage 1 = the rest
        (values patched with stage-0 roots); returns the roots of out_ids."""
        kh, ki, vb, vi = _arrays(keys_hexs, keys_indexs, values, values_indexs)
        tid = np.ascontiguousarray(trie_ids, dtype=np.int32)
        pt = None if patch_trie is None else np.ascontiguousarray(patch_trie, dtype=np.int32)
        po = None if patch_off is None else np.ascontiguousarray(patch_off, dtype=np.int32)
        oid = np.ascontiguousarray(out_ids, dtype=np.int32)
        out = np.zeros(32 * max(len(oid), 1), dtype=np.uint8)
        sizes = np.zeros(max(len(oid), 1), dtype=np.int32)
        _check(self._L.gmpt_block_update(self._h, _p(kh), _p(ki), _p(vb), _p(vi), _p(tid), _p(pt), _p(po),
                                         len(ki) // 2, int(n0), _p(oid), len(oid), _p(out), _p(sizes)))
        return [out[32 * i: 32 * i + sizes[i]].tobytes() for i in range(len(oid))]

    def block_update_device(self, d_keys, d_kidx, d_vals, d_vidx, d_tid, d_ptrie, d_poff, n: int, n0: int,
                            keys_bytes: int, values_bytes: int, out_ids, out=None, sizes=None) -> list:
        """block_update with device-resident inputs (raw addresses; d_ptrie / d_poff may be 0)."""
        oid = np.ascontiguousarray(out_ids, dtype=np.int32)
        if out is None:
            out = np.zeros(32 * max(len(oid), 1), dtype=np.uint8)
        if sizes is None:
            sizes = np.zeros(max(len(oid), 1), dtype=np.int32)
        v = lambda a: C.c_void_p(a) if a else None  # noqa: E731
        _check(self._L.gmpt_block_update_device(self._h, v(d_keys), v(d_kidx), v(d_vals), v(d_vidx), v(d_tid),
                                                v(d_ptrie), v(d_poff), int(n), int(n0), int(keys_bytes),
                                                int(values_bytes), _p(oid), len(oid), _p(out), _p(sizes)))
        return [out[32 * i: 32 * i + sizes[i]].tobytes() for i in range(len(oid))]

    def block_info(self) -> dict:
        a = np.zeros(8, dtype=np.uint32)
        _check(self._L.gmpt_block_info(self._h, _p(a)))
        tm = np.zeros(3, dtype=np.float32)
        _check(self._L.gmpt_block_times(self._h, _p(tm)))
        return {"levels": (int(a[0]), int(a[1])), "dirty": (int(a[2]), int(a[3])), "grid": int(a[4]),
                "captures": int(a[5]), "launches": int(a[6]), "t_inputs_ms": float(tm[0]),
                "t_launch_ms": float(tm[1]), "t_total_ms": float(tm[2])}

    def block_timeline(self) -> np.ndarray:
        """Device timestamps (ns) of the last block's phases, relative to its start."""
        a = np.zeros(64, dtype=np.uint64)
        n = C.c_int()
        _check(self._L.gmpt_block_timeline(self._h, _p(a), 64, C.byref(n)))
        a = a[: n.value].astype(np.int64)
        return a - a[0] if len(a) else a

    def reserve_block(self, max_keys: int, max_key_bytes: int, max_value_bytes: int, max_out: int):
        _check(self._L.gmpt_reserve_block(self._h, int(max_keys), int(max_key_bytes), int(max_value_bytes),
                                          int(max_out)))

    def reserve_nodes(self, full: int, shorts: int, values: int, records: int, key_bytes: int, value_bytes: int):
        _check(self._L.gmpt_reserve_nodes(self._h, int(full), int(shorts), int(values), int(records), int(key_bytes),
                                          int(value_bytes)))

    def reserve(self, n_keys: int, key_bytes: int, value_bytes: int):
        _check(self._L.gmpt_reserve(self._h, int(n_keys), int(key_bytes), int(value_bytes)))

    def puts_forest_device(self, two_phase: bool, d_keys, d_kidx, d_vals, d_vidx, d_tids, n: int, keys_bytes: int,
                           values_bytes: int):
        v = lambda a: C.c_void_p(a) if a else None  # noqa: E731
        _check(self._L.gmpt_puts_forest_device(self._h, 1 if two_phase else 0, v(d_keys), v(d_kidx), v(d_vals),
                                               v(d_vidx), None, v(d_tids), int(n), int(keys_bytes),
                                               int(values_bytes)))

    def gets_forest_device(self, d_keys, d_kidx, d_tids, n: int, keys_bytes: int, hps=None, sizes=None):
        """Lookups of device-resident keys; results into hps / sizes (host
        arrays of >= n entries, pinned for speed) or fresh arrays."""
        hps = np.zeros(max(n, 1), dtype=np.uint64) if hps is None else hps
        sizes = np.zeros(max(n, 1), dtype=np.int32) if sizes is None else sizes
        v = lambda a: C.c_void_p(a) if a else None  # noqa: E731
        _check(self._L.gmpt_gets_forest_device(self._h, v(d_keys), v(d_kidx), v(d_tids), int(n), int(keys_bytes),
                                               _p(hps), _p(sizes)))
        return hps[:n], sizes[:n]

    def flush_dirty(self) -> list:
        """gmpt_flush_dirty: [(hash, encoding)] of the nodes hashed since the
        last flush (needs set_option("track_dirty", 1) before the puts)."""
        h, e, ix = C.c_void_p(), C.c_void_p(), C.c_void_p()
        num = C.c_ulonglong(0)
        _check(self._L.gmpt_flush_dirty(self._h, C.byref(h), C.byref(e), C.byref(ix), C.byref(num)))
        n = num.value
        out = []
        try:
            idx = np.ctypeslib.as_array(C.cast(ix, C.POINTER(C.c_ulonglong)), shape=(2 * n,)) if n else []
            for i in range(n):
                hb = C.string_at(h.value + 32 * i, 32)
                a, z = int(idx[2 * i]), int(idx[2 * i + 1])
                out.append((hb, C.string_at(e.value + a, z - a + 1)))
        finally:
            for p in (h, e, ix):
                self._L.gmpt_free_buffer(p)
        return out

    def gets_device(self, d_keys, d_kidx, n: int, keys_bytes: int, d_out_hp, d_out_len, d_tids: int = 0):
        """Lookups of device-resident keys with device-resident results."""
        v = lambda a: C.c_void_p(a) if a else None  # noqa: E731
        _check(self._L.gmpt_gets_device(self._h, v(d_keys), v(d_kidx), v(d_tids), int(n), int(keys_bytes),
                                        v(d_out_hp), v(d_out_len)))

    def puts_raw(self, two_phase: bool, keys, keys_indexs, values, values_indexs, trie_ids=None, hps=None):
        """Put with RAW key bytes (keys_indexs: inclusive byte ranges, end =
        start - 1 for the empty key); the device expands them to nibbles +
        terminator.  Same result as the hex puts on keys_to_hexs of the keys."""
        k, ki, v, vi = _arrays(keys, keys_indexs, values, values_indexs)
        n = len(ki) // 2
        tid = None if trie_ids is None else np.ascontiguousarray(trie_ids, dtype=np.int32)
        hp_arr = None if hps is None else np.ascontiguousarray(hps, dtype=np.uint64)
        _check(self._L.gmpt_puts_raw(self._h, 1 if two_phase else 0, _p(k), _p(ki), _p(v), _p(vi),
                                     None if hp_arr is None else _p(hp_arr), None if tid is None else _p(tid), n))

    def puts_raw_device(self, two_phase: bool, d_keys, d_kidx, d_vals, d_vidx, n: int, keys_bytes: int,
                        values_bytes: int, d_tids: int = 0):
        """puts_raw with inputs already in HBM (raw device addresses)."""
        v = lambda a: C.c_void_p(a) if a else None  # noqa: E731
        _check(self._L.gmpt_puts_raw_device(self._h, 1 if two_phase else 0, v(d_keys), v(d_kidx), v(d_vals),
                                            v(d_vidx), None, v(d_tids), int(n), int(keys_bytes), int(values_bytes)))

    def puts_pipeline(self, batches, two_phase, hps=None, raw=None, raw_keys: bool = False) -> list:
        """Host batches in order, each inserted, hashed and its root read, the
        next batch's copy overlapping this one's work.  batches: objects with
        keys_hexs / keys_indexs / values / values_indexs (numpy), or raw =
        [(keys_ptr, kidx_ptr, vals_ptr, vidx_ptr, n), ...] host addresses
        (e.g. pinned tensors).  raw_keys: the key arrays hold raw key bytes
        (as puts_raw), expanded to nibbles on the device."""
        if raw is None:
            arrs = [_arrays(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs) for b in batches]
            raw = [(a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, a[3].ctypes.data, len(a[1]) // 2)
                   for a in arrs]
        k = len(raw)
        P = C.c_void_p * max(k, 1)
        cols = [P(*[C.c_void_p(r[j]) for r in raw]) for j in range(4)]
        hp = None
        if hps is not None:
            hp_arrs = [None if h is None else np.ascontiguousarray(h, dtype=np.uint64) for h in hps]
            hp = P(*[None if h is None else h.ctypes.data_as(C.c_void_p) for h in hp_arrs])
        counts = np.array([r[4] for r in raw], dtype=np.int32)
        tp = np.array([1 if x else 0 for x in two_phase], dtype=np.int32)
        out = np.zeros(32 * max(k, 1), dtype=np.uint8)
        sizes = np.zeros(max(k, 1), dtype=np.int32)
        f = self._L.gmpt_puts_pipeline_raw if raw_keys else self._L.gmpt_puts_pipeline
        _check(f(self._h, k, cols[0], cols[1], cols[2], cols[3], hp, _p(counts), _p(tp), _p(out), _p(sizes)))
        return [out[32 * i: 32 * i + sizes[i]].tobytes() for i in range(k)]

    def puts_device(self, two_phase: bool, d_keys, d_kidx, d_vals, d_vidx, n: int, keys_bytes: int,
                    values_bytes: int, d_hps: int = 0):
        """Inputs already in HBM (raw device addresses, e.g. tensor.data_ptr())."""
        f = self._L.gmpt_puts_2phase_device if two_phase else self._L.gmpt_puts_latching_device
        _check(f(self._h, C.c_void_p(d_keys), C.c_void_p(d_kidx), C.c_void_p(d_vals), C.c_void_p(d_vidx),
                 C.c_void_p(d_hps) if d_hps else None, n, keys_bytes, values_bytes))

    # -- hash / root ---------------------------------------------------------
    def hash_onepass_v2(self):
        _check(self._L.gmpt_hash_onepass(self._h))

    def pending_targets(self) -> int:
        p = C.c_void_p()
        n = C.c_int()
        _check(self._L.gmpt_pending_targets(self._h, C.byref(p), C.byref(n)))
        return n.value

    def get_root_hash(self) -> bytes:
        out = (C.c_uint8 * 32)()
        size = C.c_int()
        _check(self._L.gmpt_get_root_hash(self._h, out, C.byref(size)))
        return bytes(out)[: size.value]

    # -- lookups -------------------------------------------------------------
    def gets_parallel(self, keys_hexs, keys_indexs):
        kh, ki, _, _ = _arrays(keys_hexs, keys_indexs)
        n = len(ki) // 2
        hps = np.zeros(n, dtype=np.uint64)
        sizes = np.zeros(n, dtype=np.int32)
        _check(self._L.gmpt_gets_parallel(self._h, _p(kh), _p(ki), n, _p(hps), _p(sizes)))
        return hps, sizes

    def get_values(self, keys_hexs, keys_indexs):
        kh, ki, _, _ = _arrays(keys_hexs, keys_indexs)
        n = len(ki) // 2
        idx = np.zeros(2 * n, dtype=np.int64)
        need = C.c_int64()
        rc = self._L.gmpt_get_values(self._h, _p(kh), _p(ki), n, None, 0, _p(idx), C.byref(need))
        buf = np.zeros(max(need.value, 1), dtype=np.uint8)
        _check(self._L.gmpt_get_values(self._h, _p(kh), _p(ki), n, _p(buf), len(buf), _p(idx), C.byref(need)))
        del rc
        return [None if idx[2 * i] < 0 else buf[idx[2 * i]: idx[2 * i + 1] + 1].tobytes() for i in range(n)]

    def stats(self) -> dict:
        s = Stats()
        _check(self._L.gmpt_get_stats(self._h, C.byref(s)))
        return s.as_dict()

    def set_option(self, name: str, value: int):
        _check(self._L.gmpt_set_option(self._h, name.encode(), int(value)))

    def stream_ptr(self) -> int:
        return self._L.gmpt_stream(self._h) or 0

    def set_timing(self, on: bool = True):
        _check(self._L.gmpt_set_timing(self._h, 1 if on else 0))
