"""ctypes bindings for the CPU checkers (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` /
``--impl reference`` legs may import this module.  It loads:

* ``liboracle.so``          -- the plain-C restatement of the reference CPU MPT
                                (mpt_oracle.c; cites cpu_mpt.cuh / node.cuh /
                                rlp.cuh / utils.cuh / cpu_hash.h line ranges);
* ``_ref/libgmpt_ref*.so``  -- the reference's own ``CpuMPT::Compress::MPT``
                                compiled from its unmodified sources through the
                                shim headers in ``ref_shim/`` (see Makefile).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
MODE_REF = 0
MODE_GETH = 1

_u8p = C.POINTER(C.c_uint8)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and _ref/ when the reference tree is present)."""
    out = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


_lib = None
_ref = {}


def lib():
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        L = C.CDLL(str(path))
        L.omt_new.restype = C.c_void_p
        L.omt_new.argtypes = [C.c_int]
        L.omt_free.argtypes = [C.c_void_p]
        L.omt_puts.restype = C.c_int
        L.omt_puts.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.omt_hash.argtypes = [C.c_void_p]
        L.omt_root.restype = C.c_int
        L.omt_root.argtypes = [C.c_void_p, C.c_void_p]
        L.omt_gets.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.omt_get_stats.argtypes = [C.c_void_p, C.c_void_p]
        L.omt_count_stats.restype = C.c_uint64
        L.omt_count_stats.argtypes = [C.c_void_p]
        L.omt_keccak256.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p]
        L.omt_sha3_256.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p]
        L.omt_keccak_f1600.argtypes = [C.c_void_p]
        L.omt_keccak256_rows.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p]
        L.omt_flush.restype = C.c_int
        L.omt_flush.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.omt_free_buffer.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def ref_lib(big: bool = False):
    """The reference's CpuMPT compiled from its sources (None if not built)."""
    key = "big" if big else "small"
    if key not in _ref:
        path = HERE / "_ref" / ("libgmpt_ref_big.so" if big else "libgmpt_ref.so")
        if not path.exists():
            _ref[key] = None
            return None
        L = C.CDLL(str(path))
        L.ref_new.restype = C.c_void_p
        L.ref_delete.argtypes = [C.c_void_p]
        L.ref_set_threads.argtypes = [C.c_int]
        for f in ("ref_puts_baseline", "ref_puts_lock", "ref_puts_2phase"):
            getattr(L, f).argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.ref_hash_dirty.argtypes = [C.c_void_p]
        L.ref_root.restype = C.c_int
        L.ref_root.argtypes = [C.c_void_p, C.c_void_p]
        L.ref_root_parallel.restype = C.c_int
        L.ref_root_parallel.argtypes = [C.c_void_p, C.c_void_p]
        L.ref_gets.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.ref_keccak256.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p]
        _ref[key] = L
    return _ref[key]


# --------------------------------------------------------------------------
# Keccak


def keccak256(data: bytes) -> bytes:
    buf = np.frombuffer(bytes(data) + b"\0", dtype=np.uint8)
    out = np.zeros(32, np.uint8)
    lib().omt_keccak256(_ptr(buf), len(data), _ptr(out))
    return out.tobytes()


def keccak256_rows(msgs: np.ndarray) -> np.ndarray:
    """Keccak-256 of every row of a 2-D uint8 array -> [rows, 32] (CPU; the
    same contract as gmpt.keccak256_rows)."""
    m = np.ascontiguousarray(msgs, dtype=np.uint8)
    rows, width = m.shape
    out = np.empty((rows, 32), dtype=np.uint8)
    lib().omt_keccak256_rows(_ptr(m), rows, width, _ptr(out))
    return out


def sha3_256(data: bytes) -> bytes:
    buf = np.frombuffer(bytes(data) + b"\0", dtype=np.uint8)
    out = np.zeros(32, np.uint8)
    lib().omt_sha3_256(_ptr(buf), len(data), _ptr(out))
    return out.tobytes()


def ref_keccak256(data: bytes) -> bytes:
    L = ref_lib()
    buf = np.frombuffer(bytes(data) + b"\0" * 8, dtype=np.uint8)
    out = np.zeros(32, np.uint8)
    L.ref_keccak256(_ptr(buf), len(data), _ptr(out))
    return out.tobytes()


# --------------------------------------------------------------------------
# Tries


class OracleStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "hashed_nodes", "hashed_full", "hashed_short", "enc_bytes", "keccak_blocks",
        "keccak_calls", "nodes_full", "nodes_short", "nodes_value", "max_depth_nibbles")]


class OracleTrie:
    """The C restatement: sequential puts (last write wins) + dirty-flag hash."""

    def __init__(self, mode: int = MODE_REF):
        self._L = lib()
        self._t = self._L.omt_new(mode)

    def close(self):
        if self._t:
            self._L.omt_free(self._t)
            self._t = None

    def __del__(self):
        self.close()

    def puts(self, keys_hexs, keys_indexs, values, values_indexs):
        kh = np.ascontiguousarray(keys_hexs, dtype=np.uint8)
        ki = np.ascontiguousarray(keys_indexs, dtype=np.int32)
        vb = np.ascontiguousarray(values, dtype=np.uint8)
        vi = np.ascontiguousarray(values_indexs, dtype=np.int64)
        n = len(ki) // 2
        rc = self._L.omt_puts(self._t, _ptr(kh), _ptr(ki), _ptr(vb), _ptr(vi), n)
        if rc != 0:
            raise ValueError(f"oracle puts failed: {rc}")

    def hash(self):
        self._L.omt_hash(self._t)

    def root(self) -> bytes:
        out = np.zeros(32, np.uint8)
        n = self._L.omt_root(self._t, _ptr(out))
        return out[:n].tobytes()

    def gets(self, keys_hexs, keys_indexs):
        kh = np.ascontiguousarray(keys_hexs, dtype=np.uint8)
        ki = np.ascontiguousarray(keys_indexs, dtype=np.int32)
        n = len(ki) // 2
        ptr = np.zeros(n, np.uint64)
        ln = np.zeros(n, np.int32)
        self._L.omt_gets(self._t, _ptr(kh), _ptr(ki), n, _ptr(ptr), _ptr(ln))
        return [None if p == 0 else C.string_at(int(p), int(l)) for p, l in zip(ptr, ln)]

    def flush(self) -> list:
        """[(hash32, encoding)] of the nodes on put paths since the last
        flush that are referenced by hash or are the root (omt_flush)."""
        h, e, ix = C.c_void_p(), C.c_void_p(), C.c_void_p()
        num = C.c_uint64(0)
        if self._L.omt_flush(self._t, C.byref(h), C.byref(e), C.byref(ix), C.byref(num)) != 0:
            raise MemoryError("oracle flush")
        out = []
        try:
            n = num.value
            idx = np.ctypeslib.as_array(C.cast(ix, C.POINTER(C.c_uint64)), shape=(2 * n,)) if n else []
            for i in range(n):
                a, z = int(idx[2 * i]), int(idx[2 * i + 1])
                out.append((C.string_at(h.value + 32 * i, 32), C.string_at(e.value + a, z - a + 1)))
        finally:
            for p in (h, e, ix):
                if p.value:
                    self._L.omt_free_buffer(p)
        return out

    def stats(self) -> dict:
        self._L.omt_count_stats(self._t)
        s = OracleStats()
        self._L.omt_get_stats(self._t, C.byref(s))
        return {f: getattr(s, f) for f, _ in s._fields_}


class RefTrie:
    """The reference's own CpuMPT (compiled from its sources)."""

    def __init__(self, big: bool = False, threads: int = 1):
        self._L = ref_lib(big)
        if self._L is None:
            raise RuntimeError("oracle/_ref not built (reference tree absent)")
        self._L.ref_set_threads(threads)
        self._t = self._L.ref_new()
        self._keep = []

    def close(self):
        if self._t:
            self._L.ref_delete(self._t)
            self._t = None

    def __del__(self):
        self.close()

    def _arrs(self, keys_hexs, keys_indexs, values, values_indexs):
        kh = np.ascontiguousarray(keys_hexs, dtype=np.uint8)
        ki = np.ascontiguousarray(keys_indexs, dtype=np.int32)
        vb = np.ascontiguousarray(values, dtype=np.uint8)
        vi = np.ascontiguousarray(values_indexs, dtype=np.int64)
        self._keep.append((kh, ki, vb, vi))  # nodes point into these buffers
        return kh, ki, vb, vi

    def puts_baseline(self, *a):
        kh, ki, vb, vi = self._arrs(*a)
        self._L.ref_puts_baseline(self._t, _ptr(kh), _ptr(ki), _ptr(vb), _ptr(vi), len(ki) // 2)

    def puts_lock_and_hash(self, *a):
        kh, ki, vb, vi = self._arrs(*a)
        self._L.ref_puts_lock(self._t, _ptr(kh), _ptr(ki), _ptr(vb), _ptr(vi), len(ki) // 2)

    def puts_2phase_and_hash(self, *a):
        kh, ki, vb, vi = self._arrs(*a)
        self._L.ref_puts_2phase(self._t, _ptr(kh), _ptr(ki), _ptr(vb), _ptr(vi), len(ki) // 2)

    def hash(self):
        self._L.ref_hash_dirty(self._t)

    def root(self, parallel: bool = False) -> bytes:
        out = np.zeros(32, np.uint8)
        f = self._L.ref_root_parallel if parallel else self._L.ref_root
        n = f(self._t, _ptr(out))
        return out[:n].tobytes()

    def gets(self, keys_hexs, keys_indexs):
        kh = np.ascontiguousarray(keys_hexs, dtype=np.uint8)
        ki = np.ascontiguousarray(keys_indexs, dtype=np.int32)
        n = len(ki) // 2
        ptr = np.zeros(n, np.uint64)
        ln = np.zeros(n, np.int32)
        self._L.ref_gets(self._t, _ptr(kh), _ptr(ki), n, _ptr(ptr), _ptr(ln))
        return [None if p == 0 else C.string_at(int(p), int(l)) for p, l in zip(ptr, ln)]
