"""gmpt_keccak256_batch_noalloc: the allocation-free batched Keccak-256.

Some callers cannot allocate device memory where they call us (their
process's GPU memory is owned by another allocator, or they must not trigger
cudaMalloc/cudaFree).  This entry point stages through a fixed array inside
the library instead.  Its results must equal the allocating entry point's,
call after call (the shared array keeps the previous call's bytes, so a
shorter second call must not see them).  This file is collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def flat(msgs):
    data = np.frombuffer(b"".join(msgs) + b"\0", dtype=np.uint8)
    idx = np.zeros(2 * len(msgs), dtype=np.int64)
    pos = 0
    for i, m in enumerate(msgs):
        idx[2 * i], idx[2 * i + 1] = pos, pos + len(m) - 1
        pos += len(m)
    return data, idx


def call(fn, msgs):
    data, idx = flat(msgs)
    out = np.zeros(32 * len(msgs), dtype=np.uint8)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    rc = fn(P(data), P(idx), len(msgs), P(out))
    return rc, out.tobytes()


def test_noalloc_matches_allocating_entry_point_twice(gpu_lib):
    L = gpu_lib.lib()
    rng = np.random.default_rng(2024)
    first = [rng.integers(0, 256, int(n), dtype=np.uint8).tobytes()
             for n in rng.integers(0, 700, 3000)] + [b"\xff" * 5000]
    second = [rng.integers(0, 256, int(n), dtype=np.uint8).tobytes() for n in rng.integers(0, 150, 500)]
    for msgs in (first, second):
        rc_a, ref = call(L.gmpt_keccak256_batch, msgs)
        rc_b, got = call(L.gmpt_keccak256_batch_noalloc, msgs)
        assert rc_a == 0 and rc_b == 0, L.gmpt_last_error_message()
        assert got == ref


def test_noalloc_rejects_calls_over_its_limits(gpu_lib):
    L = gpu_lib.lib()
    rc, _ = call(L.gmpt_keccak256_batch_noalloc, [b"a"] * 32769)
    assert rc == 5 and b"32768" in L.gmpt_last_error_message()
    rc, _ = call(L.gmpt_keccak256_batch_noalloc, [b"\0" * (2 << 20), b"x"])
    assert rc == 5 and b"limit" in L.gmpt_last_error_message()
    msgs = [b"after a rejected call"]
    assert call(L.gmpt_keccak256_batch_noalloc, msgs)[1] == call(L.gmpt_keccak256_batch, msgs)[1]
