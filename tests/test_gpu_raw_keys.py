"""Raw-key batches (gmpt_puts_raw*): key bytes in, nibbles made on the device.

The reference converts keys on the host (test/experiments.cu:50-73,
util/utils.cuh:340-349) before its puts; a raw-key put must give exactly
the trie that the hex put of the converted keys gives, in both encode modes
and for both insert strategies, whatever the layout of the index pairs.
"""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import make_batch, nib
from gmpt import workloads as W

pytestmark = pytest.mark.gpu


def raw_batch(keys, vals, order=None):
    """Flat raw layout; `order` places the keys' bytes in the stream in a
    different order than the pairs list them (pairs need not tile).  The
    last listed key stays last in the stream: the stream length is its end
    + 1, as in the reference's layout."""
    order = list(range(len(keys))) if order is None else [int(i) for i in order if i != len(keys) - 1]
    if len(order) < len(keys):
        order.append(len(keys) - 1)
    stream, at = b"", {}
    for i in order:
        at[i] = len(stream)
        stream += keys[i] + b"\xAA"  # a gap byte between keys
    ki = []
    for i, k in enumerate(keys):
        ki += [at[i], at[i] + len(k) - 1]
    vb, vi, pos = b"", [], 0
    for v in vals:
        vb += v
        vi += [pos, pos + len(v) - 1]
        pos += len(v)
    return (np.frombuffer(stream, np.uint8).copy(), np.array(ki, np.int32), np.frombuffer(vb, np.uint8).copy(),
            np.array(vi, np.int64))


def random_keys(rng, n, max_len, alpha=256, dup_every=9):
    keys, vals = [], []
    for i in range(n):
        if i and i % dup_every == 0:
            keys.append(keys[int(rng.words(1)[0] % i)])
        else:
            ln = 1 + int(rng.words(1)[0] % max_len)
            keys.append(bytes(int(x) % alpha for x in rng.words(ln)))
        vals.append(rng.bytes(1 + int(rng.words(1)[0] % 70)).tobytes())
    return keys, vals


def oracle_of(mode, batches):
    o = O.OracleTrie(mode)
    for keys, vals in batches:
        b = make_batch([nib(k) for k in keys], vals)
        o.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        o.hash()
    return o


@pytest.mark.parametrize("mode", [O.MODE_REF, O.MODE_GETH])
@pytest.mark.parametrize("two_phase", [True, False])
def test_raw_puts_match_hex_oracle(gpu_lib, mode, two_phase):
    rng = W.Xoshiro256ss(0x4A1 + 2 * mode + two_phase)
    f = gpu_lib.MPT(mode=mode)
    batches = []
    for step, (n, max_len, alpha) in enumerate([(700, 12, 4), (1500, 33, 256), (400, 3, 2)]):
        keys, vals = random_keys(rng, n, max_len, alpha)
        order = list(np.random.default_rng(step).permutation(n)) if step == 1 else None
        f.puts_raw(two_phase, *raw_batch(keys, vals, order))
        f.hash_onepass_v2()
        batches.append((keys, vals))
        o = oracle_of(mode, batches)
        assert f.get_root_hash() == o.root(), step
    keys, _ = random_keys(rng, 300, 12, 4)
    probes = make_batch([nib(k) for k in keys], [b"x"] * len(keys))
    want = o.gets(probes.keys_hexs, probes.keys_indexs)
    got = f.get_values(probes.keys_hexs, probes.keys_indexs)
    assert got == want
    f.close()


def test_raw_empty_key_and_hex_empty_key(gpu_lib):
    # the empty key (pair end = start - 1) is hex [16]: the root's value slot
    keys = [b"", b"\x12", b"\x12\x34", b"\xff"]
    vals = [b"e" * 40, b"a" * 5, b"b" * 40, b"c" * 33]
    o = oracle_of(O.MODE_REF, [(keys, vals)])
    for two_phase in (True, False):
        f = gpu_lib.MPT()
        f.puts_raw(two_phase, *raw_batch(keys, vals))
        f.hash_onepass_v2()
        assert f.get_root_hash() == o.root(), two_phase
        h = gpu_lib.MPT()
        b = make_batch([nib(k) for k in keys], vals)
        (h.puts_2phase_with_valuehp if two_phase else h.puts_latching_with_valuehp_v2)(
            b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        h.hash_onepass_v2()
        assert h.get_root_hash() == o.root(), two_phase
        f.close()
        h.close()


def test_raw_forest_and_device(gpu_lib):
    rng = W.Xoshiro256ss(0x4B7)
    n_tries = 12
    keys, vals = random_keys(rng, 2000, 20, 16)
    tids = (np.arange(len(keys)) * 7 % n_tries).astype(np.int32)
    kb, ki, vb, vi = raw_batch(keys, vals)
    oracles = {}
    for t in range(n_tries):
        sel = [i for i in range(len(keys)) if tids[i] == t]
        oracles[t] = oracle_of(O.MODE_GETH, [([keys[i] for i in sel], [vals[i] for i in sel])])
    want = [oracles[t].root() for t in range(n_tries)]
    for two_phase in (True, False):
        f = gpu_lib.MPT(mode=O.MODE_GETH, max_tries=n_tries)
        f.puts_raw(two_phase, kb, ki, vb, vi, trie_ids=tids)
        f.hash_onepass_v2()
        assert f.get_roots(n=n_tries) == want, two_phase
        f.close()
        # the same batch from device memory, read in place
        d = [torch.from_numpy(a).cuda() for a in (kb, ki, vb, vi, tids)]
        g = gpu_lib.MPT(mode=O.MODE_GETH, max_tries=n_tries)
        g.puts_raw_device(two_phase, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(), len(keys),
                          len(kb), len(vb), d_tids=d[4].data_ptr())
        g.hash_onepass_v2()
        assert g.get_roots(n=n_tries) == want, two_phase
        g.close()


def test_raw_pipeline_matches_hex_pipeline(gpu_lib):
    rng = W.Xoshiro256ss(0x4C3)
    raw, hexb, tp = [], [], []
    for step in range(5):
        n = 3000 + 500 * step
        key_bytes = rng.bytes(32 * n)
        ids = np.arange(n)
        if step:
            # updates of earlier keys mixed in
            key_bytes = np.concatenate([key_bytes[: 16 * n], raw[-1][0][: 16 * n]])
        lens = np.full(n, 32)
        hk, hki = W.keys_to_hexs(key_bytes, lens)
        rki = np.empty(2 * n, np.int32)
        rki[0::2] = ids * 32
        rki[1::2] = ids * 32 + 31
        vals = rng.bytes(40 * n)
        vi = np.empty(2 * n, np.int64)
        vi[0::2] = ids * 40
        vi[1::2] = ids * 40 + 39
        raw.append((key_bytes, rki, vals, vi))
        hexb.append(W.Batch(hk, hki, vals, vi))
        tp.append(step % 2 == 0)
    a = gpu_lib.MPT()
    roots_hex = a.puts_pipeline(hexb, tp)
    b = gpu_lib.MPT()
    ptrs = [(k.ctypes.data, i.ctypes.data, v.ctypes.data, vi.ctypes.data, len(i) // 2) for k, i, v, vi in raw]
    roots_raw = b.puts_pipeline(None, tp, raw=ptrs, raw_keys=True)
    assert roots_raw == roots_hex
    o = O.OracleTrie()
    for x in hexb:
        o.puts(x.keys_hexs, x.keys_indexs, x.values, x.values_indexs)
    o.hash()
    assert roots_raw[-1] == o.root()
    a.close()
    b.close()


def test_raw_bad_ranges_rejected(gpu_lib):
    f = gpu_lib.MPT()
    kb = np.frombuffer(b"\x01\x02\x03\x04", np.uint8).copy()
    vb = np.frombuffer(b"v" * 80, np.uint8).copy()
    vi = np.array([0, 39, 40, 79], np.int64)
    # (the stream length is the last pair's end + 1, as for hex batches)
    for ki in ([0, 9, 2, 3], [-1, 1, 2, 3], [0, 1, 3, 1], [0, 1, 2000, 3]):
        for two_phase in (True, False):
            with pytest.raises(gpu_lib.GmptError):
                f.puts_raw(two_phase, kb, np.array(ki, np.int32), vb, vi)
    # the object stays usable and the rejected batches left nothing behind
    f.puts_raw(True, kb, np.array([0, 1, 2, 3], np.int32), vb, vi)
    f.hash_onepass_v2()
    o = oracle_of(O.MODE_REF, [([b"\x01\x02", b"\x03\x04"], [b"v" * 40, b"v" * 40])])
    assert f.get_root_hash() == o.root()
    f.close()
