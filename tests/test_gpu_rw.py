"""Mixed read/write batches (gmpt_puts_*_with_read) vs a sequential model.

The reference's puts_*_with_read (gpu_mpt.cuh:684-765, 1609-1713) run the
reads of a batch concurrently with its writes; the library defines the
result as the batch applied in index order.  Expected results come from a
plain dict applied op by op; roots from the oracle trie given the writes.
"""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import make_batch, nib
from gmpt import workloads as W

pytestmark = pytest.mark.gpu


def keyset(rng, n, max_len, alpha):
    out = set()
    while len(out) < n:
        ln = 1 + int(rng.words(1)[0] % max_len)
        out.add(bytes(int(x) % alpha for x in rng.words(ln)))
    return sorted(out)


def mixed_ops(rng, pool, n, p_write, fresh):
    keys, flags, vals, hps = [], [], [], []
    for i in range(n):
        u = int(rng.words(1)[0])
        k = fresh[i % len(fresh)] if (u & 7) == 0 and fresh else pool[(u >> 8) % len(pool)]
        w = ((u >> 40) % 1000) < p_write * 1000
        keys.append(k)
        flags.append(1 if w else 0)
        vals.append(rng.bytes(1 + int(rng.words(1)[0] % 60)).tobytes() if w else b"")
        hps.append(1_000_000 + i if w else 0)
    return keys, np.array(flags, np.uint8), vals, np.array(hps, np.uint64)


def expect(state, keys, flags, vals, hps, tids=None):
    """Sequential model: state maps (trie, key) -> (hp, value)."""
    got = []
    for i, k in enumerate(keys):
        t = 0 if tids is None else int(tids[i])
        if flags[i]:
            state[(t, k)] = (int(hps[i]), vals[i])
        else:
            hp, v = state.get((t, k), (0, None))
            got.append((hp, 0 if v is None else len(v)))
    return got


def oracle_root(mode, state, trie=0):
    items = sorted((k, v) for (t, k), (_, v) in state.items() if t == trie)
    if not items:
        return b""
    o = O.OracleTrie(mode)
    b = make_batch([nib(k) for k, _ in items], [v for _, v in items])
    o.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    o.hash()
    return o.root()


def load(mpt, rng, pool, two_phase):
    vals = [rng.bytes(1 + int(rng.words(1)[0] % 60)).tobytes() for _ in pool]
    hps = np.arange(1, len(pool) + 1, dtype=np.uint64)
    b = make_batch([nib(k) for k in pool], vals)
    f = mpt.puts_2phase_with_valuehp if two_phase else mpt.puts_latching_with_valuehp_v2
    f(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, hps)
    mpt.hash_onepass_v2()
    return {(0, k): (int(h), v) for k, v, h in zip(pool, vals, hps)}


@pytest.mark.parametrize("mode", [O.MODE_REF, O.MODE_GETH])
@pytest.mark.parametrize("two_phase", [True, False])
@pytest.mark.parametrize("p_write", [0.5, 0.05, 0.95])
def test_mixed_batch_matches_sequential_model(gpu_lib, mode, two_phase, p_write):
    rng = W.Xoshiro256ss(0x5A0 + 7 * mode + 3 * two_phase + int(100 * p_write))
    pool = keyset(rng, 1500, 8, 16)
    fresh = keyset(rng, 300, 9, 256)
    t = gpu_lib.MPT(mode=mode)
    state = load(t, rng, pool, two_phase)
    for step in range(2):
        keys, flags, vals, hps = mixed_ops(rng, pool, 4000, p_write, fresh)
        want = expect(state, keys, flags, vals, hps)
        b = make_batch([nib(k) for k in keys], vals)
        rh, rs = t.puts_with_read(two_phase, b.keys_hexs, b.keys_indexs, flags, b.values, b.values_indexs,
                                  values_hps=hps)
        assert len(rh) == len(want) == int((flags == 0).sum())
        assert list(zip(rh.tolist(), rs.tolist())) == want, step
        t.hash_onepass_v2()
        assert t.get_root_hash() == oracle_root(mode, state), step
    t.close()


@pytest.mark.parametrize("two_phase", [True, False])
def test_mixed_batch_edge_cases(gpu_lib, two_phase):
    rng = W.Xoshiro256ss(0x5B1 + two_phase)
    pool = keyset(rng, 500, 6, 16)
    # empty trie: reads of keys written later in the batch see nothing,
    # reads after a write see it (bulk-load path for PhaseNU)
    t = gpu_lib.MPT()
    keys = [pool[0], pool[0], pool[0], pool[0], pool[1], pool[2]]
    flags = np.array([0, 1, 0, 1, 0, 0], np.uint8)
    vals = [b"", b"a" * 40, b"", b"b" * 41, b"", b""]
    hps = np.array([0, 11, 0, 12, 0, 0], np.uint64)
    b = make_batch([nib(k) for k in keys], vals)
    rh, rs = t.puts_with_read(two_phase, b.keys_hexs, b.keys_indexs, flags, b.values, b.values_indexs,
                              values_hps=hps)
    assert list(zip(rh.tolist(), rs.tolist())) == [(0, 0), (11, 40), (0, 0), (0, 0)]
    t.hash_onepass_v2()
    assert t.get_root_hash() == oracle_root(O.MODE_REF, {(0, pool[0]): (12, b"b" * 41)})
    # reads only: trie unchanged
    state = load(t, rng, pool, two_phase)
    root = t.get_root_hash()
    keys = [pool[i % 500] for i in range(0, 3000, 7)]
    flags = np.zeros(len(keys), np.uint8)
    b = make_batch([nib(k) for k in keys], [b""] * len(keys))
    rh, rs = t.puts_with_read(two_phase, b.keys_hexs, b.keys_indexs, flags, b.values, b.values_indexs)
    assert list(zip(rh.tolist(), rs.tolist())) == [(state[(0, k)][0], len(state[(0, k)][1])) for k in keys]
    t.hash_onepass_v2()
    assert t.get_root_hash() == root
    # a bad flag rejects the whole batch
    flags = np.ones(len(keys), np.uint8)
    flags[5] = 2
    vals = [b"z" * 33] * len(keys)
    b = make_batch([nib(k) for k in keys], vals)
    with pytest.raises(gpu_lib.GmptError):
        t.puts_with_read(two_phase, b.keys_hexs, b.keys_indexs, flags, b.values, b.values_indexs)
    t.hash_onepass_v2()
    assert t.get_root_hash() == root
    t.close()


def test_mixed_batch_forest_and_device(gpu_lib):
    rng = W.Xoshiro256ss(0x5C2)
    n_tries = 9
    pool = keyset(rng, 800, 7, 16)
    keys, flags, vals, hps = mixed_ops(rng, pool, 6000, 0.5, [])
    tids = (np.arange(len(keys)) * 5 % n_tries).astype(np.int32)
    for two_phase in (True, False):
        state = {}
        want = expect(state, keys, flags, vals, hps, tids)
        roots = [oracle_root(O.MODE_GETH, state, tr) for tr in range(n_tries)]
        b = make_batch([nib(k) for k in keys], vals)
        t = gpu_lib.MPT(mode=O.MODE_GETH, max_tries=n_tries)
        rh, rs = t.puts_with_read(two_phase, b.keys_hexs, b.keys_indexs, flags, b.values, b.values_indexs,
                                  trie_ids=tids, values_hps=hps)
        assert list(zip(rh.tolist(), rs.tolist())) == want
        t.hash_onepass_v2()
        assert t.get_roots(n=n_tries) == roots
        t.close()
        # device inputs and device results; values_hps are not passed here
        d = [torch.from_numpy(np.ascontiguousarray(a)).cuda()
             for a in (b.keys_hexs, b.keys_indexs, flags, b.values, b.values_indexs, tids)]
        out_hp = torch.zeros(len(keys), dtype=torch.int64, device="cuda")
        out_len = torch.zeros(len(keys), dtype=torch.int32, device="cuda")
        g = gpu_lib.MPT(mode=O.MODE_GETH, max_tries=n_tries)
        cnt = g.puts_with_read_device(two_phase, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(),
                                      d[4].data_ptr(), len(keys), len(b.keys_hexs), len(b.values), out_hp.data_ptr(),
                                      out_len.data_ptr(), d_tids=d[5].data_ptr())
        assert cnt == len(want)
        assert out_len[:cnt].cpu().tolist() == [s for _, s in want]
        assert not out_hp[:cnt].any()
        g.hash_onepass_v2()
        assert g.get_roots(n=n_tries) == roots
        g.close()


@pytest.mark.parametrize("two_phase", [True, False])
def test_mixed_batch_hash_collisions_fall_back_exactly(gpu_lib, two_phase):
    # 3-bit key hashes: every slot is shared by different keys, so grouping
    # by hash slot is refused and the full-key sort groups the batch
    rng = W.Xoshiro256ss(0x5D3 + two_phase)
    pool = keyset(rng, 600, 7, 16)
    t = gpu_lib.MPT()
    state = load(t, rng, pool, two_phase)
    t.set_option("latch_dedup_bits", 3)
    keys, flags, vals, hps = mixed_ops(rng, pool, 3000, 0.5, keyset(rng, 50, 5, 256))
    want = expect(state, keys, flags, vals, hps)
    b = make_batch([nib(k) for k in keys], vals)
    rh, rs = t.puts_with_read(two_phase, b.keys_hexs, b.keys_indexs, flags, b.values, b.values_indexs,
                              values_hps=hps)
    assert list(zip(rh.tolist(), rs.tolist())) == want
    t.hash_onepass_v2()
    assert t.get_root_hash() == oracle_root(O.MODE_REF, state)
    t.close()


@pytest.mark.parametrize("two_phase", [False, True])
def test_mixed_batches_keep_only_the_kept_writes_keys(gpu_lib, two_phase):
    # the key arena grows by the kept writes' key bytes only: reads (and
    # overwritten writes) give their bytes back after the batch
    rng = W.Xoshiro256ss(91)
    pool = keyset(rng, 3000, 24, 256)
    t = gpu_lib.MPT()
    load = make_batch([nib(k) for k in pool], [b"v" * 8] * len(pool))
    t.puts_2phase_with_valuehp(load.keys_hexs, load.keys_indexs, load.values, load.values_indexs)
    t.hash_onepass_v2()
    state = {(0, k): (0, b"v" * 8) for k in pool}
    for rnd in range(3):
        before = t.stats()["key_bytes"]
        keys, flags, vals, hps = mixed_ops(rng, pool, 5000, 0.3 if rnd < 2 else 0.0, [])
        b = make_batch([nib(k) for k in keys], [v if f else b"" for v, f in zip(vals, flags)])
        hp, sz = t.puts_with_read(two_phase, b.keys_hexs, b.keys_indexs, flags, b.values, b.values_indexs,
                                  values_hps=hps)
        t.hash_onepass_v2()
        want = expect(state, keys, flags, vals, hps)
        assert list(zip(hp.tolist(), sz.tolist())) == want
        last = {}
        for k, f in zip(keys, flags):
            if f:
                last[k] = len(nib(k))
        grown = t.stats()["key_bytes"] - before
        assert grown == (sum(last.values()) + 7) // 8 * 8
        assert t.get_root_hash() == oracle_root(O.MODE_REF, state)
    t.close()
