"""Deletes (gmpt_deletes*): the trie after deleting keys must be the canonical
trie of the remaining keys -- the same root as an oracle trie built from
them alone, in both encode modes, after either insert strategy -- and lookups
of deleted keys must miss.  The reference has no delete path, so the oracle
here is a rebuild from the remaining key set."""
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


def oracle_root(mode, items):
    if not items:
        return b""
    o = O.OracleTrie(mode)
    ks = sorted(items)
    b = make_batch([nib(k) for k in ks], [items[k] for k in ks])
    o.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    o.hash()
    return o.root()


def put(t, two_phase, items):
    ks = list(items)
    b = make_batch([nib(k) for k in ks], [items[k] for k in ks])
    f = t.puts_2phase_with_valuehp if two_phase else t.puts_latching_with_valuehp_v2
    f(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    t.hash_onepass_v2()


def delete(t, keys, trie_ids=None):
    b = make_batch([nib(k) for k in keys], [b"x"] * len(keys))
    t.deletes(b.keys_hexs, b.keys_indexs, trie_ids)
    t.hash_onepass_v2()


@pytest.mark.parametrize("mode", [O.MODE_REF, O.MODE_GETH])
@pytest.mark.parametrize("two_phase", [True, False])
@pytest.mark.parametrize("alpha,max_len", [(2, 10), (4, 6), (256, 20)])
def test_deletes_match_rebuilt_oracle(gpu_lib, mode, two_phase, alpha, max_len):
    rng = W.Xoshiro256ss(0xDE1 + 3 * mode + two_phase + alpha)
    keys = keyset(rng, 1200 if alpha > 2 else 600, max_len, alpha)
    items = {k: rng.bytes(1 + int(rng.words(1)[0] % 50)).tobytes() for k in keys}
    t = gpu_lib.MPT(mode=mode)
    put(t, two_phase, items)
    assert t.get_root_hash() == oracle_root(mode, items)
    for step, share in enumerate([0.3, 0.5, 0.9]):
        live = sorted(items)
        sel = [k for k in live if (int(rng.words(1)[0]) % 1000) < share * 1000]
        absent = keyset(rng, 20, max_len + 3, 256)
        batch = sel + [k for k in absent if k not in items] + sel[:5]  # absent keys and repeats are ignored
        delete(t, batch)
        for k in sel:
            items.pop(k, None)
        assert t.get_root_hash() == oracle_root(mode, items), step
        # deleted keys miss, the rest still answer
        probes = sel[:200] + sorted(items)[:200]
        pb = make_batch([nib(k) for k in probes], [b"x"] * len(probes))
        got = t.get_values(pb.keys_hexs, pb.keys_indexs)
        assert got == [items.get(k) for k in probes], step
        # re-insert some deleted keys with new values: the trie keeps working
        back = {k: rng.bytes(1 + int(rng.words(1)[0] % 40)).tobytes() for k in sel[: len(sel) // 3]}
        if back:
            put(t, not two_phase, back)
            items.update(back)
            assert t.get_root_hash() == oracle_root(mode, items), step
    t.close()


def test_delete_everything_and_single_keys(gpu_lib):
    for two_phase in (True, False):
        t = gpu_lib.MPT(mode=O.MODE_GETH)
        items = {b"\x01\x02": b"a" * 40, b"\x01\x02\x03": b"b" * 40, b"\x01\x03": b"c" * 3, b"\xff": b"d" * 33}
        put(t, two_phase, items)
        delete(t, [b"\x01\x02"])  # a key that ends where a longer key branches
        items.pop(b"\x01\x02")
        assert t.get_root_hash() == oracle_root(O.MODE_GETH, items)
        delete(t, [b"\x01\x03", b"\xff"])
        items.pop(b"\x01\x03")
        items.pop(b"\xff")
        assert t.get_root_hash() == oracle_root(O.MODE_GETH, items)  # a single leaf left at the root
        delete(t, [b"\x01\x02\x03"])
        assert t.get_root_hash() == b""
        put(t, two_phase, {b"\x07": b"e" * 50})
        assert t.get_root_hash() == oracle_root(O.MODE_GETH, {b"\x07": b"e" * 50})
        t.close()


def test_deletes_forest_and_device(gpu_lib):
    rng = W.Xoshiro256ss(0xDE7)
    n_tries = 7
    keys = keyset(rng, 1500, 6, 16)
    tids = (np.arange(len(keys)) * 3 % n_tries).astype(np.int32)
    vals = [rng.bytes(1 + int(rng.words(1)[0] % 40)).tobytes() for _ in keys]
    per = [{k: v for k, v, t in zip(keys, vals, tids) if t == tr} for tr in range(n_tries)]
    for device in (False, True):
        f = gpu_lib.MPT(mode=O.MODE_GETH, max_tries=n_tries)
        b = make_batch([nib(k) for k in keys], vals)
        f.puts_forest(False, b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, tids)
        f.hash_onepass_v2()
        sel = [i for i in range(len(keys)) if i % 4 != 1]
        db = make_batch([nib(keys[i]) for i in sel], [b"x"] * len(sel))
        dt = tids[sel]
        if device:
            d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (db.keys_hexs, db.keys_indexs, dt)]
            f.deletes_device(d[0].data_ptr(), d[1].data_ptr(), len(sel), len(db.keys_hexs), d_tids=d[2].data_ptr())
        else:
            f.deletes(db.keys_hexs, db.keys_indexs, dt)
        f.hash_onepass_v2()
        left = [dict(p) for p in per]
        for i in sel:
            left[tids[i]].pop(keys[i])
        assert f.get_roots(n=n_tries) == [oracle_root(O.MODE_GETH, left[tr]) for tr in range(n_tries)], device
        f.close()
