"""The commit nodeset (gmpt_flush_dirty) against the oracle's: after each
batch + hash, the set of (hash, encoding) pairs the GPU exports equals the
oracle's nodes on that batch's paths that are referenced by hash or are the
root -- for both insert strategies, both encodings, splits of existing short
nodes, repeated keys, and a batch that changes nothing but re-puts values.
The reference exports every node on a set of key paths instead
(MPT::flush_dirty_nodes, gpu_mpt.cuh:1039-1122)."""
import numpy as np
import pytest

import oracle as O
from gmpt import workloads as W

pytestmark = pytest.mark.gpu


def batches():
    load = W.ycsb_load(1 << 15, seed=0x5EED0002)
    upd = W.ycsb_zipf_updates(1 << 15, 1 << 14, seed=0x5EED0003)
    fresh = W.vocab_keys(4000, vmin=40, vmax=200, vmu=4.5)  # new keys split existing short nodes
    same = load.subset(np.arange(0, 1 << 15, 7))  # the same values again
    return [load, upd, fresh, same]


@pytest.mark.parametrize("mode", [O.MODE_REF, O.MODE_GETH])
@pytest.mark.parametrize("strategies", [("2phase",) * 4, ("latching",) * 4, ("2phase", "latching", "2phase", "latching")])
def test_flush_dirty_equals_the_oracle_nodeset(gpu_lib, mode, strategies):
    t = gpu_lib.MPT(mode=mode)
    t.set_option("track_dirty", 1)
    o = O.OracleTrie(mode)
    for b, s in zip(batches(), strategies):
        f = t.puts_2phase_with_valuehp if s == "2phase" else t.puts_latching_with_valuehp_v2
        f(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        t.hash_onepass_v2()
        o.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        o.hash()
        got = t.flush_dirty()
        want = o.flush()
        assert len(got) == len(set(got))
        assert sorted(got) == sorted(want), s
        assert t.get_root_hash() == o.root()
    assert t.flush_dirty() == []  # nothing rehashed since
    t.close()


def test_flush_dirty_skips_nodes_a_delete_unlinked(gpu_lib):
    b = W.random_keys(20000, 32, 40, seed=0x5EED0F10)
    gone = b.subset(np.arange(0, b.n, 3))
    keep = b.subset(np.setdiff1d(np.arange(b.n), np.arange(0, b.n, 3)))
    t = gpu_lib.MPT()
    t.set_option("track_dirty", 1)
    t.puts_2phase_with_valuehp(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    t.hash_onepass_v2()
    t.flush_dirty()
    t.deletes(gone.keys_hexs, gone.keys_indexs)
    t.hash_onepass_v2()
    got = dict(t.flush_dirty())
    # every exported node is in the trie of the remaining keys
    o = O.OracleTrie()
    o.puts(keep.keys_hexs, keep.keys_indexs, keep.values, keep.values_indexs)
    o.hash()
    full = dict(o.flush())  # the whole trie of the remaining keys
    assert got and set(got) <= set(full)
    assert all(full[h] == e for h, e in got.items())
    assert t.get_root_hash() == o.root()
    t.close()


def test_flush_dirty_needs_tracking(gpu_lib):
    t = gpu_lib.MPT()
    with pytest.raises(gpu_lib.GmptError):
        t.flush_dirty()
    t.close()
