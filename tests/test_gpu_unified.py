"""Unified-memory tries (gmpt_create_ex with GMPT_CREATE_UNIFIED_MEMORY, the
reference's out-of-core UMMPT, mpt/um_mpt.cuh:13-52): the same roots and
lookups as device-memory tries, under both insert strategies, PhaseHC, a
persistent block update and deletes."""
import numpy as np
import pytest

import oracle as O
from gmpt import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("strategy", ["2phase", "latching"])
def test_unified_memory_trie_matches_the_oracle(gpu_lib, strategy):
    n = 1 << 17
    load = W.ycsb_load(n, seed=0x5EED0002)
    upd = W.ycsb_zipf_updates(n, n, seed=0x5EED0003)
    o = O.OracleTrie()
    tries = [gpu_lib.MPT(unified=True), gpu_lib.MPT()]
    for b in (load, upd):
        o.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        o.hash()
        for t in tries:
            f = t.puts_2phase_with_valuehp if strategy == "2phase" else t.puts_latching_with_valuehp_v2
            f(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
            t.hash_onepass_v2()
            assert t.get_root_hash() == o.root()
    s = upd.subset(W.sample_indices(n, 2048))
    assert tries[0].get_values(s.keys_hexs, s.keys_indexs) == o.gets(s.keys_hexs, s.keys_indexs)
    # deletes: the unified trie and the device-memory trie stay equal
    gone = load.subset(np.arange(0, n, 5))
    for t in tries:
        t.deletes(gone.keys_hexs, gone.keys_indexs)
        t.hash_onepass_v2()
    assert tries[0].get_root_hash() == tries[1].get_root_hash() != o.root()
    for t in tries:
        t.close()


def test_unified_memory_block_update_matches_device_memory(gpu_lib):
    b = W.random_keys(1 << 15, 32, 40, seed=0x5EED0F20)
    tid = np.zeros(b.n, np.int32)
    roots = []
    for unified in (False, True):
        t = gpu_lib.MPT(mode=gpu_lib.MODE_GETH, unified=unified)
        roots.append(t.block_update(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, tid, b.n, [0]))
        t.close()
    assert roots[0] == roots[1] and len(roots[0][0]) == 32


def test_unknown_creation_flags_are_rejected(gpu_lib):
    L = gpu_lib.lib()
    assert not L.gmpt_create_ex(0, 0, 1, 6)
    assert L.gmpt_last_error() == 5
