"""Persistent block updates (gmpt_block_update) on an Ethereum-shaped forest.

Every root a block returns -- the state root and each touched account's
storage root -- must equal the oracle's, where the oracle builds one trie
per storage trie, writes each storage root into its account's RLP value, and
then updates the state trie.  The one-launch path must also agree with the
per-trie and forest multi-launch paths block after block.
"""
import numpy as np
import pytest

import oracle as O
from gmpt import eth
from gmpt import workloads as W

pytestmark = pytest.mark.gpu


class OracleForest:
    def __init__(self, state: eth.EthState, mode):
        self.mode = mode
        self.state = O.OracleTrie(mode)
        b = state.batch
        self.state.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        self.state.hash()
        self.storage = {}

    def apply(self, blk: eth.EthBlock):
        b = blk.batch
        roots = {}
        for j, sid in enumerate(blk.storage_ids.tolist()):
            sub = b.subset(np.arange(blk.spans[j], blk.spans[j + 1]))
            t = self.storage.setdefault(sid, O.OracleTrie(self.mode))
            t.puts(sub.keys_hexs, sub.keys_indexs, sub.values, sub.values_indexs)
            t.hash()
            roots[sid] = t.root()
        vb = eth.patched_values(blk, roots)
        acc = W.Batch(b.keys_hexs, b.keys_indexs, vb, b.values_indexs).subset(np.arange(blk.n0, blk.n))
        self.state.puts(acc.keys_hexs, acc.keys_indexs, acc.values, acc.values_indexs)
        self.state.hash()
        return [self.state.root()] + [roots[s] for s in blk.storage_ids.tolist()]


def _forest(gpu_lib, state, mode, max_tries=1 << 14):
    f = gpu_lib.MPT(mode=mode, max_tries=max_tries)
    b = state.batch
    f.puts_2phase_with_valuehp(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    f.hash_onepass_v2()
    return f


@pytest.fixture(scope="module")
def small_state(gpu_lib):
    return eth.make_state(4000, gpu_lib.keccak256_rows)


@pytest.mark.parametrize("mode", [O.MODE_GETH, O.MODE_REF])
def test_blocks_match_oracle(gpu_lib, small_state, mode):
    f = _forest(gpu_lib, small_state, mode)
    ora = OracleForest(small_state, mode)
    assert f.get_root_hash() == ora.state.root()
    gen = eth.EthBlocks(small_state, gpu_lib.keccak256_rows, min_updates=20, max_updates=60, max_storage=400)
    for k in range(5):
        blk = gen.next()
        got = eth.apply_block(f, blk)
        want = ora.apply(blk)
        assert got == want, k
        info = f.block_info()
        assert info["levels"][0] > 0 and info["levels"][1] > 0 and info["dirty"][1] > 0
    # later blocks replay the captured graph (one capture, unless a pool grew)
    assert f.block_info()["launches"] == 5 and f.block_info()["captures"] <= 5


def test_block_paths_agree(gpu_lib, small_state):
    fa = _forest(gpu_lib, small_state, O.MODE_GETH)
    fb = _forest(gpu_lib, small_state, O.MODE_GETH)
    fc = _forest(gpu_lib, small_state, O.MODE_GETH)
    fd = _forest(gpu_lib, small_state, O.MODE_GETH)
    fd.set_option("block_graph", 0)
    fd.set_option("block_grid", 7)
    gen = eth.EthBlocks(small_state, gpu_lib.keccak256_rows, min_updates=30, max_updates=80, max_storage=2000)
    for k in range(6):
        blk = gen.next()
        ra = eth.apply_block(fa, blk)
        assert eth.apply_plain(fb, blk) == ra, k
        assert eth.apply_forest(fc, blk, two_phase=(k % 2 == 0)) == ra, k
        assert eth.apply_block(fd, blk) == ra, k
    assert fd.block_info()["grid"] == 7 and fd.block_info()["captures"] == 0


def test_block_with_no_keys_reports_roots(gpu_lib, small_state):
    f = _forest(gpu_lib, small_state, O.MODE_GETH)
    z8, z32, z64 = np.zeros(0, np.uint8), np.zeros(0, np.int32), np.zeros(0, np.int64)
    r = f.block_update(z8, z32, z8, z64, z32, 0, [0, 1, 2])
    assert r[0] == f.get_root_hash() and r[1] == b"" and r[2] == b""


def test_block_rejects_bad_inputs(gpu_lib, small_state):
    f = _forest(gpu_lib, small_state, O.MODE_GETH, max_tries=1000)
    gen = eth.EthBlocks(small_state, gpu_lib.keccak256_rows, min_updates=10, max_updates=20, max_storage=50)
    blk = gen.next()
    b = blk.batch
    root0 = f.get_root_hash()

    def call(**kw):
        a = dict(trie_ids=blk.trie_ids, n0=blk.n0, patch_trie=blk.patch_trie, patch_off=blk.patch_off)
        a.update(kw)
        return f.block_update(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, a["trie_ids"], a["n0"],
                              blk.out_ids, a["patch_trie"], a["patch_off"])

    bad_tid = blk.trie_ids.copy()
    bad_tid[3] = 5000
    with pytest.raises(gpu_lib.GmptError):
        call(trie_ids=bad_tid)
    bad_pt = blk.patch_trie.copy()
    bad_pt[0] = 1  # a stage-0 key may not be patched
    with pytest.raises(gpu_lib.GmptError):
        call(patch_trie=bad_pt)
    bad_po = blk.patch_off.copy()
    bad_po[-1] += 40  # root would run past the value
    with pytest.raises(gpu_lib.GmptError):
        call(patch_off=bad_po)
    bad_keys = b.keys_hexs.copy()
    bad_keys[5] = 17
    with pytest.raises(gpu_lib.GmptError):
        f.block_update(bad_keys, b.keys_indexs, b.values, b.values_indexs, blk.trie_ids, blk.n0, blk.out_ids,
                       blk.patch_trie, blk.patch_off)
    assert f.get_root_hash() == root0  # nothing was applied
    # still usable, and the block then matches the oracle
    ora = OracleForest(small_state, O.MODE_GETH)
    assert eth.apply_block(f, blk) == ora.apply(blk)
