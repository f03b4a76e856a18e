"""Full-size parity (needs a B200): the bulk-load configuration against the
oracle, and size-independent properties on the 16M-key YCSB configuration."""
import numpy as np
import pytest

import oracle as O
from gmpt import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("strategy", ["2phase", "latching"])
def test_random32_2pow20_root_and_4096_gets(gpu_lib, strategy):
    b = W.random_keys(1 << 20, 32, 64, seed=0x5EED0001)
    o = O.OracleTrie()
    o.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    o.hash()
    t = gpu_lib.MPT()
    f = t.puts_2phase_with_valuehp if strategy == "2phase" else t.puts_latching_with_valuehp_v2
    f(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    t.hash_onepass_v2()
    assert t.get_root_hash() == o.root()
    s = b.subset(W.sample_indices(b.n, 4096))
    assert t.get_values(s.keys_hexs, s.keys_indexs) == o.gets(s.keys_hexs, s.keys_indexs)


def test_ycsb_load_then_zipf_updates_matches_oracle_at_256k(gpu_lib):
    n = 1 << 18
    load = W.ycsb_load(n, seed=0x5EED0002)
    upd = W.ycsb_zipf_updates(n, n, seed=0x5EED0003)
    o = O.OracleTrie()
    roots = []
    for b in (load, upd):
        o.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        o.hash()
        roots.append(o.root())
    for strategies in (("2phase", "2phase"), ("2phase", "latching"), ("latching", "latching")):
        t = gpu_lib.MPT()
        for b, s, r in zip((load, upd), strategies, roots):
            f = t.puts_2phase_with_valuehp if s == "2phase" else t.puts_latching_with_valuehp_v2
            f(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
            t.hash_onepass_v2()
            assert t.get_root_hash() == r, strategies


def test_ycsb_16m_matches_oracle_roots_and_order_does_not_matter(gpu_lib, config_roots):
    # The full 16M configuration: the load root and the load + update root
    # equal the oracle's (tests/golden/config_roots.json, made by
    # tests/golden/make_config_roots.py) for both insert strategies; then
    # size-independent properties: inserting the batch in a permuted order
    # gives the same root (canonical trie), and sampled lookups return the
    # last written value.
    n = 1 << 24
    want = [bytes.fromhex(r) for r in config_roots["c2_ycsb_16m"]["roots"]]
    load = W.ycsb_load(n, seed=0x5EED0002)
    upd = W.ycsb_zipf_updates(n, n, seed=0x5EED0003)
    roots = {}
    for s in ("2phase", "latching"):
        t = gpu_lib.MPT()
        got = []
        for b in (load, upd):
            f = t.puts_2phase_with_valuehp if s == "2phase" else t.puts_latching_with_valuehp_v2
            f(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
            t.hash_onepass_v2()
            got.append(t.get_root_hash())
        assert got == want, s
        roots[s] = t.get_root_hash()
        if s == "2phase":
            idx = W.sample_indices(n, 4096, seed=9)
            probe = upd.subset(idx)
            got = t.get_values(probe.keys_hexs, probe.keys_indexs)
            # expected: the value at the last occurrence of each key in the batch
            rows = upd.keys_hexs.reshape(n, -1)  # fixed-length keys
            rv = np.ascontiguousarray(rows[::-1]).view(np.dtype((np.void, rows.shape[1]))).ravel()
            uniq, first_rev = np.unique(rv, return_index=True)
            pr = np.ascontiguousarray(rows[idx]).view(np.dtype((np.void, rows.shape[1]))).ravel()
            last = n - 1 - first_rev[np.searchsorted(uniq, pr)]
            exp = [upd.value(int(i)) for i in last]
            assert got == exp
        t.close()
    assert roots["2phase"] == roots["latching"] and len(roots["2phase"]) == 32
    perm = np.random.default_rng(3).permutation(n)
    shuffled = load.subset(perm)
    t = gpu_lib.MPT()
    t.puts_2phase_with_valuehp(shuffled.keys_hexs, shuffled.keys_indexs, shuffled.values, shuffled.values_indexs)
    t.hash_onepass_v2()
    t2 = gpu_lib.MPT()
    t2.puts_latching_with_valuehp_v2(load.keys_hexs, load.keys_indexs, load.values, load.values_indexs)
    t2.hash_onepass_v2()
    assert t.get_root_hash() == t2.get_root_hash()
