"""Forests (many tries in one object) vs one oracle trie per trie id.

Every trie of a forest must come out exactly as if it had been built alone:
same root in both encode modes, same lookups, whatever the interleaving of
trie ids inside a batch and whichever insert strategy ran.
"""
import numpy as np
import pytest

import oracle as O
from conftest import make_batch, nib
from gmpt import workloads as W

pytestmark = pytest.mark.gpu


def forest_batch(rng, n_tries, n_keys, alpha, max_len, dup_every=7):
    """A shuffled batch over n_tries tries; every 7th key repeats an earlier one."""
    keys, vals, tids = [], [], []
    for i in range(n_keys):
        if i and i % dup_every == 0:
            j = int(rng.words(1)[0] % i)
            keys.append(keys[j])
            tids.append(tids[j])
        else:
            ln = 1 + int(rng.words(1)[0] % max_len)
            keys.append(nib(bytes(int(x) % alpha for x in rng.words(ln))))
            # power-law-ish trie choice: low ids get most keys
            u = (int(rng.words(1)[0]) >> 11) / float(1 << 53)
            tids.append(min(n_tries - 1, int(n_tries * u * u)))
        vals.append(rng.bytes(1 + int(rng.words(1)[0] % 60)).tobytes())
    return keys, vals, np.array(tids, np.int32)


def oracle_forest(oracles, keys, vals, tids, mode):
    for t in sorted(set(tids.tolist())):
        sel = [i for i in range(len(keys)) if tids[i] == t]
        b = make_batch([keys[i] for i in sel], [vals[i] for i in sel])
        if t not in oracles:
            oracles[t] = O.OracleTrie(mode)
        oracles[t].puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        oracles[t].hash()


def oracle_roots(oracles, n_tries):
    return [oracles[t].root() if t in oracles else b"" for t in range(n_tries)]


@pytest.mark.parametrize("mode", [O.MODE_REF, O.MODE_GETH])
@pytest.mark.parametrize("strategies", [("2phase", "2phase"), ("latching", "latching"), ("2phase", "latching"),
                                        ("latching", "2phase")])
def test_forest_roots_match_per_trie_oracle(gpu_lib, mode, strategies):
    rng = W.Xoshiro256ss(0xF0 + 3 * mode + len(strategies[0]))
    n_tries = 40
    f = gpu_lib.MPT(mode=mode, max_tries=n_tries)
    oracles = {}
    for step, strategy in enumerate(strategies):
        keys, vals, tids = forest_batch(rng, n_tries, 600 + 400 * step, alpha=[4, 16][step], max_len=6)
        b = make_batch(keys, vals)
        f.puts_forest(strategy == "2phase", b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, tids)
        f.hash_onepass_v2()
        oracle_forest(oracles, keys, vals, tids, mode)
        assert f.get_roots(n=n_tries) == oracle_roots(oracles, n_tries), (step, strategy)
    # lookups through the forest, per trie
    keys, vals, tids = forest_batch(rng, n_tries, 300, alpha=4, max_len=6)
    probes = make_batch(keys, vals)
    hps, sizes = f.gets_forest(probes.keys_hexs, probes.keys_indexs, tids)
    for i in range(len(keys)):
        t = int(tids[i])
        want = None
        if t in oracles:
            pb = make_batch([keys[i]], [b"x"])
            want = oracles[t].gets(pb.keys_hexs, pb.keys_indexs)[0]
        assert sizes[i] == (0 if want is None else len(want)), i
    f.close()


def test_forest_trie0_is_the_single_trie_api(gpu_lib):
    rng = W.Xoshiro256ss(0xF7)
    f = gpu_lib.MPT(max_tries=3)
    keys, vals, tids = forest_batch(rng, 3, 500, alpha=16, max_len=5)
    b = make_batch(keys, vals)
    f.puts_forest(True, b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, tids)
    f.hash_onepass_v2()
    oracles = {}
    oracle_forest(oracles, keys, vals, tids, O.MODE_REF)
    assert f.get_root_hash() == oracles[0].root()
    # a plain single-trie put lands in trie 0 only
    keys2 = [nib(bytes([9, 9, i])) for i in range(20)]
    vals2 = [bytes([i]) * 40 for i in range(20)]
    b2 = make_batch(keys2, vals2)
    f.puts_latching_with_valuehp_v2(b2.keys_hexs, b2.keys_indexs, b2.values, b2.values_indexs)
    f.hash_onepass_v2()
    oracle_forest(oracles, keys2, vals2, np.zeros(20, np.int32), O.MODE_REF)
    assert f.get_roots(n=3) == oracle_roots(oracles, 3)
    assert f.get_roots([2, 0]) == [oracles[2].root(), oracles[0].root()]


def test_forest_same_keys_in_every_trie(gpu_lib):
    # identical key sets in different tries must not merge
    n_tries = 16
    f = gpu_lib.MPT(mode=O.MODE_GETH, max_tries=n_tries)
    keys, vals, tids = [], [], []
    for t in range(n_tries):
        for k in range(t + 1):
            keys.append(nib(bytes([k, 0xAB])))
            vals.append(bytes([t, k]) * (1 + t))
            tids.append(t)
    perm = np.random.default_rng(5).permutation(len(keys))
    keys = [keys[i] for i in perm]
    vals = [vals[i] for i in perm]
    tids = np.array([tids[i] for i in perm], np.int32)
    for two_phase in (True, False):
        f.reset()
        b = make_batch(keys, vals)
        f.puts_forest(two_phase, b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, tids)
        f.hash_onepass_v2()
        oracles = {}
        oracle_forest(oracles, keys, vals, tids, O.MODE_GETH)
        assert f.get_roots(n=n_tries) == oracle_roots(oracles, n_tries), two_phase


def test_forest_bad_trie_id(gpu_lib):
    f = gpu_lib.MPT(max_tries=4)
    b = make_batch([nib(b"\x01"), nib(b"\x02")], [b"a" * 40, b"b" * 40])
    for two_phase in (True, False):
        with pytest.raises(gpu_lib.GmptError):
            f.puts_forest(two_phase, b.keys_hexs, b.keys_indexs, b.values, b.values_indexs,
                          np.array([0, 4], np.int32))
    with pytest.raises(gpu_lib.GmptError):
        f.get_roots([5])
    # the object stays usable
    f.puts_forest(True, b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, np.array([1, 3], np.int32))
    f.hash_onepass_v2()
    r = f.get_roots(n=4)
    assert r[0] == b"" and r[2] == b"" and len(r[1]) == 32 and len(r[3]) == 32
