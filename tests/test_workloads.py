"""Seeded synthetic workloads: deterministic and of the stated shapes."""
import numpy as np

from gmpt import workloads as W


def test_xoshiro_deterministic():
    a = W.Xoshiro256ss(5).words(1000)
    b = W.Xoshiro256ss(5).words(1000)
    assert (a == b).all() and len(np.unique(a)) == 1000


def test_random_keys_shape():
    b = W.random_keys(100, 32, 64, seed=1)
    assert b.n == 100 and len(b.key(0)) == 65 and b.key(0)[-1] == 16 and len(b.value(0)) == 64
    assert (b.keys_hexs[b.keys_indexs[1::2]] == 16).all()


def test_ycsb_keys_format():
    kb = W.ycsb_key_bytes(np.arange(4, dtype=np.uint64)).reshape(4, 23).tobytes()
    for i in range(4):
        k = kb[23 * i: 23 * i + 23]
        assert k[:4] == b"user" and k[4:].isdigit()


def test_zipf_updates_hit_loaded_keys():
    load = W.ycsb_load(2000, seed=3)
    up = W.ycsb_zipf_updates(2000, 3000, seed=4)
    loaded = {load.key(i) for i in range(load.n)}
    keys = [up.key(i) for i in range(up.n)]
    assert all(k in loaded for k in keys)
    assert len(set(keys)) < up.n  # duplicates present


def test_vocab_keys_lengths():
    b = W.vocab_keys(2000, seed=5)
    lens = (b.keys_indexs[1::2] - b.keys_indexs[0::2] + 1 - 1) // 2
    assert lens.min() >= 8 and lens.max() <= 96
    vl = b.values_indexs[1::2] - b.values_indexs[0::2] + 1
    assert vl.min() >= 128 and vl.max() <= 4096
