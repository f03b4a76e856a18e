"""The CPU oracle, pinned before it is trusted (runs without a GPU).

* Keccak-f[1600]: the oracle's SHA3-256 (same permutation, padding 0x06)
  equals Python's hashlib.sha3_256 over seeded lengths 0..5000; its
  Keccak-256 (padding 0x01) equals the reference's own CPUHash::keccak1600.
* Trie: roots and lookups equal the golden vectors produced by the
  reference's own CpuMPT (tests/golden/make_golden.py), and, where
  oracle/_ref is built, further seeded tries run through the reference.
"""
import hashlib

import numpy as np
import pytest

import oracle as O
from conftest import make_batch, nib
from gmpt import workloads as W


def test_keccak_permutation_matches_hashlib_sha3():
    rng = np.random.default_rng(7)
    lengths = list(range(0, 300)) + [543, 544, 1000, 1087, 1088, 1089, 4096, 5000]
    for n in lengths:
        d = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert O.sha3_256(d) == hashlib.sha3_256(d).digest(), n


def test_keccak256_matches_reference_keccak1600():
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    rng = np.random.default_rng(8)
    for n in list(range(0, 280)) + [1000, 4097]:
        d = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert O.keccak256(d) == O.ref_keccak256(d), n


def test_oracle_matches_golden_vectors(golden):
    for case in golden:
        t = O.OracleTrie(O.MODE_REF)
        for b, root in zip(case["batches"], case["roots"]):
            t.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
            t.hash()
            assert t.root() == root, case["name"]
        p = case["probes"]
        assert t.gets(p.keys_hexs, p.keys_indexs) == case["probe_values"], case["name"]


@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_reference_build_on_seeded_tries(seed):
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    rng = W.Xoshiro256ss(1000 + seed)
    n = 50 + int(rng.words(1)[0] % 400)
    alpha = [2, 4, 16, 256][seed % 4]
    keys = [nib(bytes(int(x) % alpha for x in rng.words(1 + int(rng.words(1)[0] % 4)))) for _ in range(n)]
    vals = [rng.bytes(1 + int(rng.words(1)[0] % 70)).tobytes() for _ in range(n)]
    b = make_batch(keys, vals)
    ref = O.RefTrie()
    ref.puts_baseline(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    ref.hash()
    t = O.OracleTrie(O.MODE_REF)
    t.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    t.hash()
    assert t.root() == ref.root()
    assert t.gets(b.keys_hexs, b.keys_indexs) == ref.gets(b.keys_hexs, b.keys_indexs)
    ref.close()


def test_ref_and_geth_modes_agree_when_every_node_is_hashed():
    # 32-byte random keys and 64-byte values: every node encodes to >= 32 B
    b = W.random_keys(3000, seed=0x77)
    a, g = O.OracleTrie(O.MODE_REF), O.OracleTrie(O.MODE_GETH)
    for t in (a, g):
        t.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        t.hash()
    assert a.root() == g.root() and len(a.root()) == 32


def _keccak_rows(rows):
    return np.frombuffer(b"".join(O.keccak256(r.tobytes()) for r in rows), dtype=np.uint8).reshape(len(rows), 32)


@pytest.mark.parametrize("shape", ["ycsb", "vocab", "eth"])
def test_modes_agree_on_the_config_shapes(shape):
    # the other workload shapes (23 B YCSB keys / 100 B values; 8-96 B
    # vocabulary keys / 128 B-4 KB values; Keccak account keys / 71-110 B
    # account RLP): no node encodes below 32 B, so the reference encoding and
    # go-ethereum's give the same root
    from gmpt import eth

    if shape == "ycsb":
        b = W.ycsb_load(4000, seed=0x5EED0002)
    elif shape == "vocab":
        b = W.vocab_keys(1500, seed=0x5EED0004)
    else:
        b = eth.make_state(3000, _keccak_rows, seed=0x5EED0C40).batch
    a, g = O.OracleTrie(O.MODE_REF), O.OracleTrie(O.MODE_GETH)
    for t in (a, g):
        t.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        t.hash()
    assert a.root() == g.root() and len(a.root()) == 32


def test_modes_differ_on_embedded_nodes():
    b = make_batch([nib(b"a"), nib(b"b")], [b"x", b"y"])
    a, g = O.OracleTrie(O.MODE_REF), O.OracleTrie(O.MODE_GETH)
    for t in (a, g):
        t.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        t.hash()
    assert len(g.root()) == 32 and a.root() != g.root()


def test_oracle_rejects_malformed_keys():
    t = O.OracleTrie()
    with pytest.raises(ValueError):
        t.puts(*_flat(make_batch([[1, 17, 16]], [b"v"])))
    with pytest.raises(ValueError):  # terminator not last
        t.puts(*_flat(make_batch([[1, 16, 2]], [b"v"])))
    t2 = O.OracleTrie()
    with pytest.raises(ValueError):  # a key that is a prefix of another (no terminator)
        t2.puts(*_flat(make_batch([[1, 2, 3], [1, 2]], [b"v", b"w"])))


def _flat(b):
    return b.keys_hexs, b.keys_indexs, b.values, b.values_indexs


def test_oracle_reaches_the_committed_config_roots_at_1m():
    # tests/golden/config_roots.json was made by make_config_roots.py with
    # this oracle (and its 1M cases checked against the reference build):
    # the YCSB load + zipf update case at 2^20 keys is re-run here
    import json
    from pathlib import Path

    from gmpt import workloads as W

    cases = json.loads((Path(__file__).resolve().parent / "golden" / "config_roots.json").read_text())["cases"]
    n = 1 << 20
    t = O.OracleTrie()
    got = []
    for b in (W.ycsb_load(n, seed=0x5EED0002), W.ycsb_zipf_updates(n, n, seed=0x5EED0003)):
        t.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        t.hash()
        got.append(t.root().hex())
    assert got == cases["c2_ycsb_1m"]["roots"]
    assert cases["c2_ycsb_1m"]["reference_build_agrees"]


def test_cpu_keccak_rows_matches_single_messages():
    rows = np.random.default_rng(1).integers(0, 256, (37, 20), dtype=np.uint8)
    out = O.keccak256_rows(rows)
    assert [O.keccak256(r.tobytes()) for r in rows] == [o.tobytes() for o in out]


def test_oracle_flush_exports_the_changed_paths_once():
    # two batches: the flush after each exports the nodes on that batch's
    # paths, every exported hash is Keccak-256 of its encoding (or the root's
    # raw encoding), and a flush with no puts in between exports nothing
    b1 = W.random_keys(3000, 32, 40, seed=21)
    b2 = W.random_keys(500, 32, 40, seed=22)
    t = O.OracleTrie()
    t.puts(b1.keys_hexs, b1.keys_indexs, b1.values, b1.values_indexs)
    t.hash()
    f1 = t.flush()
    assert len(f1) == len({h for h, _ in f1})
    for h, enc in f1:
        assert O.keccak256(enc) == h
    root = t.root()
    assert f1[-1][0] == root  # children first: the root comes last
    assert t.flush() == []
    t.puts(b2.keys_hexs, b2.keys_indexs, b2.values, b2.values_indexs)
    t.hash()
    f2 = t.flush()
    assert 0 < len(f2) < len(f1) and f2[-1][0] == t.root()
