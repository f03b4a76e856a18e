"""GPU path vs the oracle, through the C ABI (needs a B200).

Bit-exact bar: every root and every lookup equals the reference's CPU MPT on
the same seeded inputs (golden vectors from the reference itself, and the C
restatement for larger / generated cases).
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from conftest import make_batch, nib
from gmpt import workloads as W

pytestmark = pytest.mark.gpu

STRATEGIES = ["2phase", "latching"]


def put(t, b, strategy, hps=None):
    f = t.puts_2phase_with_valuehp if strategy == "2phase" else t.puts_latching_with_valuehp_v2
    f(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, hps)


def oracle_root(batches, mode=O.MODE_REF):
    t = O.OracleTrie(mode)
    roots = []
    for b in batches:
        t.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        t.hash()
        roots.append(t.root())
    return roots, t


@pytest.mark.parametrize("strategy", STRATEGIES)
def test_golden_roots_and_gets(gpu_lib, golden, strategy):
    for case in golden:
        t = gpu_lib.MPT()
        for b, root in zip(case["batches"], case["roots"]):
            put(t, b, strategy)
            t.hash_onepass_v2()
            assert t.get_root_hash() == root, (case["name"], strategy)
        p = case["probes"]
        assert t.get_values(p.keys_hexs, p.keys_indexs) == case["probe_values"], case["name"]
        t.close()


def test_empty_trie_root_is_empty(gpu_lib):
    t = gpu_lib.MPT()
    t.hash_onepass_v2()
    assert t.get_root_hash() == b""


@pytest.mark.parametrize("mode", [O.MODE_REF, O.MODE_GETH])
@pytest.mark.parametrize("strategy", STRATEGIES)
def test_small_node_tries_both_modes(gpu_lib, mode, strategy):
    rng = W.Xoshiro256ss(42 + mode)
    for trial in range(12):
        n = 1 + int(rng.words(1)[0] % 300)
        alpha = [2, 3, 16, 256][trial % 4]
        keys = [nib(bytes(int(x) % alpha for x in rng.words(1 + int(rng.words(1)[0] % 3)))) for _ in range(n)]
        vals = [rng.bytes(1 + int(rng.words(1)[0] % 40)).tobytes() for _ in range(n)]
        b = make_batch(keys, vals)
        roots, o = oracle_root([b], mode)
        t = gpu_lib.MPT(mode=mode)
        put(t, b, strategy)
        t.hash_onepass_v2()
        assert t.get_root_hash() == roots[0], (trial, strategy, mode)
        assert t.get_values(b.keys_hexs, b.keys_indexs) == o.gets(b.keys_hexs, b.keys_indexs)


@pytest.mark.parametrize("strategy", STRATEGIES + ["mixed"])
def test_incremental_batches_split_existing_nodes(gpu_lib, strategy):
    # keys over a small alphabet so later batches split short nodes of earlier ones
    rng = W.Xoshiro256ss(99)
    batches = []
    for k in range(12):
        n = 5 + int(rng.words(1)[0] % 120)
        keys = [nib(bytes(int(x) % 5 for x in rng.words(2 + int(rng.words(1)[0] % 5)))) for _ in range(n)]
        vals = [rng.bytes(8 + int(rng.words(1)[0] % 50)).tobytes() for _ in range(n)]
        batches.append(make_batch(keys, vals))
    roots, o = oracle_root(batches)
    t = gpu_lib.MPT()
    for k, (b, root) in enumerate(zip(batches, roots)):
        s = strategy if strategy != "mixed" else STRATEGIES[k % 2]
        put(t, b, s)
        t.hash_onepass_v2()
        assert t.get_root_hash() == root, (k, s)
    for b in batches:
        assert t.get_values(b.keys_hexs, b.keys_indexs) == o.gets(b.keys_hexs, b.keys_indexs)


@pytest.mark.parametrize("strategy", STRATEGIES)
def test_two_puts_before_one_hash(gpu_lib, strategy):
    b1 = W.random_keys(500, seed=11)
    b2 = W.random_keys(500, seed=12)
    roots, _ = oracle_root([b1, b2])
    t = gpu_lib.MPT()
    put(t, b1, strategy)
    put(t, b2, strategy)
    t.hash_onepass_v2()
    assert t.get_root_hash() == roots[-1]


@pytest.mark.parametrize("strategy", STRATEGIES)
def test_duplicates_last_write_wins(gpu_lib, strategy):
    base = W.random_keys(64, seed=5)
    idx = np.array([i % 64 for i in range(640)])  # every key 10 times, distinct values
    rng = W.Xoshiro256ss(6)
    keys = [list(base.key(i)) for i in idx]
    vals = [rng.bytes(33).tobytes() for _ in idx]
    b = make_batch(keys, vals)
    roots, o = oracle_root([b])
    t = gpu_lib.MPT()
    put(t, b, strategy)
    t.hash_onepass_v2()
    assert t.get_root_hash() == roots[0]
    got = t.get_values(b.keys_hexs, b.keys_indexs)
    assert got == [vals[576 + (i % 64)] for i in range(640)]


def test_gets_echo_host_pointers_and_absent_keys(gpu_lib):
    b = W.random_keys(300, seed=21)
    hps = np.arange(1, 301, dtype=np.uint64) * 4096
    t = gpu_lib.MPT()
    t.puts_2phase_with_valuehp(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, hps)
    t.hash_onepass_v2()
    got_hp, got_len = t.gets_parallel(b.keys_hexs, b.keys_indexs)
    assert (got_hp == hps).all() and (got_len == 64).all()
    miss = W.random_keys(50, seed=22)
    hp2, len2 = t.gets_parallel(miss.keys_hexs, miss.keys_indexs)
    assert (hp2 == 0).all() and (len2 == 0).all()


@pytest.mark.parametrize("strategy", STRATEGIES)
def test_bad_keys_are_rejected_without_killing_the_trie(gpu_lib, strategy):
    t = gpu_lib.MPT()
    good = W.random_keys(100, seed=31)
    put(t, good, strategy)
    t.hash_onepass_v2()
    root = t.get_root_hash()
    with pytest.raises(gpu_lib.GmptError):
        put(t, make_batch([[1, 2, 20, 16]], [b"v"]), strategy)  # nibble > 16
    with pytest.raises(gpu_lib.GmptError):
        put(t, make_batch([[1, 16, 2, 16]], [b"v"]), strategy)  # terminator not last
    t2 = gpu_lib.MPT()
    put(t2, good, strategy)
    t2.hash_onepass_v2()
    assert t2.get_root_hash() == root


def test_reset_gives_a_fresh_trie(gpu_lib):
    b1 = W.random_keys(400, seed=41)
    b2 = W.ycsb_load(400, seed=42)
    roots, _ = oracle_root([b2])
    t = gpu_lib.MPT()
    t.puts_2phase_with_valuehp(b1.keys_hexs, b1.keys_indexs, b1.values, b1.values_indexs)
    t.hash_onepass_v2()
    t.reset()
    t.puts_2phase_with_valuehp(b2.keys_hexs, b2.keys_indexs, b2.values, b2.values_indexs)
    t.hash_onepass_v2()
    assert t.get_root_hash() == roots[0]


def test_device_resident_inputs_match_host_inputs(gpu_lib):
    import torch

    b = W.ycsb_load(5000, seed=51)
    roots, _ = oracle_root([b])
    dk = torch.from_numpy(b.keys_hexs).cuda()
    di = torch.from_numpy(b.keys_indexs).cuda()
    dv = torch.from_numpy(b.values).cuda()
    dvi = torch.from_numpy(b.values_indexs).cuda()
    for two_phase in (True, False):
        t = gpu_lib.MPT()
        t.puts_device(two_phase, dk.data_ptr(), di.data_ptr(), dv.data_ptr(), dvi.data_ptr(), b.n,
                      b.key_bytes(), b.value_bytes())
        t.hash_onepass_v2()
        assert t.get_root_hash() == roots[0]


def test_reference_c_abi_handle_and_global_calls(gpu_lib):
    L = gpu_lib.lib()
    b = W.random_keys(700, seed=61)
    roots, _ = oracle_root([b])
    kh, ki, vb, vi = (np.ascontiguousarray(x) for x in (b.keys_hexs, b.keys_indexs, b.values, b.values_indexs))
    args = [kh.ctypes.data_as(ctypes.c_void_p), ki.ctypes.data_as(ctypes.c_void_p),
            vb.ctypes.data_as(ctypes.c_void_p), vi.ctypes.data_as(ctypes.c_void_p), None, b.n]
    for fn in (L.insert_mpt_2phase, L.insert_mpt_olc):
        h = L.init_mpt()
        r = fn(h, *args)
        assert r and ctypes.string_at(r, 32) == roots[0]
        L.gmpt_free_buffer(r)
        L.free_mpt(h)
    assert L.preprocess() == 1
    for tt, fn in ((0, L.build_mpt_2phase), (1, L.build_mpt_olc), (2, L.build_mpt_2phase)):
        r = fn(tt, *args)
        assert r and ctypes.string_at(r, 32) == roots[0]
        L.gmpt_free_buffer(r)


def test_get_all_nodes_exports_hash_consistent_encodings(gpu_lib):
    L = gpu_lib.lib()
    assert L.preprocess() == 1
    b = W.random_keys(300, seed=71)
    kh, ki, vb, vi = (np.ascontiguousarray(x) for x in (b.keys_hexs, b.keys_indexs, b.values, b.values_indexs))
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    r = L.build_mpt_2phase(0, P(kh), P(ki), P(vb), P(vi), None, b.n)
    root = ctypes.string_at(r, 32)
    ns = L.get_all_nodes(0, P(kh), P(ki), b.n)
    assert ns.num > b.n  # every leaf plus the branches above them
    hashes = ctypes.string_at(ns.hashs, 32 * ns.num)
    idx = np.ctypeslib.as_array(ctypes.cast(ns.encs_indexs, ctypes.POINTER(ctypes.c_ulonglong)), (2 * ns.num,))
    total = int(idx[-1]) + 1
    encs = ctypes.string_at(ns.encs, total)
    seen_root = False
    for i in range(ns.num):
        enc = encs[idx[2 * i]: idx[2 * i + 1] + 1]
        h = hashes[32 * i: 32 * i + 32]
        assert O.keccak256(enc) == h
        seen_root |= h == root
    assert seen_root
    for p in (ns.hashs, ns.encs, ns.encs_indexs):
        L.gmpt_free_buffer(p)


def test_batched_keccak256_matches_oracle(gpu_lib):
    rng = np.random.default_rng(17)
    msgs = [rng.integers(0, 256, n, dtype=np.uint8).tobytes()
            for n in list(range(0, 300)) + [543, 544, 1087, 1088, 1089, 4096, 5000]]
    assert gpu_lib.keccak256_batch(msgs) == [O.keccak256(m) for m in msgs]


def test_cpp_facade_runs_reference_fixture(gpu_lib, golden, tmp_path):
    import os
    import subprocess
    from pathlib import Path

    repo = Path(__file__).resolve().parents[1]
    exe = tmp_path / "facade_example"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(repo / "include"),
                    str(repo / "tests" / "cpp" / "facade_example.cpp"), "-L", str(gpu_lib.LIB_PATH.parent),
                    "-lgmpt_b200", "-o", str(exe)], check=True)
    env = dict(os.environ, LD_LIBRARY_PATH=str(gpu_lib.LIB_PATH.parent) + ":" + os.environ.get("LD_LIBRARY_PATH", ""))
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr
    doe = [c for c in golden if c["name"] == "doe_dog_dogglesworth"][0]
    assert bytes.fromhex(r.stdout.strip()) == doe["roots"][0]


@pytest.mark.parametrize("local", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_pipeline_knobs_do_not_change_results(gpu_lib, local):
    # device-wide levels vs CTA-local completion of the sort and the build
    rng = W.Xoshiro256ss(1234)
    batches = [W.vocab_keys(3000, seed=77, vmin=40, vmax=300, vmu=4.5),
               W.ycsb_load(6000, seed=78), W.random_keys(5000, seed=79)]
    # small alphabet: deep tries and many ties
    keys = [nib(bytes(int(x) % 3 for x in rng.words(3 + int(rng.words(1)[0] % 9)))) for _ in range(4000)]
    batches.append(make_batch(keys, [rng.bytes(40).tobytes() for _ in keys]))
    roots, o = oracle_root(batches)
    t = gpu_lib.MPT()
    t.set_option("local_build", local[0])
    t.set_option("local_sort", local[1])
    for b, r in zip(batches, roots):
        t.puts_2phase_with_valuehp(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        t.hash_onepass_v2()
        assert t.get_root_hash() == r
    for b in batches:
        assert t.get_values(b.keys_hexs, b.keys_indexs) == o.gets(b.keys_hexs, b.keys_indexs)


@pytest.mark.parametrize("dedup,bits", [(0, 64), (2, 64), (2, 3), (1, 64)])
def test_locknu_dedup_does_not_change_results(gpu_lib, dedup, bits):
    # duplicate-heavy LockNU batches with the repeated-key filter off, on, and
    # on with a 3-bit hash (different keys share hashes: the insert must fall
    # back to walking every key), forest and single trie
    load = W.ycsb_load(20000, seed=81)
    upd = [W.ycsb_zipf_updates(20000, 70000, theta=1.1, seed=82 + k) for k in range(2)]
    roots, o = oracle_root([load] + upd)
    t = gpu_lib.MPT()
    t.set_option("latch_dedup", dedup)
    t.set_option("latch_dedup_bits", bits)
    for b, r in zip([load] + upd, roots):
        t.puts_latching_with_valuehp_v2(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        t.hash_onepass_v2()
        assert t.get_root_hash() == r
    u = upd[-1]
    assert t.get_values(u.keys_hexs, u.keys_indexs) == o.gets(u.keys_hexs, u.keys_indexs)
    # the same keys in two tries of a forest must not be merged by the filter
    f = gpu_lib.MPT(max_tries=2)
    f.set_option("latch_dedup", dedup)
    f.set_option("latch_dedup_bits", bits)
    b = upd[0]
    tids = (np.arange(b.n) % 2).astype(np.int32)
    f.puts_forest(False, b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, tids)
    f.hash_onepass_v2()
    want = []
    for tr in (0, 1):
        ot = O.OracleTrie()
        sub = b.subset(np.nonzero(tids == tr)[0])
        ot.puts(sub.keys_hexs, sub.keys_indexs, sub.values, sub.values_indexs)
        ot.hash()
        want.append(ot.root())
    assert f.get_roots(n=2) == want


def test_key_streams_with_gaps_between_keys(gpu_lib):
    # index pairs need not tile the key stream; bytes between keys are ignored
    b = W.random_keys(2000, seed=91)
    gap = 3
    kh = np.zeros(len(b.keys_hexs) + gap * b.n, dtype=np.uint8) + 0xEE  # junk > 16 in the gaps
    ki = np.zeros_like(b.keys_indexs)
    for i in range(b.n):
        s, e = b.keys_indexs[2 * i], b.keys_indexs[2 * i + 1]
        ns = s + gap * (i + 1)
        kh[ns: ns + (e - s + 1)] = b.keys_hexs[s: e + 1]
        ki[2 * i], ki[2 * i + 1] = ns, ns + (e - s)
    roots, _ = oracle_root([b])
    for strategy in STRATEGIES:
        t = gpu_lib.MPT()
        f = t.puts_2phase_with_valuehp if strategy == "2phase" else t.puts_latching_with_valuehp_v2
        f(kh, ki, b.values, b.values_indexs)
        t.hash_onepass_v2()
        assert t.get_root_hash() == roots[0]
        bad = kh.copy()
        bad[ki[10] + 5] = 16  # a terminator inside a key
        with pytest.raises(gpu_lib.GmptError):
            f(bad, ki, b.values, b.values_indexs)


@pytest.mark.parametrize("strategies", [(1, 0, 0, 1), (0, 0, 1, 1), (1, 1, 1, 1)])
def test_pipelined_host_batches(gpu_lib, strategies):
    # next batch's copy overlaps this batch's insert + hash; roots after every
    # batch, lookups and echoed host pointers must be as if run one by one
    batches = [W.ycsb_load(30000, seed=201), W.ycsb_zipf_updates(30000, 40000, seed=202),
               W.vocab_keys(20000, seed=203, vmin=40, vmax=300, vmu=4.5),
               W.ycsb_zipf_updates(30000, 25000, theta=0.5, seed=204)]
    roots, o = oracle_root(batches)
    t = gpu_lib.MPT()
    hps = [np.arange(b.n, dtype=np.uint64) + 1000 * (k + 1) for k, b in enumerate(batches)]
    got = t.puts_pipeline(batches, [bool(x) for x in strategies], hps=hps)
    assert got == roots
    last = batches[-1]
    assert t.get_values(last.keys_hexs, last.keys_indexs) == o.gets(last.keys_hexs, last.keys_indexs)
    h, sizes = t.gets_parallel(last.keys_hexs, last.keys_indexs)
    # a key's echoed pointer is the one given with the last batch position that wrote it
    assert np.all(sizes > 0) and np.all(h >= 1000)


@pytest.mark.parametrize("mode,bits", [(0, 64), (1, 64), (2, 64), (2, 3)])
def test_phasenu_repeat_filter_does_not_change_results(gpu_lib, mode, bits):
    # PhaseNU batches heavy with repeated keys (70000 zipf updates of 20000
    # keys: the 1 % sample trigger fires), with the repeat filter off,
    # sampled, forced, and forced with a 3-bit hash (different keys share
    # hashes: the sort must fall back to the whole batch); then a forest
    load = W.ycsb_load(20000, seed=91)
    upd = [W.ycsb_zipf_updates(20000, 70000, theta=1.1, seed=92 + k) for k in range(2)]
    roots, o = oracle_root([load] + upd)
    t = gpu_lib.MPT()
    t.set_option("sort_dedup", mode)
    t.set_option("latch_dedup_bits", bits)
    for b, r in zip([load] + upd, roots):
        t.puts_2phase_with_valuehp(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        t.hash_onepass_v2()
        assert t.get_root_hash() == r
    u = upd[-1]
    assert t.get_values(u.keys_hexs, u.keys_indexs) == o.gets(u.keys_hexs, u.keys_indexs)
    f = gpu_lib.MPT(max_tries=2)
    f.set_option("sort_dedup", mode)
    f.set_option("latch_dedup_bits", bits)
    b = upd[0]
    tids = (np.arange(b.n) % 2).astype(np.int32)
    f.puts_forest(True, b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, tids)
    f.hash_onepass_v2()
    want = []
    for tr in (0, 1):
        ot = O.OracleTrie()
        sub = b.subset(np.nonzero(tids == tr)[0])
        ot.puts(sub.keys_hexs, sub.keys_indexs, sub.values, sub.values_indexs)
        ot.hash()
        want.append(ot.root())
    assert f.get_roots(n=2) == want
