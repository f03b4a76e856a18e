"""The benchmark configurations at their own shapes and sizes, against oracle
roots computed on the CPU (tests/golden/config_roots.json, made by
tests/golden/make_config_roots.py from the C restatement of the reference
CPU MPT; its 1M-key cases also agree with the reference's own CpuMPT).

* variable-length vocabulary keys (8-96 B) with 128 B - 4 KB values: leaves
  of 1 to 31 Keccak blocks, deep short-node splits -- at 2^20 and 8M keys,
  through both insert strategies, plus lookups of sampled keys;
* the Ethereum-shaped forest at 2^20 accounts: 16 blocks through the
  persistent block launch, every block's state root and a digest of all the
  roots it returns.
"""
import numpy as np
import pytest

import oracle as O
from conftest import last_occurrence
from gmpt import eth
from gmpt import workloads as W

pytestmark = pytest.mark.gpu


def put(t, strategy, b):
    f = t.puts_2phase_with_valuehp if strategy == "2phase" else t.puts_latching_with_valuehp_v2
    f(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    t.hash_onepass_v2()


@pytest.fixture(scope="module")
def vocab_1m():
    return W.vocab_keys(1 << 20)


@pytest.mark.parametrize("strategy", ["2phase", "latching"])
def test_vocab_keys_1m_large_values_match_oracle(gpu_lib, config_roots, vocab_1m, strategy):
    b = vocab_1m
    sizes = b.values_indexs[1::2] - b.values_indexs[0::2] + 1
    assert sizes.min() >= 128 and sizes.max() == 4096  # leaves up to 31 Keccak blocks
    t = gpu_lib.MPT()
    put(t, strategy, b)
    assert t.get_root_hash() == bytes.fromhex(config_roots["c3_vocab_1m"]["roots"][0])
    # lookups return the value of each key's last occurrence in the batch
    idx = W.sample_indices(b.n, 4096, seed=11)
    probe = b.subset(idx)
    want = [b.value(int(j)) for j in last_occurrence(b, idx)]
    assert t.get_values(probe.keys_hexs, probe.keys_indexs) == want
    t.close()


def test_vocab_keys_1m_geth_mode_same_root(gpu_lib, config_roots, vocab_1m):
    # no node of this shape encodes below 32 bytes, so both encodings agree
    t = gpu_lib.MPT(mode=gpu_lib.MODE_GETH)
    put(t, "2phase", vocab_1m)
    assert t.get_root_hash() == bytes.fromhex(config_roots["c3_vocab_1m"]["roots"][0])
    t.close()


def test_vocab_keys_8m_matches_oracle_in_both_strategies(gpu_lib, config_roots):
    b = W.vocab_keys(8 << 20)
    want = bytes.fromhex(config_roots["c3_vocab_8m"]["roots"][0])
    for strategy in ("2phase", "latching"):
        t = gpu_lib.MPT()
        put(t, strategy, b)
        assert t.get_root_hash() == want, strategy
        t.close()


def test_vocab_keys_split_into_two_batches(gpu_lib, config_roots, vocab_1m):
    # the same keys as a load and a second batch into the existing trie
    # (PhaseNU walk + splits, LockNU CAS splits) end at the same root
    b = vocab_1m
    h = b.n // 2
    first, second = b.subset(np.arange(h)), b.subset(np.arange(h, b.n))
    want = bytes.fromhex(config_roots["c3_vocab_1m"]["roots"][0])
    for s1, s2 in (("2phase", "2phase"), ("latching", "2phase"), ("2phase", "latching")):
        t = gpu_lib.MPT()
        put(t, s1, first)
        put(t, s2, second)
        assert t.get_root_hash() == want, (s1, s2)
        t.close()


def test_ethereum_blocks_1m_accounts_match_oracle(gpu_lib, config_roots):
    case = config_roots["c4_eth_1m"]
    state = eth.make_state(case["accounts"], gpu_lib.keccak256_rows)
    f = gpu_lib.MPT(mode=gpu_lib.MODE_GETH, max_tries=1 << 14)
    b = state.batch
    f.puts_2phase_with_valuehp(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    f.hash_onepass_v2()
    assert f.get_root_hash().hex() == case["state_root"]
    gen = eth.EthBlocks(state, gpu_lib.keccak256_rows)
    for k, want in enumerate(case["blocks"]):
        blk = gen.next()
        assert blk.n == want["keys"]
        roots = eth.apply_block(f, blk)
        assert len(roots) == want["tries"]
        assert roots[0].hex() == want["state_root"], k
        digest = O.keccak256(b"".join(r[:32].ljust(32, b"\0") for r in roots))
        assert digest.hex() == want["roots_digest"], k
    f.close()
