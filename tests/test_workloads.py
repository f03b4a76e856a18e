"""Seeded synthetic workloads: deterministic and of the stated shapes."""
import numpy as np
import pytest

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


# -- Ethereum-shaped forest workload -------------------------------------------

def _oracle_keccak_rows(msgs):
    import oracle as O

    return np.array([np.frombuffer(O.keccak256(m.tobytes()), np.uint8) for m in msgs]).reshape(-1, 32)


def _rlp_items(buf: bytes):
    """Decode one RLP list of short strings (enough for accounts)."""
    assert buf[0] == 0xF8 and buf[1] == len(buf) - 2
    items, p = [], 2
    while p < len(buf):
        h = buf[p]
        assert 0x80 <= h <= 0xB7
        items.append(buf[p + 1: p + 1 + h - 0x80])
        p += 1 + h - 0x80
    assert p == len(buf)
    return items


def test_empty_root_constant_is_keccak_of_empty_rlp():
    import oracle as O
    from gmpt import eth

    assert eth.EMPTY_ROOT == O.keccak256(b"\x80")


def test_account_values_are_rlp_accounts():
    from gmpt import eth

    rng = W.Xoshiro256ss(3)
    roots = rng.bytes(32 * 500).reshape(500, 32)
    vb, vi, roff = eth.account_values(rng, 500, roots)
    for i in range(500):
        v = vb[vi[2 * i]: vi[2 * i + 1] + 1].tobytes()
        assert 71 <= len(v) <= 110
        nonce, balance, sroot, code = _rlp_items(v)
        assert len(sroot) == 32 and len(code) == 32 and 1 <= len(balance) <= 32 and len(nonce) <= 8
        assert v[roff[i]: roff[i] + 32] == roots[i].tobytes() == sroot
        if len(balance) == 1:
            assert balance[0] >= 0x80
        elif balance:
            assert balance[0] != 0


def test_power_law_sizes_range_and_skew():
    from gmpt import eth

    s = eth.power_law_sizes(W.Xoshiro256ss(4), 200000)
    assert s.min() >= 1 and s.max() <= 5000
    # density ~ s^-1.5 on [1, 5000]: mean ~ 70, median ~ 3.9
    assert 55 < s.mean() < 90 and 2 <= np.median(s) <= 6


def test_eth_block_layout():
    from gmpt import eth

    st = eth.make_state(500, _oracle_keccak_rows)
    gen = eth.EthBlocks(st, _oracle_keccak_rows, min_updates=5, max_updates=12, max_storage=40)
    seen = set()
    for _ in range(3):
        blk = gen.next()
        b = blk.batch
        assert blk.n0 == int(blk.spans[-1]) and blk.n == blk.n0 + len(blk.accounts)
        assert np.all(blk.patch_trie[: blk.n0] == -1) and np.all(blk.trie_ids[blk.n0:] == 0)
        assert np.all(blk.patch_trie[blk.n0:] == blk.storage_ids)
        assert len(set(blk.storage_ids.tolist())) == len(blk.storage_ids) and 0 not in set(blk.storage_ids.tolist())
        for j in range(len(blk.accounts)):
            a, z = blk.spans[j], blk.spans[j + 1]
            assert np.all(blk.trie_ids[a:z] == blk.storage_ids[j])
        # index pairs tile both streams
        assert b.keys_indexs[0] == 0 and np.all(b.keys_indexs[2::2] == b.keys_indexs[1:-1:2] + 1)
        assert b.values_indexs[0] == 0 and np.all(b.values_indexs[2::2] == b.values_indexs[1:-1:2] + 1)
        for j in range(blk.n0, blk.n):
            ln = b.values_indexs[2 * j + 1] - b.values_indexs[2 * j] + 1
            assert blk.patch_off[j] == ln - 65
        # an account keeps its storage trie id across blocks
        for a, s in zip(blk.accounts.tolist(), blk.storage_ids.tolist()):
            assert gen.sid_of[a] == s
            seen.add(a)


def test_keys_to_hexs_fixed_and_ragged_paths_agree_with_per_key_expansion():
    from conftest import nib

    rng = W.Xoshiro256ss(11)
    for lens in (np.full(50, 7), np.array([3, 1, 9, 9, 2, 16, 5] * 5)):
        kb = rng.bytes(int(lens.sum()))
        kh, ki = W.keys_to_hexs(kb, lens)
        pos = 0
        for i, ln in enumerate(lens.tolist()):
            want = nib(kb[pos: pos + ln].tobytes())
            pos += ln
            assert kh[ki[2 * i]: ki[2 * i + 1] + 1].tolist() == want


def test_request_groups_keep_each_tenants_order():
    from gmpt import serve as S

    tenants = S.make_tenants([10, 10, 10, 10])
    reqs = S.make_stream(5, 200, tenants, 0.5, 10, 100, load_frac=0.2)
    groups = S._groups(reqs)
    assert sorted(r.i for g in groups for r in g) == [r.i for r in reqs]
    for g in groups:
        assert len({r.kind for r in g}) == 1
    # per tenant, the order of its requests is unchanged
    seen = {}
    for g in groups:
        for r in g:
            seen.setdefault(r.tenant, []).append(r.i)
    for t, order in seen.items():
        assert order == sorted(order)
    assert len(groups) < len(reqs)


def test_hexs_to_keys_inverts_keys_to_hexs():
    rng = np.random.default_rng(11)
    for lens in (np.full(50, 23), rng.integers(0, 9, 200)):
        kb = rng.integers(0, 256, int(lens.sum()), dtype=np.uint8)
        kh, ki = W.keys_to_hexs(kb, lens)
        raw, ri = W.hexs_to_keys(kh, ki)
        assert np.array_equal(raw, kb)
        assert np.array_equal(ri[1::2] - ri[0::2] + 1, lens)
    with pytest.raises(ValueError):
        W.hexs_to_keys(np.array([1, 2, 3, 16], np.uint8), np.array([0, 3], np.int32))


def test_last_occurrence_helper_matches_a_dictionary():
    from conftest import last_occurrence

    b = W.vocab_keys(20000, vmin=1, vmax=8, vmu=1.0)
    last = {}
    for i in range(b.n):
        last[b.key(i)] = i
    idx = W.sample_indices(b.n, 500, seed=5)
    got = last_occurrence(b, idx)
    assert [last[b.key(int(i))] for i in idx] == got.tolist()
    assert any(g != i for g, i in zip(got, idx))  # the sample holds repeated keys
