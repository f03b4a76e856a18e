"""Ethereum-shaped forest workload: a state trie of accounts plus one storage
trie per account, updated block by block.

Shapes (seeded, synthetic; stand-ins for mainnet data the reference reads
from absent dumps, mpt-with-compress/include/bench/ethtxn.cuh:17):

* state trie (trie 0): key = Keccak-256(random 20-byte address), value = RLP
  list [nonce, balance, storageRoot, codeHash] of 71..110 bytes;
* a block updates U[150, 400] distinct accounts; each touched account's
  storage trie (its own trie id, kept across blocks) receives a power-law
  number of entries, p(s) ~ s^-alpha on [1, 5000] with alpha = 1.5, keys =
  Keccak-256 of a 32-byte slot number, values 1..32 random bytes;
* the account's new value carries its storage trie's new root as
  storageRoot, so storage tries are hashed before the state trie.

Three ways to apply a block, all giving the same roots:

* ``apply_plain``      one insert + one hash + one root read per trie (what a
                       one-trie-per-object API such as the reference's
                       GpuMPT::Compress::MPT allows), storage roots patched
                       into the account values on the host;
* ``apply_forest``     one forest insert + hash for all storage tries, roots
                       read back, patched on the host, then the state trie;
* ``apply_block``      one persistent graph-replayed launch (gmpt_block_update).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import workloads as W

# Keccak-256 of RLP("") (0x80): the root of an empty trie in go-ethereum
EMPTY_ROOT = bytes.fromhex("56e81f171bcc55a6ff8345e692c0f86e5b48e01b996cadc001622fb5e363b421")

MAX_ACCOUNT_BYTES = 110


def _rlp_uint_bytes(rng: W.Xoshiro256ss, n: int, max_len: int, min_len: int):
    """Random big-endian integers of min_len..max_len bytes, RLP-ready: a
    nonzero leading byte, and >= 0x80 when one byte long (so the encoding is
    always 0x80+len followed by the bytes)."""
    lens = min_len + (rng.words(n) % np.uint64(max_len - min_len + 1)).astype(np.int64)
    raw = rng.bytes(n * max_len).reshape(n, max_len)
    lead = raw[:, 0].copy()
    lead = np.where(lens == 1, lead | 0x80, np.where(lead == 0, 1, lead)).astype(np.uint8)
    raw[:, 0] = lead
    return lens, raw


def account_values(rng: W.Xoshiro256ss, n: int, storage_roots: np.ndarray | None = None):
    """RLP accounts [nonce, balance, storageRoot, codeHash].

    Returns (values, values_indexs, root_off): root_off[i] is the byte offset
    of storageRoot inside value i (always len - 65).  Every field sits at its
    largest offset in a 110-column row and one mask keeps the bytes in use,
    so the row-major compaction is the concatenated encodings."""
    ln, nb = _rlp_uint_bytes(rng, n, 8, 0)
    lb, bb = _rlp_uint_bytes(rng, n, 32, 1)
    code = rng.bytes(32 * n).reshape(n, 32)
    if storage_roots is None:
        storage_roots = np.tile(np.frombuffer(EMPTY_ROOT, np.uint8), (n, 1))
    total = 70 + ln + lb
    arr = np.empty((n, MAX_ACCOUNT_BYTES), dtype=np.uint8)
    arr[:, 0] = 0xF8
    arr[:, 1] = (total - 2).astype(np.uint8)
    arr[:, 2] = (0x80 + ln).astype(np.uint8)
    arr[:, 3:11] = nb
    arr[:, 11] = (0x80 + lb).astype(np.uint8)
    arr[:, 12:44] = bb
    arr[:, 44] = 0xA0
    arr[:, 45:77] = storage_roots
    arr[:, 77] = 0xA0
    arr[:, 78:110] = code
    col = np.arange(MAX_ACCOUNT_BYTES)
    mask = np.ones((n, MAX_ACCOUNT_BYTES), dtype=bool)
    mask[:, 3:11] = col[None, 3:11] - 3 < ln[:, None]
    mask[:, 12:44] = col[None, 12:44] - 12 < lb[:, None]
    vb = arr[mask]
    offs = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(total, out=offs[1:])
    vi = np.empty(2 * n, dtype=np.int64)
    vi[0::2] = offs[:-1]
    vi[1::2] = offs[1:] - 1
    return vb, vi, (total - 65).astype(np.int32)


def power_law_sizes(rng: W.Xoshiro256ss, n: int, alpha: float = 1.5, lo: int = 1, hi: int = 5000) -> np.ndarray:
    """Integer sizes with density ~ s^-alpha on [lo, hi] (inverse CDF)."""
    u = rng.uniform(n)
    a = 1.0 - alpha
    x = (u * (hi ** a - lo ** a) + lo ** a) ** (1.0 / a)
    return np.clip(np.floor(x).astype(np.int64), lo, hi)


@dataclass
class EthState:
    n_accounts: int
    keys: np.ndarray          # [n, 32] state keys (Keccak of the addresses)
    batch: W.Batch            # the initial state trie batch


def make_state(n_accounts: int, keccak_rows, seed: int = 0x5EED0C40, chunk: int = 1 << 21) -> EthState:
    """The pre-existing state trie: n accounts with empty storage."""
    rng = W.Xoshiro256ss(seed)
    keys = np.empty((n_accounts, 32), dtype=np.uint8)
    vbs, vis, vbase = [], [], 0
    for a in range(0, n_accounts, chunk):
        k = min(chunk, n_accounts - a)
        keys[a: a + k] = keccak_rows(rng.bytes(20 * k).reshape(k, 20))
        vb, vi, _ = account_values(rng, k)
        vbs.append(vb)
        vis.append(vi + vbase)
        vbase += len(vb)
    kh, ki = W.keys_to_hexs(keys.reshape(-1), np.full(n_accounts, 32, dtype=np.int64))
    return EthState(n_accounts, keys, W.Batch(kh, ki, np.concatenate(vbs), np.concatenate(vis)))


@dataclass
class EthBlock:
    """One block in the gmpt_block_update layout: storage keys (stage 0)
    followed by the account keys (stage 1)."""

    batch: W.Batch
    trie_ids: np.ndarray      # int32 [n]
    patch_trie: np.ndarray    # int32 [n], -1 for storage keys
    patch_off: np.ndarray     # int32 [n]
    n0: int
    accounts: np.ndarray      # int64 [m] touched accounts
    storage_ids: np.ndarray   # int32 [m] their storage tries
    spans: np.ndarray         # int64 [m + 1] storage key ranges per account

    @property
    def n(self) -> int:
        return self.batch.n

    @property
    def out_ids(self) -> np.ndarray:
        return np.concatenate([[0], self.storage_ids]).astype(np.int32)


@dataclass
class EthBlocks:
    """Block generator; storage trie ids persist across blocks."""

    state: EthState
    keccak_rows: object
    seed: int = 0x5EED0C41
    min_updates: int = 150
    max_updates: int = 400
    alpha: float = 1.5
    max_storage: int = 5000
    sid_of: dict = field(default_factory=dict)
    next_sid: int = 1

    def __post_init__(self):
        self.rng = W.Xoshiro256ss(self.seed)

    def next(self) -> EthBlock:
        rng = self.rng
        want = self.min_updates + int(rng.words(1)[0] % np.uint64(self.max_updates - self.min_updates + 1))
        acc = np.unique((rng.words(2 * want) % np.uint64(self.state.n_accounts)).astype(np.int64))[:want]
        m = len(acc)
        sids = np.empty(m, dtype=np.int32)
        for j, a in enumerate(acc.tolist()):
            sid = self.sid_of.get(a)
            if sid is None:
                sid = self.next_sid
                self.sid_of[a] = sid
                self.next_sid += 1
            sids[j] = sid
        sizes = power_law_sizes(rng, m, self.alpha, 1, self.max_storage)
        spans = np.zeros(m + 1, dtype=np.int64)
        np.cumsum(sizes, out=spans[1:])
        ns = int(spans[-1])
        # storage slot keys: Keccak-256 of 32-byte big-endian slot numbers
        slot_msgs = np.zeros((ns, 32), dtype=np.uint8)
        slot_msgs[:, 24:] = rng.bytes(8 * ns).reshape(ns, 8)
        skeys = self.keccak_rows(slot_msgs)
        svb, svi = W.var_values(rng, 1 + (rng.words(ns) % np.uint64(32)).astype(np.int64))
        avb, avi, roff = account_values(rng, m, np.zeros((m, 32), dtype=np.uint8))
        akeys = self.state.keys[acc]
        kb = np.concatenate([skeys.reshape(-1), akeys.reshape(-1)])
        kh, ki = W.keys_to_hexs(kb, np.full(ns + m, 32, dtype=np.int64))
        vb = np.concatenate([svb, avb])
        vi = np.concatenate([svi, avi + len(svb)])
        tids = np.concatenate([np.repeat(sids, sizes), np.zeros(m, np.int32)]).astype(np.int32)
        ptrie = np.concatenate([np.full(ns, -1, np.int32), sids]).astype(np.int32)
        poff = np.concatenate([np.zeros(ns, np.int32), roff]).astype(np.int32)
        return EthBlock(W.Batch(kh, ki, vb, vi), tids, ptrie, poff, ns, acc, sids, spans)


def patched_values(blk: EthBlock, roots: dict) -> np.ndarray:
    """The block's value stream with each account's storageRoot filled in
    (roots: storage trie id -> root bytes, zero-padded to 32)."""
    vb = blk.batch.values.copy()
    vi = blk.batch.values_indexs
    for j in range(blk.n0, blk.n):
        t = int(blk.patch_trie[j])
        if t < 0:
            continue
        r = roots[t][:32].ljust(32, b"\0")
        at = int(vi[2 * j]) + int(blk.patch_off[j])
        vb[at: at + 32] = np.frombuffer(r, np.uint8)
    return vb


def apply_plain(mpt, blk: EthBlock) -> list:
    """One insert + hash + root read per trie (latching inserts)."""
    b = blk.batch
    roots = {}
    for j, sid in enumerate(blk.storage_ids.tolist()):
        a, z = int(blk.spans[j]), int(blk.spans[j + 1])
        sub = b.subset(np.arange(a, z))
        mpt.puts_forest(False, sub.keys_hexs, sub.keys_indexs, sub.values, sub.values_indexs,
                        np.full(z - a, sid, np.int32))
        mpt.hash_onepass_v2()
        roots[sid] = mpt.get_roots([sid])[0]
    vb = patched_values(blk, roots)
    acc = W.Batch(b.keys_hexs, b.keys_indexs, vb, b.values_indexs).subset(np.arange(blk.n0, blk.n))
    mpt.puts_latching_with_valuehp_v2(acc.keys_hexs, acc.keys_indexs, acc.values, acc.values_indexs)
    mpt.hash_onepass_v2()
    return [mpt.get_roots([0])[0]] + [roots[s] for s in blk.storage_ids.tolist()]


def apply_forest(mpt, blk: EthBlock, two_phase: bool = False) -> list:
    """All storage tries in one forest insert + hash, then the state trie."""
    b = blk.batch
    st = b.subset(np.arange(0, blk.n0))
    mpt.puts_forest(two_phase, st.keys_hexs, st.keys_indexs, st.values, st.values_indexs, blk.trie_ids[: blk.n0])
    mpt.hash_onepass_v2()
    sroots = mpt.get_roots(blk.storage_ids)
    roots = dict(zip(blk.storage_ids.tolist(), sroots))
    vb = patched_values(blk, roots)
    acc = W.Batch(b.keys_hexs, b.keys_indexs, vb, b.values_indexs).subset(np.arange(blk.n0, blk.n))
    mpt.puts_forest(two_phase, acc.keys_hexs, acc.keys_indexs, acc.values, acc.values_indexs,
                    np.zeros(blk.n - blk.n0, np.int32))
    mpt.hash_onepass_v2()
    return [mpt.get_roots([0])[0]] + sroots


def apply_block(mpt, blk: EthBlock) -> list:
    """One persistent launch for the whole block."""
    b = blk.batch
    return mpt.block_update(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, blk.trie_ids, blk.n0,
                            blk.out_ids, blk.patch_trie, blk.patch_off)
