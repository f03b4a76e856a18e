"""Seeded synthetic workloads with the shapes of the reference's datasets.

The reference reads YCSB / Wikipedia / Ethereum dumps from absent files
(mpt-with-compress/include/bench/ycsb.cuh:17, wiki.cuh:19, ethtxn.cuh:17);
these generators stand in for them with fixed seeds so every run (CPU oracle,
GPU path, bench) sees the same bytes.

Batch layout is the reference's: hex-nibble keys (one byte per nibble, 16 =
terminator, util/utils.cuh:340-349) with inclusive ``[start, end]`` int32
index pairs, raw value bytes with inclusive int64 index pairs
(util/utils.cuh:254-301).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _rotl(x, k):
    k = np.uint64(k)
    return (x << k) | (x >> (np.uint64(64) - k))


def _splitmix64(x):
    x = x + np.uint64(0x9E3779B97F4A7C15)
    z = x
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x, z ^ (z >> np.uint64(31))


class Xoshiro256ss:
    """xoshiro256** (Blackman & Vigna) run as ``lanes`` independent streams
    seeded by splitmix64; output word t*lanes + l comes from lane l, step t."""

    def __init__(self, seed: int, lanes: int = 1 << 16):
        with np.errstate(over="ignore"):
            x = np.uint64(seed) + np.arange(lanes, dtype=np.uint64) * np.uint64(0x632BE59BD9B4E019)
            s = []
            for _ in range(4):
                x, z = _splitmix64(x)
                s.append(z)
        self.s = s
        self.lanes = lanes

    def words(self, n: int) -> np.ndarray:
        steps = (n + self.lanes - 1) // self.lanes
        out = np.empty((steps, self.lanes), dtype=np.uint64)
        s0, s1, s2, s3 = self.s
        with np.errstate(over="ignore"):
            for t in range(steps):
                out[t] = _rotl(s1 * np.uint64(5), 7) * np.uint64(9)
                tt = s1 << np.uint64(17)
                s2 ^= s0
                s3 ^= s1
                s1 ^= s2
                s0 ^= s3
                s2 ^= tt
                s3 = _rotl(s3, 45)
        self.s = [s0, s1, s2, s3]
        return out.reshape(-1)[:n]

    def bytes(self, n: int) -> np.ndarray:
        return self.words((n + 7) // 8).view(np.uint8)[:n].copy()

    def uniform(self, n: int) -> np.ndarray:
        return (self.words(n) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))

    def normal(self, n: int) -> np.ndarray:
        u1 = np.maximum(self.uniform(n), 1e-300)
        u2 = self.uniform(n)
        return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def fnv1a64(ids: np.ndarray) -> np.ndarray:
    """FNV-1a 64 over the 8 little-endian bytes of each id (YCSB FNVhash64)."""
    h = np.full(ids.shape, 0xCBF29CE484222325, dtype=np.uint64)
    v = ids.astype(np.uint64)
    with np.errstate(over="ignore"):
        for _ in range(8):
            h ^= v & np.uint64(0xFF)
            h *= np.uint64(1099511628211)
            v >>= np.uint64(8)
    return h


@dataclass
class Batch:
    """One put batch in the reference's flat layout."""

    keys_hexs: np.ndarray      # uint8 nibbles, 16 = terminator
    keys_indexs: np.ndarray    # int32 [2n] inclusive pairs
    values: np.ndarray         # uint8
    values_indexs: np.ndarray  # int64 [2n] inclusive pairs

    @property
    def n(self) -> int:
        return len(self.keys_indexs) // 2

    def key(self, i: int) -> bytes:
        return self.keys_hexs[self.keys_indexs[2 * i]: self.keys_indexs[2 * i + 1] + 1].tobytes()

    def value(self, i: int) -> bytes:
        return self.values[self.values_indexs[2 * i]: self.values_indexs[2 * i + 1] + 1].tobytes()

    def subset(self, idx) -> "Batch":
        idx = np.asarray(idx, dtype=np.int64)
        kh, ki = _gather_flat(self.keys_hexs, self.keys_indexs.astype(np.int64), idx)
        vb, vi = _gather_flat(self.values, self.values_indexs, idx)
        return Batch(kh, ki.astype(np.int32), vb, vi)

    def key_bytes(self) -> int:
        return int(self.keys_indexs[-1]) + 1 if self.n else 0

    def value_bytes(self) -> int:
        return int(self.values_indexs[-1]) + 1 if self.n else 0


def _gather_flat(flat, pairs, idx):
    starts = pairs[0::2][idx]
    lens = pairs[1::2][idx] - starts + 1
    offs = np.zeros(len(idx) + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    total = int(offs[-1])
    src = np.repeat(starts - offs[:-1], lens) + np.arange(total, dtype=np.int64)
    out = flat[src]
    new_pairs = np.empty(2 * len(idx), dtype=np.int64)
    new_pairs[0::2] = offs[:-1]
    new_pairs[1::2] = offs[1:] - 1
    return out, new_pairs


def keys_to_hexs(key_bytes: np.ndarray, key_lens: np.ndarray):
    """Flat key bytes + lengths -> (keys_hexs, keys_indexs) with terminators
    (util/utils.cuh:340-349 applied per key)."""
    key_lens = key_lens.astype(np.int64)
    n = len(key_lens)
    if n and np.all(key_lens == key_lens[0]):
        # fixed length: one (n, 2L+1) array, nibbles interleaved + terminator
        L = int(key_lens[0])
        kb = np.asarray(key_bytes, dtype=np.uint8).reshape(n, L)
        rows = np.empty((n, 2 * L + 1), dtype=np.uint8)
        rows[:, 0:2 * L:2] = kb >> 4
        rows[:, 1:2 * L:2] = kb & 15
        rows[:, 2 * L] = 16
        if n * (2 * L + 1) >= 2 ** 31:
            raise ValueError("key stream exceeds the int32 index range")
        starts = np.arange(n, dtype=np.int64) * (2 * L + 1)
        idx = np.empty(2 * n, dtype=np.int32)
        idx[0::2] = starts
        idx[1::2] = starts + 2 * L
        return rows.reshape(-1), idx
    hex_lens = 2 * key_lens + 1
    hoffs = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(hex_lens, out=hoffs[1:])
    out = np.empty(int(hoffs[-1]), dtype=np.uint8)
    boffs = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(key_lens, out=boffs[1:])
    # position of every key byte in the hex stream
    kid = np.repeat(np.arange(n, dtype=np.int64), key_lens)
    within = np.arange(len(key_bytes), dtype=np.int64) - boffs[kid]
    pos = hoffs[kid] + 2 * within
    out[pos] = key_bytes >> 4
    out[pos + 1] = key_bytes & 15
    out[hoffs[1:] - 1] = 16
    idx = np.empty(2 * n, dtype=np.int64)
    idx[0::2] = hoffs[:-1]
    idx[1::2] = hoffs[1:] - 1
    if hoffs[-1] >= 2 ** 31:
        raise ValueError("key stream exceeds the int32 index range")
    return out, idx.astype(np.int32)


def hexs_to_keys(keys_hexs: np.ndarray, keys_indexs: np.ndarray):
    """Inverse of keys_to_hexs for terminated keys of whole bytes: (raw key
    bytes back to back, int32 inclusive byte pairs) for gmpt_puts_raw."""
    ki = np.asarray(keys_indexs, dtype=np.int64).reshape(-1, 2)
    n = len(ki)
    nib = ki[:, 1] - ki[:, 0]  # nibbles before the terminator
    if n == 0:
        return np.zeros(0, dtype=np.uint8), np.zeros(0, dtype=np.int32)
    if np.any(nib % 2) or np.any(keys_hexs[ki[:, 1]] != 16):
        raise ValueError("keys must be whole bytes with a terminator")
    lens = nib // 2
    offs = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    kid = np.repeat(np.arange(n, dtype=np.int64), lens)
    within = np.arange(int(offs[-1]), dtype=np.int64) - offs[kid]
    src = ki[kid, 0] + 2 * within
    kh = np.asarray(keys_hexs, dtype=np.uint8)
    out = ((kh[src] << 4) | kh[src + 1]).astype(np.uint8)
    idx = np.empty(2 * n, dtype=np.int32)
    idx[0::2] = offs[:-1]
    idx[1::2] = offs[1:] - 1
    return out, idx


def fixed_values(rng: Xoshiro256ss, n: int, size: int):
    vb = rng.bytes(n * size)
    vi = np.empty(2 * n, dtype=np.int64)
    starts = np.arange(n, dtype=np.int64) * size
    vi[0::2] = starts
    vi[1::2] = starts + size - 1
    return vb, vi


def var_values(rng: Xoshiro256ss, sizes: np.ndarray):
    sizes = sizes.astype(np.int64)
    offs = np.zeros(len(sizes) + 1, dtype=np.int64)
    np.cumsum(sizes, out=offs[1:])
    vb = rng.bytes(int(offs[-1]))
    vi = np.empty(2 * len(sizes), dtype=np.int64)
    vi[0::2] = offs[:-1]
    vi[1::2] = offs[1:] - 1
    return vb, vi


# --------------------------------------------------------------------------
# Workload shapes


def random_keys(n: int, key_bytes: int = 32, value_bytes: int = 64, seed: int = 0x5EED0001) -> Batch:
    """Uniformly random fixed-length keys and values (empty-trie bulk load)."""
    rng = Xoshiro256ss(seed)
    kb = rng.bytes(n * key_bytes)
    kh, ki = keys_to_hexs(kb, np.full(n, key_bytes, dtype=np.int64))
    vb, vi = fixed_values(rng, n, value_bytes)
    return Batch(kh, ki, vb, vi)


def ycsb_key_bytes(ids: np.ndarray) -> np.ndarray:
    """'user' + 19 decimal digits of FNV-1a-64(id) mod 10^19 (23 bytes each)."""
    h = fnv1a64(ids) % np.uint64(10 ** 19)
    n = len(ids)
    out = np.empty((n, 23), dtype=np.uint8)
    out[:, :4] = np.frombuffer(b"user", dtype=np.uint8)
    for d in range(18, -1, -1):
        out[:, 4 + d] = (h % np.uint64(10)).astype(np.uint8) + ord("0")
        h //= np.uint64(10)
    return out.reshape(-1)


def ycsb_load(n: int, value_bytes: int = 100, seed: int = 0x5EED0002) -> Batch:
    rng = Xoshiro256ss(seed)
    kb = ycsb_key_bytes(np.arange(n, dtype=np.uint64))
    kh, ki = keys_to_hexs(kb, np.full(n, 23, dtype=np.int64))
    vb, vi = fixed_values(rng, n, value_bytes)
    return Batch(kh, ki, vb, vi)


def zipf_from_uniform(u: np.ndarray, n_items: int, theta: float) -> np.ndarray:
    """Gray et al.'s zipfian generator (as in YCSB's ZipfianGenerator) on
    given uniforms in [0, 1)."""
    if theta <= 0.0:
        return (u * n_items).astype(np.int64).clip(0, n_items - 1)
    i = np.arange(1, n_items + 1, dtype=np.float64)
    zetan = float(np.sum(i ** -theta))
    zeta2 = 1.0 + 0.5 ** theta
    alpha = 1.0 / (1.0 - theta) if theta != 1.0 else 1e9
    eta = (1.0 - (2.0 / n_items) ** (1.0 - theta)) / (1.0 - zeta2 / zetan)
    uz = u * zetan
    r = (n_items * np.power(np.maximum(eta * u - eta + 1.0, 0.0), alpha)).astype(np.int64)
    r = np.where(uz < 1.0, 0, np.where(uz < 1.0 + 0.5 ** theta, 1, r))
    return np.clip(r, 0, n_items - 1)


def zipf_ranks(rng: Xoshiro256ss, n_items: int, n: int, theta: float) -> np.ndarray:
    """n zipfian ranks over n_items (zipf_from_uniform of the next n draws)."""
    return zipf_from_uniform(rng.uniform(n), n_items, theta)


def ycsb_zipf_updates(n_loaded: int, n: int, theta: float = 0.99, value_bytes: int = 100,
                      seed: int = 0x5EED0003) -> Batch:
    """Updates whose keys are drawn zipfian over the loaded ids, scrambled by
    FNV so the hot keys spread over the key space (YCSB ScrambledZipfian)."""
    rng = Xoshiro256ss(seed)
    ranks = zipf_ranks(rng, n_loaded, n, theta)
    ids = (fnv1a64(ranks.astype(np.uint64)) % np.uint64(n_loaded)).astype(np.uint64)
    kb = ycsb_key_bytes(ids)
    kh, ki = keys_to_hexs(kb, np.full(n, 23, dtype=np.int64))
    vb, vi = fixed_values(rng, n, value_bytes)
    return Batch(kh, ki, vb, vi)


def vocab_keys(n: int, seed: int = 0x5EED0004, vocab_size: int = 10000,
               mu: float = 3.0, sigma: float = 0.5, min_len: int = 8, max_len: int = 96,
               vmin: int = 128, vmax: int = 4096, vmu: float = 6.0, vsigma: float = 0.8) -> Batch:
    """Variable-length ASCII keys made of words from a seeded synthetic
    vocabulary (random lowercase strings), lognormal key and value sizes."""
    rng = Xoshiro256ss(seed)
    wl = 2 + (rng.words(vocab_size) % np.uint64(9)).astype(np.int64)         # 2..10 letters
    woff = np.zeros(vocab_size + 1, dtype=np.int64)
    np.cumsum(wl, out=woff[1:])
    letters = (rng.words(int(woff[-1])) % np.uint64(26)).astype(np.uint8) + ord("a")
    klen = np.clip(np.rint(np.exp(mu + sigma * rng.normal(n))), min_len, max_len).astype(np.int64)
    max_words = max_len // 2 + 1
    # word j of key i comes from uniform draw (i, j) of one block of n *
    # max_words draws; ranks are computed only for the words a key uses
    # (column by column while its length is not reached)
    u = rng.uniform(n * max_words).reshape(n, max_words)
    words = np.zeros((n, max_words), dtype=np.int64)
    wlen = np.zeros((n, max_words), dtype=np.int64)
    cum_all = np.zeros((n, max_words), dtype=np.int64)
    cum = np.zeros(n, dtype=np.int64)
    for j in range(max_words):
        rows = np.nonzero(cum < klen)[0]
        if len(rows) == 0:
            break
        words[rows, j] = zipf_from_uniform(u[rows, j], vocab_size, 0.8)
        wlen[rows, j] = wl[words[rows, j]]
        cum_all[rows, j] = cum[rows]
        cum[rows] += wlen[rows, j]
    # concatenate words, truncate to klen
    take = (cum_all < klen[:, None]) & (wlen > 0)            # words that contribute
    piece = np.minimum(wlen, klen[:, None] - cum_all) * take  # bytes taken from each word
    flat_piece = piece.reshape(-1)
    flat_word = words.reshape(-1)
    total = int(flat_piece.sum())
    src_start = np.repeat(woff[flat_word], flat_piece)
    pstart = np.zeros(len(flat_piece) + 1, dtype=np.int64)
    np.cumsum(flat_piece, out=pstart[1:])
    within = np.arange(total, dtype=np.int64) - np.repeat(pstart[:-1], flat_piece)
    kb = letters[src_start + within]
    kh, ki = keys_to_hexs(kb, klen)
    vsz = np.clip(np.rint(np.exp(vmu + vsigma * rng.normal(n))), vmin, vmax).astype(np.int64)
    vb, vi = var_values(rng, vsz)
    return Batch(kh, ki, vb, vi)


def sample_indices(n: int, count: int, seed: int = 0x5EED00FF) -> np.ndarray:
    rng = Xoshiro256ss(seed, lanes=1024)
    return (rng.words(count) % np.uint64(max(n, 1))).astype(np.int64)
